"""GPU Lexi-order renumbering (ptiIndexRenumber / orderit / ptiB200Renumber)
against the reference's orderit (src/sptensor/orderit.c, compiled from its
sources) where the ordering is unique, and against the oracle's restatement
(equal row lists keep their current order) where it is not.  Exact."""
import numpy as np
import pytest

from hiparti_b200 import COOTensor, DeviceTensor
from test_renumber import CASES, random_tensor, tie_free

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,nnz,its", CASES)
@pytest.mark.parametrize("seed", [0, 1])
def test_matches_reference_orderit(lib, cuda, ref, dims, nnz, its, seed):
    inds, vals = random_tensor(dims, nnz, seed)
    assert tie_free(dims, inds)
    got = COOTensor(dims, inds, vals).renumber(its)
    want = ref.orderit(dims, inds, vals, its)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dims,nnz,its,seed", [((30, 40, 50), 200, 1, 0), ((30, 40, 50), 400, 3, 1),
                                               ((12, 200, 7, 9), 900, 2, 2), ((500, 3, 4), 700, 2, 3)])
def test_matches_oracle_with_equal_row_lists(lib, cuda, dims, nnz, its, seed):
    from oracle.oracle import lexi_order
    inds, vals = random_tensor(dims, nnz, seed)
    want = lexi_order(dims, inds, its)
    coo = COOTensor(dims, inds, vals)
    dt = DeviceTensor.from_coo(coo)
    got = dt.renumber(its, apply=True)
    new_inds, new_vals = dt.coo_arrays()
    dt.free()
    for m, (a, b) in enumerate(zip(got, want)):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(new_inds[m], a[inds[m]])  # the tensor was renumbered in place
    np.testing.assert_array_equal(new_vals, vals)


def test_renumbering_gathers_planted_blocks(lib, cuda):
    """Dense 8x8x8 blocks on the diagonal of a 256^3 tensor, indices then
    scrambled: Lexi-order brings each block's indices back together, so the
    HiCOO form with 8-wide blocks needs about one block per planted block."""
    rng = np.random.default_rng(5)
    nblk, w = 32, 8
    coords = []
    for b in range(nblk):
        g = np.stack(np.meshgrid(*[np.arange(w) + b * w] * 3, indexing="ij"), -1).reshape(-1, 3)
        coords.append(g)
    c = np.concatenate(coords)
    perms = [rng.permutation(nblk * w) for _ in range(3)]
    inds = [perms[m][c[:, m]].astype(np.uint32) for m in range(3)]
    vals = rng.random(c.shape[0]).astype(np.float32)
    dims = (nblk * w,) * 3
    before = DeviceTensor.from_coo(COOTensor(dims, inds, vals))
    h0 = before.to_hicoo(3, 6, 8)
    dt = DeviceTensor.from_coo(COOTensor(dims, inds, vals))
    dt.renumber(2, apply=True)
    h1 = dt.to_hicoo(3, 6, 8)
    nb0, nb1 = h0.nb, h1.nb
    for t in (before, h0, dt, h1):
        t.free()
    assert nb1 == nblk  # one HiCOO block per planted block
    assert nb0 > 8 * nblk
