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


# ---------------------------------------------------------------------------
# BFS-like (renumber == 2) and impl_num 2
# ---------------------------------------------------------------------------
def test_bfs_like_matches_golden_reference_vectors(lib, cuda):
    from test_renumber import _bfs_cases
    for dims, inds, vals, want in _bfs_cases():
        got = COOTensor(dims, inds, vals).renumber(method="bfs")
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dims,nnz,seed", [((300, 200, 100), 20000, 1), ((60, 50, 40, 30), 15000, 2),
                                           ((5000, 40, 30), 12000, 3)])
def test_bfs_like_matches_reference_and_oracle(lib, cuda, ref, dims, nnz, seed):
    from oracle.oracle import Ref, bfs_like
    from hiparti_b200 import synth
    inds, vals = synth.zipf_tensor(dims, nnz, s=1.1, seed=seed)
    got = COOTensor(dims, inds, vals).renumber(method="bfs")
    again = COOTensor(dims, [i.copy() for i in inds], vals.copy()).renumber(method="bfs")
    want = ref.bfs_like(list(dims), inds, vals) if Ref.bfs_available() else bfs_like(list(dims), inds)
    for a, b, c in zip(got, again, want):
        np.testing.assert_array_equal(a, b)  # deterministic
        np.testing.assert_array_equal(a, c)
        assert np.array_equal(np.sort(a), np.arange(a.size))


def test_bfs_like_edge_cases(lib, cuda):
    from oracle.oracle import bfs_like
    # empty tensor, a mode of size one, indices without nonzeros
    for dims, inds in [((4, 3, 2), [np.empty(0, np.uint32)] * 3),
                       ((9, 1, 5), [np.array([0, 3, 3, 8], np.uint32), np.zeros(4, np.uint32),
                                    np.array([4, 0, 2, 4], np.uint32)])]:
        vals = np.ones(inds[0].size, np.float32)
        got = COOTensor(dims, inds, vals).renumber(method="bfs")
        for a, b in zip(got, bfs_like(list(dims), inds)):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("dims,nnz,its", CASES)
def test_impl_num_2_matches_reference(lib, cuda, ref, dims, nnz, its):
    inds, vals = random_tensor(dims, nnz, 0)
    assert tie_free(dims, inds)
    got = COOTensor(dims, inds, vals).renumber(its, impl_num=2)
    want = ref.renumber(list(dims), inds, vals, its, impl_num=2)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
