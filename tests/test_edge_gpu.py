"""Edge cases of the paths around MTTKRP on the GPU: empty tensors through
TTM/TTV, renumbering and the loader; a mode of size one; the largest
supported TTM rank."""
import numpy as np
import pytest

from hiparti_b200 import COOTensor, DeviceTensor, PtiError

pytestmark = pytest.mark.gpu


def _empty(dims):
    return COOTensor(dims, [np.empty(0, np.uint32) for _ in dims], np.empty(0, np.float32))


def test_empty_tensor_ttm_ttv(lib, cuda, ref):
    dims = (5, 6, 7)
    U = np.ones((7, 4), np.float32)
    Y = _empty(dims).ttm(U, 2)
    assert Y["vals"].shape == (0, 8) and all(i.size == 0 for i in Y["inds"])
    Yv = _empty(dims).ttv(np.ones(6, np.float32), 1)
    assert Yv["vals"].shape == (0, 8)
    assert COOTensor.from_semi_sparse(Y).nnz == 0


def test_empty_tensor_renumber(lib, cuda):
    maps = _empty((4, 3, 5)).renumber(2)
    for d, m in zip((4, 3, 5), maps):
        np.testing.assert_array_equal(m, np.arange(d, dtype=np.uint32))


def test_empty_and_header_only_files(lib, cuda, ref, tmp_path):
    for name, text in [("empty.tns", ""), ("hdr.tns", "3\n4 5 6\n"), ("one.tns", "3\n4 5 6\n1 2 3 4.5")]:
        p = tmp_path / name
        p.write_text(text)
        rc, dims, inds, vals = ref.load(p, 1)
        if rc != 0:
            with pytest.raises(PtiError):
                COOTensor.load(str(p))
            continue
        t = COOTensor.load(str(p))
        assert t.dims == [int(d) for d in dims] and t.nnz == vals.size
        np.testing.assert_array_equal(t.vals, vals)


def test_mode_of_size_one(lib, cuda, ref):
    dims = (40, 1, 30)
    rng = np.random.default_rng(3)
    lin = rng.choice(40 * 30, 500, replace=False)
    i0, i2 = np.unravel_index(lin, (40, 30))
    inds = [i0.astype(np.uint32), np.zeros(500, np.uint32), i2.astype(np.uint32)]
    vals = rng.random(500).astype(np.float32)
    U = rng.random((1, 16)).astype(np.float32)
    finds, yv, _ = ref.ttm(dims, inds, vals, U, 1)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    ours = coo.ttm(U, 1)
    np.testing.assert_array_equal(ours["vals"].view(np.uint32), yv.view(np.uint32))
    maps = COOTensor(dims, inds, vals).renumber(1)
    np.testing.assert_array_equal(maps[1], [0])


def test_ttm_largest_rank(lib, cuda, ref):
    dims = (30, 20, 10)
    rng = np.random.default_rng(4)
    lin = rng.choice(6000, 2000, replace=False)
    inds = [i.astype(np.uint32) for i in np.unravel_index(lin, dims)]
    vals = rng.standard_normal(2000).astype(np.float32)
    U = rng.standard_normal((10, 256)).astype(np.float32)
    finds, yv, _ = ref.ttm(dims, inds, vals, U, 2)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    np.testing.assert_array_equal(coo.ttm(U, 2)["vals"].view(np.uint32), yv.view(np.uint32))
    with pytest.raises(PtiError):
        COOTensor(dims, [i.copy() for i in inds], vals.copy()).ttm(np.ones((10, 257), np.float32), 2)
