"""Parity on the reference's own example tensors (data/tensors/*.tns of the
reference tree; the file bytes and the reference library's results for them
are committed as tests/golden/data_*.npz by make_data_golden.py).

CPU: the oracle reproduces the reference's ptiMTTKRP, ptiSparseTensorToHiCOO
and ptiMTTKRPHiCOO outputs on them bit for bit.  GPU: the GPU loader returns
exactly what the reference's ptiLoadSparseTensor returned for the same bytes
(including the headerless example, which the reference reads as an empty
3-D tensor), the GPU conversion gives the reference's HiCOO arrays, and the
GPU MTTKRPs agree with the reference's outputs (normwise 1e-5)."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from hiparti_b200 import COOTensor, HiCOOTensor

FILES = ["data_3d_7.npz", "data_3d_24.npz", "data_3d_dense.npz", "data_3D_12031.npz", "data_4d_3_16.npz"]
MTTKRP_FILES = FILES[:4]


def _tensor(g):
    dims = [int(x) for x in g["dims"]]
    return dims, [g[f"ind{m}"] for m in range(len(dims))], g["vals"]


def test_fixture_set_is_complete():
    loaded = {f: int(load_golden(f)["load_rc"]) for f in FILES}
    assert all(rc == 0 for rc in loaded.values()), loaded
    for f in MTTKRP_FILES:
        assert "coo_out0" in load_golden(f), f
    g = load_golden("data_4d_3_16.npz")
    assert g["vals"].size == 0 and list(g["dims"]) == [3, 2, 2]


@pytest.mark.parametrize("case", MTTKRP_FILES)
def test_orc_matches_reference_on_examples(orc, case):
    g = load_golden(case)
    dims, inds, vals = _tensor(g)
    R = int(g["R"])
    mats = [g[f"mat{m}"] for m in range(3)]
    for m in range(3):
        np.testing.assert_array_equal(orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]], g[f"coo_out{m}"])
    h = orc.hicoo_build(dims, inds, vals, int(g["sb"]), int(g["sk"]), int(g["sc"]))
    for key in ["bptr", "vals", "kptr", "cptr"]:
        np.testing.assert_array_equal(h[key], g[f"h_{key}"], err_msg=key)
    for m in range(3):
        np.testing.assert_array_equal(h["binds"][m], g[f"h_binds{m}"])
        np.testing.assert_array_equal(h["einds"][m], g[f"h_einds{m}"])
        np.testing.assert_array_equal(orc.mttkrp_hicoo(h, mats, R, m)[: dims[m]], g[f"hicoo_out{m}"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", FILES)
def test_gpu_loader_matches_reference_on_examples(lib, cuda, tmp_path, case):
    g = load_golden(case)
    path = tmp_path / case.replace(".npz", ".tns")
    path.write_bytes(g["file_bytes"].tobytes())
    t = COOTensor.load(str(path), 1)
    dims, inds, vals = _tensor(g)
    assert list(t.dims) == dims
    assert t.vals.size == vals.size
    for a, b in zip(t.inds, inds):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(t.vals.view(np.uint32), vals.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("case", MTTKRP_FILES)
def test_gpu_conversion_and_mttkrp_match_reference_on_examples(lib, cuda, case):
    g = load_golden(case)
    dims, inds, vals = _tensor(g)
    R = int(g["R"])
    mats = [g[f"mat{m}"] for m in range(3)]
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    for m in range(3):
        assert rel_err(coo.mttkrp(mats, R, m)[: dims[m]], g[f"coo_out{m}"]) < 1e-5
    h = coo.to_hicoo(int(g["sb"]), int(g["sk"]), int(g["sc"]))
    np.testing.assert_array_equal(h.bptr, g["h_bptr"])
    np.testing.assert_array_equal(h.vals.view(np.uint32), g["h_vals"].view(np.uint32))
    np.testing.assert_array_equal(h.kptr, g["h_kptr"])
    np.testing.assert_array_equal(h.cptr, g["h_cptr"])
    for m in range(3):
        np.testing.assert_array_equal(h.binds[m], g[f"h_binds{m}"])
        np.testing.assert_array_equal(h.einds[m], g[f"h_einds{m}"])
    hr = HiCOOTensor(dims, g["sb"], g["sk"], g["sc"], g["h_bptr"], [g[f"h_binds{m}"] for m in range(3)],
                     [g[f"h_einds{m}"] for m in range(3)], g["h_vals"], kptr=g["h_kptr"])
    for m in range(3):
        for variant in ["seq", "cuda"]:
            assert rel_err(hr.mttkrp(mats, R, m, variant)[: dims[m]], g[f"hicoo_out{m}"]) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("case", MTTKRP_FILES)
def test_gpu_ttm_matches_reference_on_examples(lib, cuda, ref, case):
    """ptiSparseTensorMulMatrix of the compiled reference on its example
    tensors, every mode: fibers, coordinates and FP32 values bit for bit."""
    g = load_golden(case)
    dims, inds, vals = _tensor(g)
    rng = np.random.default_rng(len(case))
    for mode in range(3):
        U = rng.standard_normal((dims[mode], 8)).astype(np.float32)
        finds, yv, (xinds, xvals, xso) = ref.ttm(dims, inds, vals, U, mode)
        coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
        ours = coo.ttm(U, mode)
        for a, b in zip(ours["inds"], finds):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(ours["vals"].view(np.uint32), yv.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["coo", "hicoo"])
def test_gpu_cpd_on_example_tensor(lib, cuda, orc, fmt):
    """CPD-ALS of the 12031-nonzero example tensor (integer values 1..14),
    R = 8, 10 iterations from seeded factors: every fit within 1e-4 of the
    FP64 oracle's, and the final fit equal to the model's fit evaluated at
    the nonzeros."""
    from test_cpd_gpu import _device_cpd
    g = load_golden("data_3D_12031.npz")
    dims, inds, vals = _tensor(g)
    R, iters = 8, 10
    rng = np.random.default_rng(12031)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    lam, facs, fits = _device_cpd(dims, inds, vals, init, iters, fmt=fmt)
    o = orc.cpd_als(dims, inds, vals, R, iters, init)
    np.testing.assert_allclose(fits, o["fits"], atol=1e-4)
    direct = orc.kruskal_fit(dims, inds, vals, lam.astype(np.float64), [f.astype(np.float64) for f in facs])
    assert abs(direct - fits[-1]) < 1e-4
