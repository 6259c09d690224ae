"""GPU CPD-ALS against the FP64 oracle (a restatement of src/sptensor/cpd.c in
double precision) and the reference library.  Tolerance: fit within 1e-4 of
the FP64 oracle; factors and lambda within relative 1e-4 after a few
iterations from the same start."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from hiparti_b200 import COOTensor, DeviceTensor, HiCOOTensor, synth

pytestmark = pytest.mark.gpu


def _device_cpd(dims, inds, vals, init, iters, fmt="coo", **kw):
    import torch
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    if fmt == "coo":
        dt = DeviceTensor.from_coo(coo)
    else:
        dt = DeviceTensor.from_hicoo(coo.to_hicoo(4, 6, 8))
    R = init[0].shape[1]
    stride = ((R - 1) // 8 + 1) * 8
    fac = []
    for a in init:
        t = torch.zeros((a.shape[0], stride), dtype=torch.float32)
        t[:, :R] = torch.from_numpy(a)
        fac.append(t.cuda())
    lam, fits = dt.cpd_als(fac, iters, rank=R, **kw)
    torch.cuda.synchronize()
    dt.free()
    return lam.cpu().numpy(), [f[:, :R].cpu().numpy() for f in fac], fits


def test_golden_cpd(lib, cuda, orc):
    g = load_golden("cpd3_planted.npz")
    dims = [int(x) for x in g["dims"]]
    inds = [g[f"ind{m}"] for m in range(3)]
    init = [g[f"init{m}"] for m in range(3)]
    R, iters = int(g["R"]), int(g["iters"])
    lam, facs, fits = _device_cpd(dims, inds, g["vals"], init, iters)
    for m in range(3):
        assert rel_err(facs[m], g[f"ref_factor{m}"]) < 1e-4
    assert rel_err(lam, g["ref_lambda"]) < 1e-4
    o = orc.cpd_als(dims, inds, g["vals"], R, iters, init)
    assert abs(fits[-1] - o["fit"]) < 1e-4
    np.testing.assert_allclose(fits, o["fits"], atol=1e-4)


@pytest.mark.parametrize("fmt", ["coo", "hicoo"])
@pytest.mark.parametrize("dims,R", [((200, 150, 100), 8), ((60, 50, 40, 30), 16), ((500, 400, 300), 32)])
def test_cpd_vs_oracle(lib, cuda, orc, fmt, dims, R):
    nnz = 30000
    inds, vals, _ = synth.planted_tensor(dims, nnz, 5, 0.01, seed=R)
    rng = np.random.default_rng(R + 1)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    iters = 10
    lam, facs, fits = _device_cpd(dims, inds, vals, init, iters, fmt=fmt)
    o = orc.cpd_als(dims, inds, vals, R, iters, init)
    assert abs(fits[-1] - o["fit"]) < 1e-4, (fits[-1], o["fit"])
    direct = orc.kruskal_fit(dims, inds, vals, lam.astype(np.float64), [f.astype(np.float64) for f in facs])
    assert abs(direct - fits[-1]) < 1e-4


def test_cpd_bf16_mixed(lib, cuda, orc):
    dims = (400, 300, 200)
    inds, vals, _ = synth.planted_tensor(dims, 50000, 6, 0.01, seed=3)
    R = 16
    rng = np.random.default_rng(4)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    iters = 20
    o = orc.cpd_als(dims, inds, vals, R, iters, init)
    lam, facs, fits = _device_cpd(dims, inds, vals, init, iters, precision="bf16", fp32_sweeps=2)
    assert abs(fits[-1] - o["fit"]) < 1e-4, (fits[-1], o["fit"])


def test_cpd_tol_stops_early(lib, cuda):
    dims = (100, 80, 60)
    inds, vals, _ = synth.planted_tensor(dims, 10000, 3, 0.0, seed=9)
    rng = np.random.default_rng(10)
    init = [np.abs(rng.standard_normal((d, 3))).astype(np.float32) for d in dims]
    lam, facs, fits = _device_cpd(dims, inds, vals, init, 200, tol=1e-6)
    assert 1 < len(fits) < 200
    assert abs(fits[-1] - fits[-2]) < 1e-6


def test_reference_entry_points_run(lib, cuda):
    """ptiCpdAls / ptiCudaCpdAls / ptiOmpCpdAls with the reference's i+j+1
    initial factors: the call succeeds and fills ktensor."""
    dims = (30, 20, 10)
    inds, vals = synth.uniform_tensor(dims, 2000, seed=1)
    coo = COOTensor(dims, inds, vals)
    for variant in ["seq", "cuda", "omp"]:
        res = coo.cpd_als(4, 3, variant=variant)
        assert [f.shape for f in res["factors"]] == [(d, 4) for d in dims]
        assert res["lambda_"].shape == (4,)


def test_cpd_bf16_on_a_low_rank_million_nonzero_tensor(lib, cuda, orc):
    """BF16 factors where the fit is far from 0: a 4-D tensor of exact CP rank
    5 (each component on 22 rows of every mode, 1.17M nonzeros) plus
    N(0, 0.05^2), R = 5, 30 iterations from one seeded start.  The FP64 oracle
    reaches a fit near 0.99; the BF16 run with two closing FP32 sweeps must end
    within 1e-4 of that fit with the same factors (factor match score >= 0.99,
    Acar et al.: best column pairing, product of cosines times the weight
    ratio)."""
    from bench import factor_match_score
    dims = (2000, 2000, 2000, 100)
    inds, vals, _ = synth.sparse_lowrank_tensor(dims, 5, 22, noise=0.05, seed=21)
    assert vals.size >= 1_000_000
    R, iters = 5, 30
    rng = np.random.default_rng(22)
    init = [rng.random((d, R)).astype(np.float32) for d in dims]
    o = orc.cpd_als(list(dims), inds, vals, R, iters, init)
    assert o["fit"] > 0.9
    for fmt in ("hicoo", "coo"):
        lam, facs, fits = _device_cpd(dims, inds, vals, init, iters, fmt=fmt, precision="bf16", fp32_sweeps=2)
        assert abs(fits[-1] - o["fit"]) < 1e-4, (fmt, fits[-1], o["fit"])
        assert factor_match_score(lam, facs, o["lambda_"], o["factors"]) >= 0.99
