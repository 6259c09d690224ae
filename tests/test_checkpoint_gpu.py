"""GPU tests of CPD-ALS checkpoint / resume (ptiB200CpdAlsCheckpoint).

A run stopped after k iterations and resumed from its checkpoint must follow
the uninterrupted run.  The restored fits are the stored ones bit for bit.  Two
runs differ only in the order of their FP32 atomic additions, so later fits
agree within 1e-5 and weights and factors within relative 1e-3 (FP32
factors).  With BF16 factor copies, such a last-bit difference can flip the
rounding of a BF16 element (2^-8 relative), which the climbing phase of ALS
amplifies, so there the converged fits (the last ten) are compared within
1e-4, and weights and factors within 1e-2.  The FP32 runs also stay within 1e-4 of the FP64 oracle's fit.  The test
tensor has exact CP rank R, so ALS converges and the factors are determined."""
import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import COOTensor, DeviceTensor, PtiError, load_cpd_checkpoint, synth

pytestmark = pytest.mark.gpu

DIMS = (300, 200, 150)
R = 8


@pytest.fixture(scope="module")
def problem():
    inds, vals, _ = synth.sparse_lowrank_tensor(DIMS, R, 20, noise=0.05, seed=11)
    rng = np.random.default_rng(12)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in DIMS]
    return inds, vals, init


def _device(inds, vals, fmt):
    coo = COOTensor(DIMS, [i.copy() for i in inds], vals.copy())
    return DeviceTensor.from_coo(coo) if fmt == "coo" else DeviceTensor.from_hicoo(coo.to_hicoo(4, 6, 8))


def _factors(init, scale=1.0):
    import torch
    stride = ((R - 1) // 8 + 1) * 8
    out = []
    for a in init:
        t = torch.zeros((a.shape[0], stride), dtype=torch.float32)
        t[:, :R] = torch.from_numpy(a) * scale
        out.append(t.cuda())
    return out


def _run(dt, init, iters, scale=1.0, **kw):
    import torch
    fac = _factors(init, scale)
    lam, fits = dt.cpd_als(fac, iters, rank=R, **kw)
    torch.cuda.synchronize()
    return lam.cpu().numpy(), [f[:, :R].cpu().numpy() for f in fac], fits


@pytest.mark.parametrize("fmt", ["coo", "hicoo"])
@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_resume_follows_uninterrupted_run(lib, cuda, orc, tmp_path, problem, fmt, precision):
    inds, vals, init = problem
    total, stop = 30, 7
    dt = _device(inds, vals, fmt)
    # No closing FP32 sweeps: the stopped run must take the same BF16/FP32
    # schedule as the first `stop` iterations of the whole run.
    kw = dict(precision=precision, fp32_sweeps=0)
    lam_a, fac_a, fits_a = _run(dt, init, total, **kw)

    ck = tmp_path / "cpd.ckpt"
    lam_b, fac_b, fits_b = _run(dt, init, stop, checkpoint=ck, checkpoint_every=5, **kw)
    assert len(fits_b) == stop
    # The checkpoint holds the state after the last iteration, finished as
    # the loop finishes its result.
    saved = load_cpd_checkpoint(ck)
    assert saved["iters"] == stop and saved["fit"] == fits_b[-1]
    assert rel_err(saved["lambda_"], lam_b) < 1e-5
    for a, b in zip(saved["factors"], fac_b):
        assert rel_err(a, b) < 1e-5

    # Resume from garbage initial factors: the checkpoint replaces them.
    lam_c, fac_c, fits_c = _run(dt, init, total, scale=-7.0, checkpoint=ck, checkpoint_every=5, resume=True,
                                **kw)
    dt.free()
    assert len(fits_c) == total
    assert fits_c[:stop] == fits_b
    if precision == "fp32":
        fit_tol, fac_tol = 1e-5, 1e-3
        np.testing.assert_allclose(fits_c, fits_a, atol=fit_tol, rtol=0)
    else:
        # Mid-trajectory, two BF16 runs drift apart by up to a few 1e-3 in
        # fit (a flipped BF16 rounding is amplified while the fit climbs);
        # they meet again once ALS has converged.
        fit_tol, fac_tol = 1e-4, 1e-2
        np.testing.assert_allclose(fits_c[-10:], fits_a[-10:], atol=fit_tol, rtol=0)
    assert fits_a[-1] > 0.98  # BF16-only iterations reach about 0.99
    assert rel_err(lam_c, lam_a) < fac_tol
    for a, c in zip(fac_a, fac_c):
        assert rel_err(c, a) < fac_tol
    if precision == "fp32":
        o = orc.cpd_als(list(DIMS), inds, vals, R, total, init)
        assert abs(fits_c[-1] - o["fit"]) < 1e-4
    assert load_cpd_checkpoint(ck)["iters"] == total


def test_resume_without_file_starts_fresh(lib, cuda, tmp_path, problem):
    inds, vals, init = problem
    dt = _device(inds, vals, "coo")
    _, _, fits_a = _run(dt, init, 6)
    ck = tmp_path / "new.ckpt"
    _, _, fits_b = _run(dt, init, 6, checkpoint=ck, resume=True)
    dt.free()
    np.testing.assert_allclose(fits_b, fits_a, atol=1e-6, rtol=0)
    assert load_cpd_checkpoint(ck)["iters"] == 6


def test_converged_run_is_not_iterated_again(lib, cuda, tmp_path):
    dims = (100, 80, 60)
    inds, vals, _ = synth.planted_tensor(dims, 10000, 3, 0.0, seed=9)
    rng = np.random.default_rng(10)
    init = [np.abs(rng.standard_normal((d, 3))).astype(np.float32) for d in dims]
    import torch
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    dt = DeviceTensor.from_coo(coo)
    ck = tmp_path / "tol.ckpt"
    facs = [torch.from_numpy(np.pad(a, ((0, 0), (0, 5)))).cuda() for a in init]
    _, fits = dt.cpd_als(facs, 200, tol=1e-4, rank=3, checkpoint=ck)
    assert len(fits) < 200
    facs2 = [torch.zeros_like(f) for f in facs]
    lam2, fits2 = dt.cpd_als(facs2, 200, tol=1e-4, rank=3, checkpoint=ck, resume=True)
    torch.cuda.synchronize()
    dt.free()
    assert fits2 == fits
    assert float(lam2.abs().sum()) > 0


def test_resume_rejects_other_tensor_or_rank(lib, cuda, tmp_path, problem):
    inds, vals, init = problem
    ck = tmp_path / "x.ckpt"
    dt = _device(inds, vals, "coo")
    _run(dt, init, 4, checkpoint=ck)
    # more stored iterations than requested
    with pytest.raises(PtiError, match="more iterations"):
        _run(dt, init, 3, checkpoint=ck, resume=True)
    dt.free()
    # same shape and nonzero count, other values
    other = _device(inds, vals * 2.0, "coo")
    with pytest.raises(PtiError, match="another tensor"):
        _run(other, init, 8, checkpoint=ck, resume=True)
    other.free()
    # other rank
    import torch
    dt = _device(inds, vals, "coo")
    fac = [torch.zeros((d, 8), dtype=torch.float32, device=cuda) for d in DIMS]
    with pytest.raises(PtiError, match="shape or rank"):
        dt.cpd_als(fac, 8, rank=4, checkpoint=ck, resume=True)
    dt.free()
