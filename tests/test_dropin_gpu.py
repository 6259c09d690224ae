"""GPU: the drop-in proof.  tests/dropin/dropin_main.c is a C caller of the
reference's API compiled against the reference's own header (HiParTI.h, not
include/hiparti_b200.h) and linked against libhiparti_b200.so.  It loads a
.tns file, runs ptiMTTKRP, ptiSparseTensorToHiCOO, ptiMTTKRPHiCOO, the dense
ALS helpers, ptiCpdAls, CpdAlsStep and KruskalTensorFit, and writes every
result to disk; this test compares them with the reference library compiled
from its sources (oracle/_ref) on the same inputs:

* loader, conversion and maximum block size: bit for bit;
* MTTKRPs: normwise relative 1e-5; ptiMatrixDotMulSeqTriangle and
  ptiMatrixMaxNorm bit for bit; ptiMatrixSolveNormals 1e-5 of FP64 and 1e-4
  of the reference; ptiMatrix2Norm 1e-5;
* CpdAlsStep from the same seeded factors: factors and weights 1e-4 of the
  reference's CpdAlsStep, fit 1e-4 of the FP64 oracle; KruskalTensorFit of the
  result 1e-5 of the model evaluated at every nonzero; ptiCpdAls runs and
  returns finite factors.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import synth

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "tests" / "dropin" / "_build" / "dropin"
R, SB, SK, SC, ITERS = 8, 4, 6, 8, 5


def _fill(nrows, mode, stride):
    i = np.arange(nrows, dtype=np.uint32)[:, None]
    j = np.arange(stride, dtype=np.uint32)[None, :]
    v = (0.1 + ((i * 7 + j * 3 + mode * 5) % 11).astype(np.float32) / 10.0).astype(np.float32)
    v[:, R:] = 0
    return v


def _gram_upper(A):
    st = A.shape[1]
    G = (A[:, :R].T.astype(np.float64) @ A[:, :R].astype(np.float64))
    out = np.zeros((R, st), np.float32)
    iu = np.triu_indices(R)
    out[iu] = G[iu].astype(np.float32)
    return out


def _sym(G):
    g = G[:, :R].astype(np.float64)
    return np.triu(g) + np.triu(g, 1).T


def _read(out, name, dtype, shape=None):
    a = np.fromfile(out / f"{name}.bin", dtype=dtype)
    return a.reshape(shape) if shape else a


def test_dropin_caller_against_reference(lib, cuda, ref, orc, tmp_path):
    import ctypes as C
    from oracle.oracle import _Matrix
    if not BIN.exists():
        pytest.fail(f"{BIN} was not built (make -C tests/dropin, run by __graft_entry__.build())")
    dims = (300, 200, 100)
    inds, vals = synth.uniform_tensor(dims, 20000, seed=31)
    tns = tmp_path / "x.tns"
    with open(tns, "w") as f:
        f.write(f"3\n{dims[0]} {dims[1]} {dims[2]}\n")
        for a, b, c, v in zip(inds[0], inds[1], inds[2], vals):
            f.write(f"{a + 1} {b + 1} {c + 1} {v:.6f}\n")
    out = tmp_path / "out"
    out.mkdir()
    res = subprocess.run([str(BIN), str(tns), str(out), str(R), str(SB), str(SK), str(SC), str(ITERS)],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "dropin ok" in res.stdout
    stride = 8
    rc, rdims, rinds, rvals = ref.load(tns)
    assert rc == 0 and list(rdims) == list(dims)
    np.testing.assert_array_equal(_read(out, "ndims", np.uint32), rdims)
    for m in range(3):
        np.testing.assert_array_equal(_read(out, f"coo_ind{m}", np.uint32), rinds[m])
    np.testing.assert_array_equal(_read(out, "coo_vals", np.float32), rvals)
    mats = [_fill(d, m, stride) for m, d in enumerate(dims)]
    for mode in range(3):
        want = ref.mttkrp_coo(list(dims), rinds, rvals, mats, R, mode)
        got = _read(out, f"mttkrp_coo{mode}", np.float32, (dims[mode], stride))
        assert rel_err(got[:, :R], want[:, :R]) < 1e-5
    h = ref.to_hicoo(list(dims), rinds, rvals, SB, SK, SC)
    np.testing.assert_array_equal(_read(out, "h_bptr", np.uint64), h["bptr"])
    np.testing.assert_array_equal(_read(out, "h_kptr", np.uint64), h["kptr"])
    np.testing.assert_array_equal(_read(out, "h_cptr", np.uint64), h["cptr"])
    np.testing.assert_array_equal(_read(out, "h_vals", np.float32), h["vals"])
    assert int(_read(out, "h_max_nnzb", np.uint64)[0]) == h["max_nnzb"]
    for m in range(3):
        np.testing.assert_array_equal(_read(out, f"h_binds{m}", np.uint32), h["binds"][m])
        np.testing.assert_array_equal(_read(out, f"h_einds{m}", np.uint8), h["einds"][m])
    for mode in range(3):
        want = ref.mttkrp_hicoo(list(dims), h, mats, R, mode)
        got = _read(out, f"mttkrp_hicoo{mode}", np.float32, (dims[mode], stride))
        assert rel_err(got[:, :R], want[:, :R]) < 1e-5
    # dense helpers, on the Grams the caller formed (upper triangles only)
    ata = [_gram_upper(m) for m in mats] + [np.zeros((R, stride), np.float32)]
    arr = (C.POINTER(_Matrix) * 4)(*[C.pointer(_Matrix(R, R, R, stride, a.ctypes.data)) for a in ata])
    keep = ata
    assert ref.L.ptiMatrixDotMulSeqTriangle(C.c_uint32(0), C.c_uint32(3), arr) == 0
    np.testing.assert_array_equal(_read(out, "dotmul_tri", np.float32, (R, stride))[:, :R], keep[3][:, :R])
    rhs = _fill(dims[0], 7, stride)
    V = _sym(_gram_upper(mats[1])) * _sym(_gram_upper(mats[2]))
    want64 = np.linalg.solve(V, rhs[:, :R].astype(np.float64).T).T
    got = _read(out, "solve_normals", np.float32, (dims[0], stride))
    assert rel_err(got[:, :R], want64) < 1e-5
    ata2 = [_gram_upper(m) for m in mats] + [np.zeros((R, stride), np.float32)]
    arr2 = (C.POINTER(_Matrix) * 4)(*[C.pointer(_Matrix(R, R, R, stride, a.ctypes.data)) for a in ata2])
    rrhs = rhs.copy()
    assert ref.L.ptiMatrixSolveNormals(C.c_uint32(0), C.c_uint32(3), arr2,
                                       C.pointer(_Matrix(dims[0], R, dims[0], stride, rrhs.ctypes.data))) == 0
    assert rel_err(got[:, :R], rrhs[:, :R]) < 1e-4
    # 2-norm of the solved matrix, max-norm of a fresh one
    a = got.copy()
    lr = np.zeros(R, np.float32)
    assert ref.L.ptiMatrix2Norm(C.pointer(_Matrix(dims[0], R, dims[0], stride, a.ctypes.data)),
                                lr.ctypes.data_as(C.c_void_p)) == 0
    assert rel_err(_read(out, "norm2_lambda", np.float32), lr) < 1e-5
    assert rel_err(_read(out, "norm2_matrix", np.float32, (dims[0], stride))[:, :R], a[:, :R]) < 1e-5
    b = _fill(dims[0], 9, stride)
    assert ref.L.ptiMatrixMaxNorm(C.pointer(_Matrix(dims[0], R, dims[0], stride, b.ctypes.data)),
                                  lr.ctypes.data_as(C.c_void_p)) == 0
    np.testing.assert_array_equal(_read(out, "maxnorm_lambda", np.float32), lr)
    np.testing.assert_array_equal(_read(out, "maxnorm_matrix", np.float32, (dims[0], stride))[:, :R], b[:, :R])
    lam = (1.0 + 0.25 * np.arange(R)).astype(np.float64)
    H = np.ones((R, R))
    for m in mats:
        H *= _sym(_gram_upper(m))
    assert abs(_read(out, "kruskal_normsq", np.float64)[0] - lam @ H @ lam) < 1e-6 * (lam @ H @ lam)
    nx = float((rvals.astype(np.float64) ** 2).sum())
    assert abs(_read(out, "tensor_normsq", np.float64)[0] - nx) < 1e-9 * nx
    # CPD: ptiCpdAls ran; CpdAlsStep against the reference's own step
    assert np.all(np.isfinite(_read(out, "cpd_lambda", np.float32)))
    assert np.isfinite(_read(out, "cpd_fit", np.float64)[0])
    for m in range(3):
        assert np.all(np.isfinite(_read(out, f"cpd_factor{m}", np.float32)))
    init = [_fill(d, m, stride)[:, :R] for m, d in enumerate(dims)]
    rfit, rlam, rfacs = ref.cpd_als_step(list(dims), rinds, rvals, R, ITERS, init)
    slam = _read(out, "step_lambda", np.float32)
    sfacs = [_read(out, f"step_factor{m}", np.float32, (d, stride))[:, :R] for m, d in enumerate(dims)]
    assert rel_err(slam, rlam) < 1e-4
    for m in range(3):
        assert rel_err(sfacs[m], rfacs[m]) < 1e-4
    o = orc.cpd_als(list(dims), rinds, rvals, R, ITERS, init)
    assert abs(_read(out, "step_fit", np.float64)[0] - o["fit"]) < 1e-4
    direct = orc.kruskal_fit(list(dims), rinds, rvals, slam.astype(np.float64), [f.astype(np.float64) for f in sfacs])
    assert abs(_read(out, "kruskal_fit", np.float64)[0] - direct) < 1e-5
