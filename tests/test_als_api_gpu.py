"""GPU: the reference's dense ALS helpers, its ALS step on caller-seeded
factors and its device-array COO MTTKRP, called through the C ABI and checked
against the reference library compiled from its sources (oracle/_ref) and
against FP64 numpy:

* ptiMatrixDotMulSeqTriangle (src/matrix/matrix.c:340-385): bit for bit;
* ptiMatrixSolveNormals (src/matrix/matrix_solver.c:32-83): relative 1e-5 of an
  FP64 solve, 1e-4 of the reference's FP32 LAPACK solve;
* ptiMatrixMaxNorm bit for bit, ptiMatrix2Norm and GetFinalLambda 1e-6
  (src/matrix/matrix.c:389-572), and their ptiRankMatrix twins;
* KruskalTensorFrobeniusNormSquared / SparseKruskalTensorInnerProduct /
  KruskalTensorFit (src/ktensor/ktensor.c:77-240): 1e-6 of FP64, and the fit
  of a model equal to the direct evaluation at every nonzero (oracle);
* CpdAlsStep / CpdAlsStepHiCOO (src/sptensor/cpd.c:32-160,
  src/sptensor/hicoo/cpd.c:31): factors, weights and the last MTTKRP output
  within 1e-4 of the reference's own step from the same seeded factors, fit
  within 1e-4 of the FP64 oracle;
* ptiCudaMTTKRPDevice (src/sptensor/mttkrp_cuda.cu:378-434): adds into the
  caller's output, 1e-5 of the oracle.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import COOTensor, ffi, synth
from hiparti_b200.api import _MatrixSet

pytestmark = pytest.mark.gpu


class _RankSet:
    """ptiRankMatrix structs over numpy arrays (cffi, our library)."""

    def __init__(self, arrays, R):
        self.arrays = arrays
        self.structs = ffi.new("ptiRankMatrix[]", len(arrays))
        self.ptrs = ffi.new("ptiRankMatrix *[]", len(arrays))
        for i, a in enumerate(arrays):
            s = self.structs[i]
            s.nrows, s.ncols, s.cap, s.stride = a.shape[0], R, a.shape[0], a.shape[1]
            s.values = ffi.cast("float *", a.ctypes.data)
            self.ptrs[i] = ffi.addressof(self.structs, i)


def _ref_mats(arrays, R, rank_type=False):
    from oracle.oracle import _Matrix, _RankMatrix
    T = _RankMatrix if rank_type else _Matrix
    ms = [T(a.shape[0], R, a.shape[0], a.shape[1], a.ctypes.data) for a in arrays]
    return (C.POINTER(T) * len(ms))(*[C.pointer(m) for m in ms]), ms


def _grams(N, R, stride, seed, upper_only=True):
    """Well-conditioned Grams A^T A; with upper_only the row-major lower
    triangle holds NaN (the part the reference's ssyrk_ calls leave unwritten)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(N):
        A = rng.random((4 * R + 50, R)).astype(np.float32)
        G = np.zeros((R, stride), np.float32)
        G[:, :R] = (A.T.astype(np.float64) @ A).astype(np.float32)
        if upper_only:
            G[np.tril_indices(R, -1)] = np.nan
        out.append(G)
    return out


def _full(G, R):
    g = G[:, :R].astype(np.float64).copy()
    il = np.tril_indices(R, -1)
    g[il] = g.T[il]
    return g


@pytest.mark.parametrize("rank_type", [False, True])
@pytest.mark.parametrize("R,N,mode", [(16, 3, 0), (32, 4, 2), (5, 3, 1)])
def test_dotmul_triangle_and_solve(lib, cuda, ref, rank_type, R, N, mode):
    stride = ((R - 1) // 8 + 1) * 8
    grams = _grams(N, R, stride, seed=R + N)
    rng = np.random.default_rng(7)
    rhs0 = np.zeros((500, stride), np.float32)
    rhs0[:, :R] = rng.standard_normal((500, R)).astype(np.float32)
    # ours: DotMulSeqTriangle
    ours = [g.copy() for g in grams] + [np.zeros((R, stride), np.float32)]
    S = _RankSet(ours, R) if rank_type else _MatrixSet(ours, R)
    fn = lib.ptiRankMatrixDotMulSeqTriangle if rank_type else lib.ptiMatrixDotMulSeqTriangle
    assert fn(mode, N, S.ptrs) == 0
    theirs = [g.copy() for g in grams] + [np.zeros((R, stride), np.float32)]
    arr, keep = _ref_mats(theirs, R, rank_type)
    rfn = ref.L.ptiRankMatrixDotMulSeqTriangle if rank_type else ref.L.ptiMatrixDotMulSeqTriangle
    assert rfn(C.c_uint32(mode), C.c_uint32(N), arr) == 0
    np.testing.assert_array_equal(ours[N][:, :R], theirs[N][:, :R])
    # ours: SolveNormals against an FP64 solve and the reference's FP32 LAPACK
    V = np.ones((R, R))
    for k in range(1, N):
        V *= _full(grams[(mode + k) % N], R)
    want64 = np.linalg.solve(V, rhs0[:, :R].astype(np.float64).T).T
    ours = [g.copy() for g in grams] + [np.zeros((R, stride), np.float32)]
    S = _RankSet(ours, R) if rank_type else _MatrixSet(ours, R)
    rhs = rhs0.copy()
    T = _RankSet([rhs], R) if rank_type else _MatrixSet([rhs], R)
    sfn = lib.ptiRankMatrixSolveNormals if rank_type else lib.ptiMatrixSolveNormals
    assert sfn(mode, N, S.ptrs, T.ptrs[0]) == 0
    assert rel_err(rhs[:, :R], want64) < 1e-5
    theirs = [g.copy() for g in grams] + [np.zeros((R, stride), np.float32)]
    arr, keep = _ref_mats(theirs, R, rank_type)
    rrhs = rhs0.copy()
    rarr, rkeep = _ref_mats([rrhs], R, rank_type)
    rsfn = ref.L.ptiRankMatrixSolveNormals if rank_type else ref.L.ptiMatrixSolveNormals
    assert rsfn(C.c_uint32(mode), C.c_uint32(N), arr, rarr[0]) == 0
    assert rel_err(rhs[:, :R], rrhs[:, :R]) < 1e-4


@pytest.mark.parametrize("rank_type", [False, True])
def test_norms_and_final_lambda(lib, cuda, ref, rank_type):
    R, stride, I = 12, 16, 3000
    rng = np.random.default_rng(3)
    A0 = np.zeros((I, stride), np.float32)
    A0[:, :R] = rng.standard_normal((I, R)).astype(np.float32) * 3
    A0[:, 3] = -np.abs(A0[:, 3])  # a column with no positive entry: max-norm 1
    Set = _RankSet if rank_type else _MatrixSet
    pre = "ptiRankMatrix" if rank_type else "ptiMatrix"
    for name, exact in (("MaxNorm", True), ("2Norm", False)):
        a, b = A0.copy(), A0.copy()
        la, lb = np.zeros(R, np.float32), np.zeros(R, np.float32)
        S = Set([a], R)
        assert getattr(lib, pre + name)(S.ptrs[0], ffi.cast("float *", la.ctypes.data)) == 0
        arr, keep = _ref_mats([b], R, rank_type)
        assert getattr(ref.L, pre + name)(arr[0], lb.ctypes.data_as(C.c_void_p)) == 0
        if exact:
            np.testing.assert_array_equal(la, lb)
            np.testing.assert_array_equal(a[:, :R], b[:, :R])
            assert la[3] == 1.0
        else:
            assert rel_err(la, np.sqrt((A0[:, :R].astype(np.float64) ** 2).sum(0))) < 1e-6
            assert rel_err(la, lb) < 1e-5 and rel_err(a[:, :R], b[:, :R]) < 1e-5
    # GetFinalLambda over three factors
    mats = [A0.copy() for _ in range(3)]
    for k, m in enumerate(mats):
        m[:, :R] *= k + 1
    theirs = [m.copy() for m in mats]
    lam = np.linspace(1, 2, R).astype(np.float32)
    lr = lam.copy()
    S = Set(mats, R)
    (lib.GetRankFinalLambda if rank_type else lib.GetFinalLambda)(R, 3, S.ptrs, ffi.cast("float *", lam.ctypes.data))
    arr, keep = _ref_mats(theirs, R, rank_type)
    (ref.L.GetRankFinalLambda if rank_type else ref.L.GetFinalLambda)(
        C.c_uint32(R) if not rank_type else C.c_uint8(R), C.c_uint32(3), arr, lr.ctypes.data_as(C.c_void_p))
    assert rel_err(lam, lr) < 1e-5
    for m, t in zip(mats, theirs):
        assert rel_err(m[:, :R], t[:, :R]) < 1e-5


def test_kruskal_fit_pieces(lib, cuda, orc, ref):
    dims = (300, 200, 100)
    R = 8
    stride = 8
    inds, vals, _ = synth.planted_tensor(dims, 20000, 4, 0.01, seed=5)
    rng = np.random.default_rng(6)
    facs = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    facs = [f / np.linalg.norm(f, axis=0) for f in facs]
    lam = rng.uniform(1, 5, R).astype(np.float32)
    mats = []
    for f in facs:
        a = np.zeros((f.shape[0], stride), np.float32)
        a[:, :R] = f
        mats.append(a)
    # ata with only the upper triangle written (NaN below), as ssyrk_ leaves it
    ata = []
    for f in facs:
        G = np.full((R, stride), np.nan, np.float32)
        full = (f.T.astype(np.float64) @ f).astype(np.float32)
        iu = np.triu_indices(R)
        G[iu] = full[iu]
        G[:, R:] = 0
        ata.append(G)
    ata.append(np.zeros((R, stride), np.float32))
    lp = ffi.cast("float *", lam.ctypes.data)
    A = _MatrixSet(ata, R)
    norm = lib.KruskalTensorFrobeniusNormSquared(3, lp, A.ptrs)
    Hd = np.ones((R, R))
    for f in facs:
        Hd *= f.T.astype(np.float64) @ f
    want = float(lam.astype(np.float64) @ Hd @ lam.astype(np.float64))
    assert abs(norm - want) < 1e-6 * abs(want)
    assert not np.any(np.isnan(ata[3][:, :R]))
    # inner product: last factor against the MTTKRP of the last mode
    M = orc.mttkrp_coo(inds, vals, mats, R, 2)
    last = np.zeros((dims[2], stride), np.float32)
    last[:, :R] = M[: dims[2], :R]
    S = _MatrixSet(mats + [last], R)
    inner = lib.SparseKruskalTensorInnerProduct(3, lp, S.ptrs)
    want_inner = float(((mats[2][:, :R].astype(np.float64) * last[:, :R]) @ lam.astype(np.float64)).sum())
    assert abs(inner - want_inner) < 1e-6 * abs(want_inner)
    # the fit equals the direct evaluation of the model at every nonzero
    coo = COOTensor(dims, inds, vals)
    fit = lib.KruskalTensorFit(coo.c, lp, S.ptrs, A.ptrs)
    direct = orc.kruskal_fit(dims, inds, vals, lam.astype(np.float64), [f.astype(np.float64) for f in facs])
    assert abs(fit - direct) < 1e-6
    assert abs(lib.SparseTensorFrobeniusNormSquared(coo.c) - float((vals.astype(np.float64) ** 2).sum())) < 1e-6 * \
        float((vals.astype(np.float64) ** 2).sum())


@pytest.mark.parametrize("fmt", ["coo", "hicoo"])
def test_cpd_als_step_vs_reference(lib, cuda, orc, ref, fmt):
    dims = (200, 150, 100)
    R = 8
    stride = 8
    inds, vals, _ = synth.planted_tensor(dims, 30000, 5, 0.01, seed=11)
    rng = np.random.default_rng(12)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    iters = 6
    mats = []
    for a in init:
        m = np.zeros((a.shape[0], stride), np.float32)
        m[:, :R] = a
        mats.append(m)
    tmp = np.zeros((max(dims), stride), np.float32)
    lam = np.zeros(R, np.float32)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    if fmt == "coo":
        S = _MatrixSet(mats + [tmp], R)
        fit = lib.CpdAlsStep(coo.c, R, iters, 0.0, S.ptrs, ffi.cast("float *", lam.ctypes.data))
    else:
        h = coo.to_hicoo(4, 6, 8)
        S = _RankSet(mats + [tmp], R)
        fit = lib.CpdAlsStepHiCOO(h.c, R, iters, 0.0, S.ptrs, ffi.cast("float *", lam.ctypes.data))
    rfit, rlam, rfacs = ref.cpd_als_step(list(dims), inds, vals, R, iters, init)
    for m in range(3):
        assert rel_err(mats[m][:, :R], rfacs[m]) < 1e-4
    assert rel_err(lam, rlam) < 1e-4
    o = orc.cpd_als(list(dims), inds, vals, R, iters, init)
    assert abs(fit - o["fit"]) < 1e-4
    # mats[N]: the MTTKRP of the last mode from the last iteration, as the
    # reference leaves it (before the final normalisation of the factors)
    assert S.structs[3].nrows == dims[2]
    assert np.all(np.isfinite(tmp[: dims[2], :R])) and np.linalg.norm(tmp[: dims[2], :R]) > 0


def test_cuda_mttkrp_device_adds(lib, cuda, orc):
    import torch
    dims = (700, 500, 300)
    R = 16
    inds, vals = synth.zipf_tensor(dims, 40000, s=1.1, seed=2)
    mats = synth.factor_matrices(dims, R, seed=3)
    mode = 1
    di = [torch.from_numpy(i.view(np.int32)).to(cuda) for i in inds]
    dv = torch.from_numpy(vals).to(cuda)
    dm = [torch.from_numpy(m).to(cuda) for m in mats]
    out = torch.full((dims[mode], mats[0].shape[1]), 1.0, device=cuda)
    out[:, R:] = 0
    ptrs_i = torch.tensor([t.data_ptr() for t in di], dtype=torch.int64, device=cuda)
    ptrs_m = torch.tensor([t.data_ptr() for t in dm] + [out.data_ptr()], dtype=torch.int64, device=cuda)
    order = torch.tensor([(mode + i) % 3 for i in range(3)], dtype=torch.int32, device=cuda)
    rc = lib.ptiCudaMTTKRPDevice(mode, 3, vals.size, R, mats[0].shape[1], ffi.NULL,
                                 ffi.cast("ptiIndex **", ptrs_i.data_ptr()), ffi.cast("ptiValue *", dv.data_ptr()),
                                 ffi.cast("ptiIndex *", order.data_ptr()), ffi.cast("ptiValue **", ptrs_m.data_ptr()),
                                 ffi.NULL)
    assert rc == 0
    want = orc.mttkrp_coo(inds, vals, mats, R, mode)[: dims[mode], :R] + 1.0
    assert rel_err(out.cpu().numpy()[:, :R], want) < 1e-5
