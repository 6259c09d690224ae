"""GPU parity: MTTKRP through the C ABI against the oracle and the reference's
golden outputs.  Tolerance: normwise relative 1e-5 in FP32 (the GPU adds in a
different order than the sequential reference), and every element within the
FP32 summation bound of the FP64 result."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from hiparti_b200 import COOTensor, DeviceTensor, HiCOOTensor, synth

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _check(out, ref32, orc=None, inds=None, vals=None, mats=None, R=None, mode=None):
    assert out.shape == ref32.shape
    assert rel_err(out, ref32) < TOL
    if orc is not None:
        exact = orc.mttkrp_coo_f64(inds, vals, mats, R, mode)[: out.shape[0]]
        absmats = [np.abs(m) for m in mats]
        bound = orc.mttkrp_coo_f64(inds, np.abs(vals), absmats, R, mode)[: out.shape[0]]
        nnz_row = np.bincount(inds[mode], minlength=out.shape[0]).max()
        eps = np.float64(np.finfo(np.float32).eps)
        assert np.all(np.abs(out - exact) <= (len(inds) + nnz_row) * eps * bound + 1e-30)
    # pad columns stay zero
    if R is not None and R < out.shape[1]:
        assert np.all(out[:, R:] == 0)


@pytest.mark.parametrize("case", ["coo3_uniform.npz", "coo4_uniform.npz", "coo3_zipf.npz"])
def test_golden_coo_and_hicoo(lib, cuda, case):
    g = load_golden(case)
    dims = [int(x) for x in g["dims"]]
    N = len(dims)
    R = int(g["R"])
    inds = [g[f"ind{m}"] for m in range(N)]
    mats = [g[f"mat{m}"] for m in range(N)]
    coo = COOTensor(dims, inds, g["vals"])
    h = HiCOOTensor(dims, g["sb"], g["sk"], g["sc"], g["h_bptr"], [g[f"h_binds{m}"] for m in range(N)],
                    [g[f"h_einds{m}"] for m in range(N)], g["h_vals"], kptr=g["h_kptr"])
    for m in range(N):
        for variant in ["seq", "omp", "cuda", "onekernel"]:
            _check(coo.mttkrp(mats, R, m, variant), g[f"coo_out{m}"])
        for variant in ["seq", "omp", "cuda"]:
            _check(h.mttkrp(mats, R, m, variant), g[f"hicoo_out{m}"])


@pytest.mark.parametrize("R", [1, 3, 8, 16, 32, 64, 100, 128, 200])
def test_coo_ranks(lib, cuda, orc, R):
    dims = (300, 200, 100)
    inds, vals = synth.uniform_tensor(dims, 30000, seed=R)
    mats = synth.factor_matrices(dims, R, seed=R + 1)
    coo = COOTensor(dims, inds, vals)
    for m in range(3):
        ref = orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]]
        _check(coo.mttkrp(mats, R, m), ref, orc, inds, vals, mats, R, m)


@pytest.mark.parametrize("N", [2, 3, 4, 5, 8])
def test_orders(lib, cuda, orc, N):
    dims = tuple([40, 30, 20, 12, 9, 7, 5, 4][:N])
    nnz = min(4000, int(np.prod(dims)) // 2)
    inds, vals = synth.uniform_tensor(dims, nnz, seed=N)
    R = 16
    mats = synth.factor_matrices(dims, R, seed=N + 10)
    coo = COOTensor(dims, inds, vals)
    for m in range(N):
        ref = orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]]
        _check(coo.mttkrp(mats, R, m), ref, orc, inds, vals, mats, R, m)
    if N in (3, 4):
        h = orc.hicoo_build(dims, inds, vals, 2, 3, 4)
        ht = HiCOOTensor(dims, 2, 3, 4, h["bptr"], h["binds"], h["einds"], h["vals"], kptr=h["kptr"])
        for m in range(N):
            ref = orc.mttkrp_hicoo(h, mats, R, m)[: dims[m]]
            _check(ht.mttkrp(mats, R, m), ref)


@pytest.mark.parametrize("sb", [1, 4, 7, 8])
def test_hicoo_block_sizes(lib, cuda, orc, sb):
    dims = (700, 500, 300)
    inds, vals = synth.zipf_tensor(dims, 40000, s=1.1, seed=sb)
    R = 32
    mats = synth.factor_matrices(dims, R, seed=sb + 3)
    h = orc.hicoo_build(dims, inds, vals, sb, max(sb, 9), max(sb, 10))
    ht = HiCOOTensor(dims, sb, max(sb, 9), max(sb, 10), h["bptr"], h["binds"], h["einds"], h["vals"])
    for m in range(3):
        ref = orc.mttkrp_hicoo(h, mats, R, m)[: dims[m]]
        _check(ht.mttkrp(mats, R, m), ref)


def test_edge_cases(lib, cuda, orc):
    # single nonzero
    dims = (5, 6, 7)
    coo = COOTensor(dims, [np.array([4], np.uint32), np.array([0], np.uint32), np.array([6], np.uint32)],
                    np.array([2.5], np.float32))
    mats = synth.factor_matrices(dims, 8, seed=1)
    for m in range(3):
        ref = orc.mttkrp_coo(coo.inds, coo.vals, mats, 8, m)[: dims[m]]
        np.testing.assert_allclose(coo.mttkrp(mats, 8, m), ref, rtol=1e-6)
    # empty tensor: output is all zeros
    empty = COOTensor(dims, [np.zeros(0, np.uint32)] * 3, np.zeros(0, np.float32))
    assert np.all(empty.mttkrp(mats, 8, 1) == 0)
    # every nonzero in one output row (one huge slice)
    dims = (4, 3000, 200)
    rng = np.random.default_rng(3)
    n = 50000
    keys = rng.choice(3000 * 200, n, replace=False)
    inds = [np.zeros(n, np.uint32), (keys // 200).astype(np.uint32), (keys % 200).astype(np.uint32)]
    vals = rng.random(n, dtype=np.float32)
    mats = synth.factor_matrices(dims, 16, seed=2)
    coo = COOTensor(dims, inds, vals)
    ref = orc.mttkrp_coo(inds, vals, mats, 16, 0)[:4]
    assert rel_err(coo.mttkrp(mats, 16, 0), ref) < TOL
    h = orc.hicoo_build(dims, inds, vals, 7, 7, 7)
    ht = HiCOOTensor(dims, 7, 7, 7, h["bptr"], h["binds"], h["einds"], h["vals"])
    assert rel_err(ht.mttkrp(mats, 16, 0), ref) < TOL


def test_shape_errors(lib):
    from hiparti_b200 import PtiError
    dims = (5, 6, 7)
    coo = COOTensor(dims, [np.array([1], np.uint32)] * 3, np.array([1.0], np.float32))
    mats = synth.factor_matrices((5, 6, 8), 8, seed=1)  # wrong rows in mode 2
    with pytest.raises(PtiError) as e:
        coo.mttkrp(mats, 8, 0)
    assert e.value.code == 2


def test_out_of_range_coordinate_is_an_error(lib, cuda):
    from hiparti_b200 import PtiError
    dims = (5, 6, 7)
    coo = COOTensor(dims, [np.array([1], np.uint32), np.array([9], np.uint32), np.array([1], np.uint32)],
                    np.array([1.0], np.float32))
    mats = synth.factor_matrices(dims, 8, seed=1)
    with pytest.raises(PtiError) as e:
        coo.mttkrp(mats, 8, 0)
    assert e.value.code == 3
    # a HiCOO tensor whose element offset runs past the mode size
    h = HiCOOTensor(dims, 3, 3, 3, np.array([0, 1], np.uint64),
                    [np.array([0], np.uint32)] * 3, [np.array([1], np.uint8), np.array([7], np.uint8),
                                                      np.array([1], np.uint8)],
                    np.array([1.0], np.float32))
    with pytest.raises(PtiError) as e:
        h.mttkrp(mats, 8, 0)
    assert e.value.code == 3


@pytest.mark.parametrize("fmt", ["coo", "hicoo"])
@pytest.mark.parametrize("dtype", ["float32", "bfloat16"])
def test_device_api_torch(lib, cuda, orc, fmt, dtype):
    import torch
    dims = (400, 300, 200)
    inds, vals = synth.zipf_tensor(dims, 60000, s=1.1, seed=7)
    R = 32
    mats = synth.factor_matrices(dims, R, seed=8)
    tdt = getattr(torch, dtype)
    dmats = [torch.from_numpy(m).to(cuda).to(tdt) for m in mats]
    # the oracle sees the same (rounded) factor values
    ref_mats = [d.float().cpu().numpy() for d in dmats]
    if fmt == "coo":
        dt = DeviceTensor.from_coo(COOTensor(dims, inds, vals))
    else:
        h = orc.hicoo_build(dims, inds, vals, 7, 9, 12)
        dt = DeviceTensor.from_hicoo(HiCOOTensor(dims, 7, 9, 12, h["bptr"], h["binds"], h["einds"], h["vals"]))
    for m in range(3):
        out = dt.mttkrp(dmats, m, rank=R)
        torch.cuda.synchronize()
        ref = orc.mttkrp_coo(inds, vals, ref_mats, R, m)[: dims[m]]
        assert rel_err(out.cpu().numpy(), ref) < TOL
    dt.check()  # no device error recorded by the asynchronous calls
    dt.free()


@pytest.mark.parametrize("N", [3, 4])
@pytest.mark.parametrize("dtype", ["float32", "bfloat16"])
@pytest.mark.parametrize("R", [1, 3, 8, 16, 24, 32, 40, 64, 100, 128, 129, 200])
def test_scheduled_hicoo_ranks(lib, cuda, orc, N, dtype, R):
    """Every lane-group shape of the scheduled HiCOO walks: the in-kernel
    decode (3-D, FP32 factors) and the pre-decoded records (4-D, and BF16
    factors) from 1 lane per nonzero up to 32, both BF16 row widths, and the
    direct kernel above R = 128; the BF16 case against the oracle on the
    same BF16-rounded factors."""
    import torch
    dims = (300, 200, 100) if N == 3 else (120, 90, 60, 40)
    inds, vals = synth.zipf_tensor(dims, 30000, s=1.1, seed=R + N)
    mats = synth.factor_matrices(dims, R, seed=R + 1)
    tdt = getattr(torch, dtype)
    dmats = [torch.from_numpy(m).to(cuda).to(tdt) for m in mats]
    ref_mats = [d.float().cpu().numpy() for d in dmats]
    h = orc.hicoo_build(dims, inds, vals, 5, 7, 9)
    dt = DeviceTensor.from_hicoo(HiCOOTensor(dims, 5, 7, 9, h["bptr"], h["binds"], h["einds"], h["vals"]))
    for m in range(N):
        out = dt.mttkrp(dmats, m, rank=R)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = orc.mttkrp_coo(inds, vals, ref_mats, R, m)[: dims[m]]
        assert rel_err(got[:, :R], ref[:, :R]) < TOL, (m, R)
        assert np.all(got[:, R:] == 0)
    dt.check()
    dt.free()


@pytest.mark.parametrize("R", [10, 32])
def test_rank_matrix_entry_points_match_reference(lib, cuda, ref, R):
    """ptiMTTKRPHiCOO_MatrixTiling and the OpenMP MatrixTiling variants
    (ptiRankMatrix factors, 8-bit ncols and stride) against the reference's
    ptiMTTKRPHiCOO_MatrixTiling (src/sptensor/hicoo/mttkrp.c:313-542)."""
    from hiparti_b200 import ffi
    dims = (700, 500, 300)
    inds, vals = synth.zipf_tensor(dims, 30000, s=1.1, seed=R)
    mats = synth.factor_matrices(dims, R, seed=R + 3)
    h = ref.to_hicoo(list(dims), inds, vals, 4, 9, 10)
    ht = HiCOOTensor(dims, 4, 9, 10, h["bptr"], h["binds"], h["einds"], h["vals"], kptr=h["kptr"])
    stride = mats[0].shape[1]
    for mode in range(3):
        want = ref.mttkrp_hicoo_rank(list(dims), h, mats, R, mode)
        for variant in ("seq", "omp", "sched", "reduce", "two"):
            out = np.full((dims[mode], stride), np.nan, np.float32)
            keep = [np.ascontiguousarray(m) for m in mats] + [out]
            rms = [ffi.new("ptiRankMatrix *") for _ in keep]
            for r, a in zip(rms, keep):
                r.nrows, r.ncols, r.cap, r.stride = a.shape[0], R, a.shape[0], stride
                r.values = ffi.cast("ptiValue *", a.ctypes.data)
            arr = ffi.new("ptiRankMatrix *[]", rms)
            order = ffi.new("ptiIndex[]", [(mode + i) % 3 for i in range(3)])
            L = lib
            rc = {"seq": lambda: L.ptiMTTKRPHiCOO_MatrixTiling(ht.c, arr, order, mode),
                  "omp": lambda: L.ptiOmpMTTKRPHiCOO_MatrixTiling(ht.c, arr, order, mode, 8, 1),
                  "sched": lambda: L.ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled(ht.c, arr, order, mode, 8, 1, 0),
                  "reduce": lambda: L.ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce(ht.c, arr, ffi.NULL, order,
                                                                                      mode, 8, 1, 1),
                  "two": lambda: L.ptiOmpMTTKRPHiCOO_MatrixTiling_Scheduled_Reduce_Two(ht.c, arr, ffi.NULL, order,
                                                                                       mode, 8, 1)}[variant]()
            assert rc == 0
            err = float(np.abs(out[:, :R] - want[:, :R]).max() / max(np.abs(want[:, :R]).max(), 1e-30))
            assert err < 1e-5, (mode, variant, err)
            assert not out[:, R:].any()


def test_lock_variant_and_mutex_pool(lib, cuda, orc):
    """ptiOmpMTTKRP_Lock with a pool from ptiMutexAlloc gives the COO MTTKRP."""
    from hiparti_b200 import ffi
    dims = (60, 50, 40)
    inds, vals = synth.uniform_tensor(dims, 5000, seed=4)
    R = 16
    mats = synth.factor_matrices(dims, R, seed=5)
    coo = COOTensor(dims, inds, vals)
    stride = mats[0].shape[1]
    pool = lib.ptiMutexAlloc()
    assert pool != ffi.NULL
    for mode in range(3):
        out = np.zeros((dims[mode], stride), np.float32)
        keep = [np.ascontiguousarray(m) for m in mats] + [out]
        ms = [ffi.new("ptiMatrix *") for _ in keep]
        for m, a in zip(ms, keep):
            m.nrows, m.ncols, m.cap, m.stride = a.shape[0], R, a.shape[0], stride
            m.values = ffi.cast("ptiValue *", a.ctypes.data)
        arr = ffi.new("ptiMatrix *[]", ms)
        order = ffi.new("ptiIndex[]", [(mode + i) % 3 for i in range(3)])
        assert lib.ptiOmpMTTKRP_Lock(coo.c, arr, order, mode, 8, pool) == 0
        want = orc.mttkrp_coo(inds, vals, mats, R, mode)[: dims[mode]]
        assert rel_err(out[:, :R], want[:, :R]) < 1e-5
    lib.ptiMutexFree(pool)


def _hicoo_by_hand(dims, inds, vals, sb):
    """A HiCOO tensor of any order built directly: nonzeros sorted by block
    coordinates (lexicographically), one block per distinct tuple."""
    N = len(dims)
    bl = [(i >> sb).astype(np.int64) for i in inds]
    order = np.lexsort(tuple(bl[::-1]))
    bl = [b[order] for b in bl]
    change = np.ones(vals.size, bool)
    change[1:] = np.any([b[1:] != b[:-1] for b in bl], axis=0)
    starts = np.flatnonzero(change)
    bptr = np.append(starts, vals.size).astype(np.uint64)
    binds = [b[starts].astype(np.uint32) for b in bl]
    einds = [(inds[m][order] & ((1 << sb) - 1)).astype(np.uint8) for m in range(N)]
    return bptr, binds, einds, vals[order].copy()


@pytest.mark.parametrize("N", [2, 5])
def test_hicoo_dropin_other_orders(lib, cuda, orc, N):
    """ptiMTTKRPHiCOO on hand-built 2-D and 5-D HiCOO tensors (the reference's
    conversion makes only 3-D and 4-D ones): the copies of the arrays a mode's
    schedule does not start from overlap the schedule build, and the result
    must still equal the oracle's COO MTTKRP."""
    dims = (300, 200) if N == 2 else (12, 10, 9, 8, 7)
    nnz = 20000 if N == 2 else 15000
    inds, vals = synth.uniform_tensor(dims, nnz, seed=N + 50)
    R = 16
    mats = synth.factor_matrices(dims, R, seed=N + 51)
    sb = 3 if N == 2 else 2
    bptr, binds, einds, hv = _hicoo_by_hand(dims, inds, vals, sb)
    ht = HiCOOTensor(dims, sb, sb + 2, sb + 3, bptr, binds, einds, hv)
    for m in range(N):
        ref = orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]]
        _check(ht.mttkrp(mats, R, m), ref)
