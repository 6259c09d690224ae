"""GPU TTM / TTV against the reference's own ptiSparseTensorMulMatrix and
ptiSparseTensorMulVector (src/sptensor/mmul.c, vmul.c, compiled from its
sources): the fibers, their coordinates, every FP32 value (bit for bit: the
same multiply-then-add sequence per fiber), and the caller's tensor as the
reference leaves it (sorted with the mode last, or untouched when its
sortorder already says so).  The device API is checked against the host
result, and at 10M nonzeros against an FP64 torch reference (normwise 1e-6)."""
import numpy as np
import pytest

from hiparti_b200 import COOTensor, DeviceTensor

pytestmark = pytest.mark.gpu


def _tensor(dims, nnz, seed):
    rng = np.random.default_rng(seed)
    lin = rng.choice(int(np.prod(dims)), nnz, replace=False)
    inds = [i.astype(np.uint32) for i in np.unravel_index(lin, dims)]
    return inds, (rng.standard_normal(nnz) * 10.0 ** rng.integers(-3, 3, nnz)).astype(np.float32)


def _check(ours, theirs, coo, mode):
    finds, yv, (xinds, xvals, xso) = theirs
    assert ours["mode"] == mode
    for m, (a, b) in enumerate(zip(ours["inds"], finds)):
        np.testing.assert_array_equal(a, b)
    assert ours["vals"].shape == yv.shape
    np.testing.assert_array_equal(ours["vals"].view(np.uint32), yv.view(np.uint32))
    for a, b in zip(coo.inds, xinds):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(coo.vals.view(np.uint32), xvals.view(np.uint32))
    np.testing.assert_array_equal(coo._so, xso)


@pytest.mark.parametrize("dims,nnz", [((40, 30, 20), 5000), ((15, 12, 10, 9), 6000), ((300, 7), 1500)])
@pytest.mark.parametrize("R", [1, 5, 8, 16, 17, 32, 40, 100])
def test_ttm_matches_reference(lib, cuda, ref, dims, nnz, R):
    inds, vals = _tensor(dims, nnz, R)
    rng = np.random.default_rng(R + 100)
    for mode in range(len(dims)):
        U = rng.standard_normal((dims[mode], R)).astype(np.float32)
        theirs = ref.ttm(dims, inds, vals, U, mode)
        coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
        _check(coo.ttm(U, mode), theirs, coo, mode)


def test_ttm_trusts_sortorder_like_the_reference(lib, cuda, ref):
    """A tensor whose sortorder already reads (other modes, then mode) is not
    sorted by the reference: its fibers are runs in the input order."""
    dims = (20, 15, 12)
    inds, vals = _tensor(dims, 900, 7)
    U = np.random.default_rng(8).standard_normal((12, 8)).astype(np.float32)
    theirs = ref.ttm(dims, inds, vals, U, 2, sortorder=np.array([0, 1, 2], np.uint32))
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())  # sortorder 0,1,2
    ours = coo.ttm(U, 2)
    _check(ours, theirs, coo, 2)
    assert ours["vals"].shape[0] > 800  # fragmented fibers, as the reference makes them


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_ttv_matches_reference(lib, cuda, ref, mode):
    dims = (50, 40, 30)
    inds, vals = _tensor(dims, 8000, mode)
    v = np.random.default_rng(mode).standard_normal(dims[mode]).astype(np.float32)
    theirs = ref.ttm(dims, inds, vals, v, mode, vector=True)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    _check(coo.ttv(v, mode), theirs, coo, mode)


def test_device_ttm_matches_host(lib, cuda):
    import torch
    dims = (60, 50, 40)
    inds, vals = _tensor(dims, 20000, 3)
    for mode, R in [(0, 16), (1, 24), (2, 64), (1, 0)]:
        width = max(R, 1)
        U = np.random.default_rng(mode).standard_normal((dims[mode], width)).astype(np.float32)
        coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
        coo._so[:] = 0  # sortorder as the text loader leaves it: the host path sorts
        host = coo.ttv(U[:, 0], mode) if R == 0 else coo.ttm(U, mode)
        dt = DeviceTensor.from_coo(COOTensor(dims, [i.copy() for i in inds], vals.copy()))
        finds, Y = dt.ttm(torch.from_numpy(U).cuda(), mode, rank=R)
        torch.cuda.synchronize()
        dt.free()
        for m in range(3):
            if m != mode:
                np.testing.assert_array_equal(finds[m].cpu().numpy().astype(np.uint32), host["inds"][m])
        np.testing.assert_array_equal(Y.cpu().numpy().view(np.uint32), host["vals"].view(np.uint32))


def test_device_ttm_large_against_fp64(lib, cuda):
    """10M Zipf nonzeros (the C2 construction's dims), R = 16, mode 2."""
    import torch
    from hiparti_b200.synth import coords_torch
    dims = (200_000, 150_000, 20_000)
    inds = coords_torch(dims, 10_000_000, 77, zipf_s=1.1, device=cuda)
    g = torch.Generator(device=cuda)
    g.manual_seed(78)
    vals = torch.rand(10_000_000, generator=g, device=cuda)
    U = torch.rand((dims[2], 16), generator=g, device=cuda)
    dt = DeviceTensor.from_torch_coo(dims, inds, vals)
    finds, Y = dt.ttm(U, 2)
    torch.cuda.synchronize()
    dt.free()
    # FP64 reference: fibers are the distinct (i0, i1) pairs in sorted order
    key = inds[0].long() * dims[1] + inds[1].long()
    uk, inv = torch.unique(key, sorted=True, return_inverse=True)
    ref = torch.zeros((uk.numel(), 16), dtype=torch.float64, device=cuda)
    ref.index_add_(0, inv, vals.double()[:, None] * U.double()[inds[2].long()])
    assert Y.shape[0] == uk.numel()
    np.testing.assert_array_equal((finds[0].long() * dims[1] + finds[1].long()).cpu().numpy(), uk.cpu().numpy())
    err = float((Y[:, :16].double() - ref).norm() / ref.norm())
    assert err < 1e-6, err


@pytest.mark.parametrize("eps", [1e-6, 0.5, 3.0])
def test_semi_sparse_to_sparse_matches_reference(lib, cuda, ref, eps):
    """ptiSemiSparseTensorToSparseTensor (src/sptensor/fromssp.c) of a TTM
    result with zeros, NaN, infinity and small values planted, against the
    reference's own conversion."""
    dims = (30, 25, 20)
    inds, vals = _tensor(dims, 3000, 11)
    U = np.random.default_rng(12).standard_normal((20, 8)).astype(np.float32)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    coo._so[:] = 0  # sorted fibers, so every coordinate of Y is distinct (ties would leave
    Y = coo.ttm(U, 2)  # the reference's unstable sort free to order equal coordinates)
    v = Y["vals"]
    v[0, 0], v[1, 1], v[2, 2], v[3, 3] = 0.0, np.nan, np.inf, 1e-40  # zero, NaN, inf, subnormal
    v[4, :8] = 1e-7
    want_inds, want_vals = ref.ssp_to_sparse(Y, eps)
    got = COOTensor.from_semi_sparse(Y, eps)
    assert got.dims == Y["dims"]
    for a, b in zip(got.inds, want_inds):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(got.vals.view(np.uint32), want_vals.view(np.uint32))


@pytest.mark.parametrize("R2", [3, 8, 20])
def test_semi_sparse_ttm_matches_reference(lib, cuda, ref, R2):
    """ptiSemiSparseTensorMulMatrix (src/ssptensor/mmul.c): a TTM result's
    dense fibers times a second matrix, bit for bit against the reference."""
    dims = (40, 30, 25)
    inds, vals = _tensor(dims, 4000, 21)
    U = np.random.default_rng(22).standard_normal((25, 12)).astype(np.float32)
    coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
    Y = coo.ttm(U, 2)
    V = np.random.default_rng(23).standard_normal((12, R2)).astype(np.float32)
    want_inds, want_vals = ref.ssp_ttm(Y, V)
    got = COOTensor.semi_sparse_ttm(Y, V)
    assert got["dims"][2] == R2
    for a, b in zip(got["inds"], want_inds):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(got["vals"].view(np.uint32), want_vals.view(np.uint32))


@pytest.mark.parametrize("dims,nnz,R", [((20000, 4, 3), 150_000, 16), ((20000, 4, 3), 150_000, 5),
                                        ((30000, 3, 2), 120_000, 32), ((10000, 40, 10), 3_600_000, 16)])
def test_ttm_very_long_fibers_match_reference(lib, cuda, ref, dims, nnz, R):
    """Fibers of more than 8192 nonzeros along mode 0 (one CTA per fiber: the
    products computed by producer warps, the column sums added by one warp in
    fiber order), mixed with shorter fibers along the other modes; the last
    case has 400 such fibers, more than the grid, so CTAs take several.  Bit
    for bit against the reference's ptiSparseTensorMulMatrix."""
    inds, vals = _tensor(dims, nnz, R + 7)
    rng = np.random.default_rng(R)
    for mode in range(3):
        U = rng.standard_normal((dims[mode], R)).astype(np.float32)
        theirs = ref.ttm(dims, inds, vals, U, mode)
        coo = COOTensor(dims, [i.copy() for i in inds], vals.copy())
        _check(coo.ttm(U, mode), theirs, coo, mode)
