"""GPU: the HiCOO MTTKRP entry point that allocates no device memory.

It exists for callers that cannot allocate while the operation runs (their
device memory belongs to a host framework's pool, or a fixed budget must not
grow mid-request).  Its scratch lives in fixed arrays inside the library, so
this test checks it through the C ABI against the oracle's HiCOO MTTKRP (the
restatement of the reference's ptiMTTKRPHiCOO) and against the allocating
entry point (ptiB200MTTKRP on an uploaded tensor), within the FP32 tolerance
of the other MTTKRP tests:

* two calls in a row on the same tensor (the second call finds the first
  call's scratch contents and must not depend on them);
* a large tensor followed by a smaller one, so the smaller call runs over a
  tile table whose entries beyond its own tiles are left from the larger call;
* 3-D with 128-wide blocks and 4-D with 16-wide blocks;
* an empty tensor, which must leave the output all zero;
* a tensor too large for the fixed scratch, refused before any GPU work.

This file is collected last so that a failure here comes after every other
test has run.
"""
import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import DeviceTensor, HiCOOTensor, ffi, synth

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _device_hicoo(hh, sb, cuda):
    """The caller's own device copies of the HiCOO arrays."""
    import torch
    return {"bptr": torch.from_numpy(hh["bptr"].view(np.int64)).to(cuda),
            "binds": [torch.from_numpy(b.view(np.int32)).to(cuda) for b in hh["binds"]],
            "einds": [torch.from_numpy(e).to(cuda) for e in hh["einds"]],
            "vals": torch.from_numpy(hh["vals"]).to(cuda), "sb": sb,
            "nnz": int(hh["vals"].size), "nb": int(hh["bptr"].size) - 1}


def _call(lib, dims, h, dmats, R, mode, out, stream):
    N = len(dims)
    order = ffi.new("ptiIndex[]", [(mode + i) % N for i in range(N)])
    nd = ffi.new("ptiIndex[]", list(dims))
    if h["nnz"]:
        binds = ffi.new("ptiBlockIndex *[]", [ffi.cast("ptiBlockIndex *", b.data_ptr()) for b in h["binds"]])
        einds = ffi.new("ptiElementIndex *[]", [ffi.cast("ptiElementIndex *", e.data_ptr()) for e in h["einds"]])
        bptr = ffi.cast("ptiNnzIndex *", h["bptr"].data_ptr())
        vals = ffi.cast("ptiValue *", h["vals"].data_ptr())
    else:
        binds = einds = bptr = vals = ffi.NULL
    mats = ffi.new("float *[]", [ffi.cast("float *", m.data_ptr()) for m in dmats])
    stride = dmats[0].shape[1]
    return lib.ptiB200MTTKRPHiCOONoAlloc(
        N, nd, h["nnz"], h["nb"], h["sb"], bptr, binds, einds, vals, mats, R, stride, order, mode,
        ffi.cast("float *", out.data_ptr()), ffi.cast("void *", stream))


def _case(orc, dims, nnz, R, sb, seed, zipf=True):
    if zipf:
        inds, vals = synth.zipf_tensor(dims, nnz, s=1.1, seed=seed)
    else:
        inds, vals = synth.uniform_tensor(dims, nnz, seed=seed)
    hh = orc.hicoo_build(dims, inds, vals, sb, sb + 2, sb + 5)
    mats = synth.factor_matrices(dims, R, seed=seed + 1)
    return hh, mats


def _check(lib, cuda, orc, dims, hh, sb, mats, R, stream, calls=2):
    import torch
    dmats = [torch.from_numpy(m).to(cuda) for m in mats]
    h = _device_hicoo(hh, sb, cuda)
    dt = DeviceTensor.from_hicoo(HiCOOTensor(dims, sb, sb + 2, sb + 5, hh["bptr"], hh["binds"], hh["einds"],
                                             hh["vals"]))
    for mode in range(len(dims)):
        want = orc.mttkrp_hicoo(hh, mats, R, mode)[: dims[mode], :R]
        alloc = dt.mttkrp(dmats, mode, rank=R)
        torch.cuda.synchronize()
        alloc = alloc.cpu().numpy()
        for _ in range(calls):  # calls in a row share the fixed scratch
            out = torch.full((dims[mode], dmats[0].shape[1]), float("nan"), device=cuda)
            assert _call(lib, dims, h, dmats, R, mode, out, stream) == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel_err(got[:, :R], want) < TOL
            assert rel_err(got, alloc) < TOL
            assert np.all(got[:, R:] == 0)
    dt.free()


@pytest.mark.parametrize("R", [16, 32])
def test_no_alloc_matches_oracle_and_allocating_entry_point(lib, cuda, orc, R):
    import torch
    dims = (3000, 2000, 1000)
    hh, mats = _case(orc, dims, 200_000, R, 7, seed=R)
    _check(lib, cuda, orc, dims, hh, 7, mats, R, torch.cuda.current_stream().cuda_stream)


def test_no_alloc_4d_small_blocks(lib, cuda, orc):
    import torch
    dims = (400, 300, 200, 50)
    hh, mats = _case(orc, dims, 150_000, 24, 4, seed=5, zipf=False)
    _check(lib, cuda, orc, dims, hh, 4, mats, 24, torch.cuda.current_stream().cuda_stream)


def test_no_alloc_larger_then_smaller(lib, cuda, orc):
    """The smaller call's tiles are a prefix of the table the larger call
    filled; its result must not see the larger call's entries."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    big_dims, small_dims = (5000, 4000, 3000), (700, 600, 500)
    big, big_mats = _case(orc, big_dims, 600_000, 16, 7, seed=11)
    small, small_mats = _case(orc, small_dims, 30_000, 16, 7, seed=12)
    hb = _device_hicoo(big, 7, cuda)
    dm = [torch.from_numpy(m).to(cuda) for m in big_mats]
    out = torch.empty((big_dims[0], dm[0].shape[1]), device=cuda)
    assert _call(lib, big_dims, hb, dm, 16, 0, out, stream) == 0
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy()[:, :16], orc.mttkrp_hicoo(big, big_mats, 16, 0)[: big_dims[0], :16]) < TOL
    _check(lib, cuda, orc, small_dims, small, 7, small_mats, 16, stream, calls=1)


def test_no_alloc_empty_tensor_zeroes_output(lib, cuda):
    import torch
    dims = (40, 30, 20)
    R = 8
    dmats = [torch.rand((d, R), device=cuda) for d in dims]
    h = {"nnz": 0, "nb": 0, "sb": 7}
    out = torch.full((dims[1], R), float("nan"), device=cuda)
    assert _call(lib, dims, h, dmats, R, 1, out, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0


def test_no_alloc_refuses_tensors_beyond_its_scratch(lib):
    # checked on the host before any device work: the pointers are never used
    N = 3
    order = ffi.new("ptiIndex[]", [0, 1, 2])
    nd = ffi.new("ptiIndex[]", [10, 10, 10])
    dummy = ffi.new("float *[]", [ffi.cast("float *", 256)] * 3)
    too_many = (1 << 18) * 1024 + 1
    rc = lib.ptiB200MTTKRPHiCOONoAlloc(N, nd, too_many, 1, 7, ffi.NULL, ffi.NULL, ffi.NULL, ffi.NULL, dummy, 8, 8,
                                       order, 0, ffi.cast("float *", 256), ffi.NULL)
    assert rc == 3  # PTIERR_VALUE_ERROR
