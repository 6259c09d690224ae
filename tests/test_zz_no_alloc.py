"""GPU: the HiCOO MTTKRP entry point that allocates no device memory.

It exists for callers that cannot allocate while the operation runs (their
device memory belongs to a host framework's pool, or a fixed budget must not
grow mid-request).  Its scratch lives in fixed arrays inside the library, so
this test checks it through the C ABI against the allocating entry point
(ptiB200MTTKRP on an uploaded tensor): the same result within the FP32
tolerance of the other MTTKRP tests, on two calls in a row (the second call
finds the first call's scratch contents and must not depend on them), and that
a tensor too large for the fixed scratch is refused before any GPU work.

This file is collected last so that a failure here comes after every other
test has run.
"""
import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import DeviceTensor, HiCOOTensor, ffi, synth

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _call(lib, dims, h, dmats, R, mode, out, stream):
    import torch
    N = len(dims)
    nnz = int(h["vals"].numel())
    nb = int(h["bptr"].numel()) - 1
    order = ffi.new("ptiIndex[]", [(mode + i) % N for i in range(N)])
    nd = ffi.new("ptiIndex[]", list(dims))
    binds = ffi.new("ptiBlockIndex *[]", [ffi.cast("ptiBlockIndex *", b.data_ptr()) for b in h["binds"]])
    einds = ffi.new("ptiElementIndex *[]", [ffi.cast("ptiElementIndex *", e.data_ptr()) for e in h["einds"]])
    mats = ffi.new("float *[]", [ffi.cast("float *", m.data_ptr()) for m in dmats])
    stride = dmats[0].shape[1]
    return lib.ptiB200MTTKRPHiCOONoAlloc(
        N, nd, nnz, nb, h["sb"], ffi.cast("ptiNnzIndex *", h["bptr"].data_ptr()), binds, einds,
        ffi.cast("ptiValue *", h["vals"].data_ptr()), mats, R, stride, order, mode,
        ffi.cast("float *", out.data_ptr()), ffi.cast("void *", stream))


@pytest.mark.parametrize("R", [16, 32])
def test_no_alloc_matches_allocating_entry_point(lib, cuda, orc, R):
    import torch
    dims = (3000, 2000, 1000)
    inds, vals = synth.zipf_tensor(dims, 200_000, s=1.1, seed=R)
    hh = orc.hicoo_build(dims, inds, vals, 7, 9, 12)
    mats = synth.factor_matrices(dims, R, seed=R + 1)
    dmats = [torch.from_numpy(m).to(cuda) for m in mats]
    dt = DeviceTensor.from_hicoo(HiCOOTensor(dims, 7, 9, 12, hh["bptr"], hh["binds"], hh["einds"], hh["vals"]))
    # the caller's own device copies of the HiCOO arrays
    h = {"bptr": torch.from_numpy(hh["bptr"].view(np.int64)).to(cuda),
         "binds": [torch.from_numpy(b.view(np.int32)).to(cuda) for b in hh["binds"]],
         "einds": [torch.from_numpy(e).to(cuda) for e in hh["einds"]],
         "vals": torch.from_numpy(hh["vals"]).to(cuda), "sb": 7}
    stream = torch.cuda.current_stream().cuda_stream
    for mode in range(3):
        ref = dt.mttkrp(dmats, mode, rank=R)
        torch.cuda.synchronize()
        ref = ref.cpu().numpy()
        for _ in range(2):  # two calls in a row share the fixed scratch
            out = torch.full((dims[mode], dmats[0].shape[1]), float("nan"), device=cuda)
            assert _call(lib, dims, h, dmats, R, mode, out, stream) == 0
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel_err(got, ref) < TOL
            assert np.all(got[:, R:] == 0)
    dt.free()


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
