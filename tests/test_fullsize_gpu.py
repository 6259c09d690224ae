"""GPU parity at the benchmark's full size: the 50M-nonzero Zipf(1.1) HiCOO
MTTKRP (200000 x 150000 x 20000, sb = 7, R = 32), every mode, FP32 and BF16
factors, against an FP64 reference computed with torch on the same GPU (in
chunks of nonzeros, index_add_ into an FP64 output).  Tolerance: normwise
relative 1e-5 (the kernels add in FP32 in another order), pad columns zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (200_000, 150_000, 20_000)
NNZ = 50_000_000
R = 32


def _reference(inds, vals, facs, mode):
    import torch
    out = torch.zeros((DIMS[mode], R), dtype=torch.float64, device=vals.device)
    others = [k for k in range(3) if k != mode]
    step = 4_000_000
    for z0 in range(0, vals.numel(), step):
        sl = slice(z0, z0 + step)
        p = vals[sl].double()[:, None]
        for k in others:
            p = p * facs[k][inds[k][sl].long(), :R].double()
        out.index_add_(0, inds[mode][sl].long(), p)
    return out


@pytest.fixture(scope="module")
def c2(cuda):
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.synth import coords_torch
    inds = coords_torch(DIMS, NNZ, 2024, zipf_s=1.1, device=cuda)
    g = torch.Generator(device=cuda)
    g.manual_seed(2025)
    vals = torch.rand(NNZ, generator=g, device=cuda, dtype=torch.float32)
    coo = DeviceTensor.from_torch_coo(DIMS, inds, vals)
    h = coo.to_hicoo(7, 10, 14)
    coo.free()
    facs = [torch.rand((d, R), generator=g, device=cuda, dtype=torch.float32) for d in DIMS]
    yield inds, vals, h, facs
    h.free()


@pytest.mark.parametrize("dtype", ["float32", "bfloat16"])
def test_fullsize_hicoo_mttkrp_against_fp64(lib, cuda, c2, dtype):
    import torch
    inds, vals, h, facs = c2
    f = [a.to(getattr(torch, dtype)) for a in facs]
    ref_facs = [a.float() for a in f]  # the reference sees the same (rounded) factors
    for m in range(3):
        out = h.mttkrp(f, m, rank=R)
        torch.cuda.synchronize()
        ref = _reference(inds, vals, ref_facs, m)
        err = float((out.double() - ref).norm() / ref.norm())
        assert err < 1e-5, (dtype, m, err)
        del out, ref
    torch.cuda.empty_cache()


def test_fullsize_mttkrp_is_linear_in_each_factor(lib, cuda, c2):
    """MTTKRP(X, A, B) is linear in every operand factor: doubling one of them
    doubles the result, bit for bit apart from the summation order."""
    import torch
    _, _, h, facs = c2
    base = h.mttkrp(facs, 0, rank=R).double()
    twice = h.mttkrp([facs[0], 2 * facs[1], facs[2]], 0, rank=R).double()
    torch.cuda.synchronize()
    err = float((twice - 2 * base).norm() / (2 * base).norm())
    assert err < 1e-6, err
    assert np.isfinite(float(base.sum()))
