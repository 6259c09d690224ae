"""GPU: gradient CP through torch.autograd (forward = CP model at the nonzeros,
backward = per-mode MTTKRP of the residual), checked against FP64 central
finite differences on a 1,000-nonzero tensor, against a gradient built from the
reference's own ptiMTTKRP, and against the oracle at a larger size."""
import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import COOTensor, DeviceTensor, synth

pytestmark = pytest.mark.gpu


def _setup(dims, nnz, R, seed, cuda):
    import torch
    inds, vals, _ = synth.planted_tensor(dims, nnz, 4, 0.05, seed=seed)
    rng = np.random.default_rng(seed + 1)
    stride = ((R - 1) // 8 + 1) * 8
    facs = []
    for d in dims:
        a = np.zeros((d, stride), np.float32)
        a[:, :R] = (0.1 * rng.standard_normal((d, R))).astype(np.float32)
        facs.append(a)
    dt = DeviceTensor.from_coo(COOTensor(dims, inds, vals))
    tf = [torch.from_numpy(a).to(cuda).requires_grad_(True) for a in facs]
    tv = torch.from_numpy(vals).to(cuda)
    return inds, vals, facs, dt, tf, tv


def _loss64(inds, vals, facs, R):
    model = np.ones((vals.size, R))
    for a, ix in zip(facs, inds):
        model *= a[ix, :R].astype(np.float64)
    r = vals.astype(np.float64) - model.sum(1)
    return 0.5 * np.dot(r, r), model.sum(1)


def test_gradient_matches_fp64_finite_differences(lib, cuda):
    from hiparti_b200.autograd import cp_loss
    dims, R = (50, 40, 30), 8
    inds, vals, facs, dt, tf, tv = _setup(dims, 1000, R, 3, cuda)
    loss = cp_loss(dt, tv, tf, rank=R)
    loss.backward()
    L64, _ = _loss64(inds, vals, facs, R)
    assert abs(loss.item() - L64) <= 1e-5 * abs(L64)
    rng = np.random.default_rng(7)
    h = 1e-6
    for k in range(3):
        g = tf[k].grad.detach().cpu().numpy()
        assert np.all(g[:, R:] == 0)
        for _ in range(25):
            i, r = int(rng.integers(dims[k])), int(rng.integers(R))
            fp = [a.astype(np.float64) for a in facs]
            fm = [a.astype(np.float64) for a in facs]
            fp[k][i, r] += h
            fm[k][i, r] -= h
            fd = (_loss64(inds, vals, fp, R)[0] - _loss64(inds, vals, fm, R)[0]) / (2 * h)
            assert abs(g[i, r] - fd) <= 1e-4 * max(1.0, abs(fd)), (k, i, r, g[i, r], fd)
    dt.free()


def test_gradient_matches_reference_mttkrp_of_residual(lib, cuda, ref):
    from hiparti_b200.autograd import cp_loss
    dims, R = (60, 50, 40), 16
    inds, vals, facs, dt, tf, tv = _setup(dims, 3000, R, 5, cuda)
    cp_loss(dt, tv, tf, rank=R).backward()
    _, model = _loss64(inds, vals, facs, R)
    resid = (model - vals.astype(np.float64)).astype(np.float32)  # dL/dmodel
    for k in range(3):
        want = ref.mttkrp_coo(list(dims), inds, resid, facs, R, k)
        got = tf[k].grad.detach().cpu().numpy()
        assert rel_err(got, want) < 1e-4
    dt.free()


def test_gradient_at_scale_vs_oracle(lib, cuda, orc):
    """100,000^3 with 200,000 nonzeros, R = 64 (the gradient workload's shape,
    fewer nonzeros): all three gradients against the oracle's MTTKRP of the
    residual computed on the GPU's own model values."""
    import torch
    from hiparti_b200.autograd import cp_values
    dims, R = (100_000, 100_000, 100_000), 64
    inds, vals, facs, dt, tf, tv = _setup(dims, 200_000, R, 9, cuda)
    model = cp_values(dt, tf, rank=R)
    _, model64 = _loss64(inds, vals, facs, R)
    assert rel_err(model.detach().cpu().numpy(), model64) < 1e-5
    loss = 0.5 * torch.dot(tv - model, tv - model)
    loss.backward()
    resid = (model.detach().cpu().numpy() - vals).astype(np.float32)
    for k in range(3):
        want = orc.mttkrp_coo(inds, resid, facs, R, k)[: dims[k]]
        assert rel_err(tf[k].grad.detach().cpu().numpy(), want) < 1e-5
    dt.free()


@pytest.mark.parametrize("N", [2, 3, 4, 5])
@pytest.mark.parametrize("R", [1, 3, 8, 17, 33, 64, 100, 128, 200])
def test_kruskal_values_every_group_shape(lib, cuda, N, R):
    """The CP model at the nonzeros for every lane-group shape (1 to 32 lanes
    per nonzero, one or two nonzeros in flight per group) and order, against
    an FP64 evaluation; nnz not a multiple of a warp's share, so the last pass
    is partial."""
    import torch
    dims = tuple([60, 50, 40, 30, 20][:N])
    nnz = min(4099, int(np.prod(dims)) // 2)  # 1,500 for the 2-mode case
    inds, vals = synth.uniform_tensor(dims, nnz, seed=10 * N + R)
    nnz = vals.size
    rng = np.random.default_rng(R)
    stride = ((R - 1) // 8 + 1) * 8
    facs = []
    for d in dims:
        a = np.zeros((d, stride), np.float32)
        a[:, :R] = rng.standard_normal((d, R)).astype(np.float32)
        facs.append(a)
    dt = DeviceTensor.from_coo(COOTensor(dims, inds, vals))
    got = dt.kruskal_values([torch.from_numpy(a).to(cuda) for a in facs], rank=R).cpu().numpy()
    model = np.ones((nnz, R))
    for a, ix in zip(facs, inds):
        model *= a[ix, :R].astype(np.float64)
    want = model.sum(1)
    assert rel_err(got, want) < 1e-5
    dt.free()
