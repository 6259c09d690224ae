"""All-at-once gradient CP in PyTorch on top of the device MTTKRP.

``cp_values(tensor, factors)`` evaluates the CP model
    model(z) = sum_r prod_k A_k[i_k(z), r]
at every nonzero z of a device COO tensor.  Its backward is hand-written: the
gradient of a loss with respect to factor k is the mode-k MTTKRP of the
incoming gradient dL/dmodel (for the least-squares loss
0.5 * sum_z (x_z - model(z))^2 that is the residual model - x).  The Hadamard
partials are recomputed inside the MTTKRP kernels rather than stored per
nonzero.  Factors are FP32 CUDA tensors of shape (I_k, stride), stride the
rank rounded up to a multiple of 8 (pad columns stay zero and get zero
gradient).
"""
from __future__ import annotations

import torch

from .api import DeviceTensor


class CPValues(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dt: DeviceTensor, rank: int, *factors):
        factors = [f.contiguous() for f in factors]
        ctx.dt = dt
        ctx.rank = rank
        ctx.save_for_backward(*factors)
        return dt.kruskal_values(factors, rank=rank)

    @staticmethod
    def backward(ctx, grad_model):
        factors = ctx.saved_tensors
        g = grad_model.contiguous().to(torch.float32)
        # the per-mode MTTKRPs are independent: each runs on a stream of its
        # own, so one mode's residual gather overlaps another mode's walk
        cur = torch.cuda.current_stream()
        streams = _side_streams(g.device, len(factors))
        grads = []
        for k, s in enumerate(streams):
            if ctx.needs_input_grad[2 + k]:
                s.wait_stream(cur)
                with torch.cuda.stream(s):
                    grads.append(ctx.dt.mttkrp_values(g, list(factors), k, rank=ctx.rank))
                g.record_stream(s)
                for f in factors:
                    f.record_stream(s)
            else:
                grads.append(None)
        for k, s in enumerate(streams):
            if grads[k] is not None:
                cur.wait_stream(s)
                grads[k].record_stream(cur)
        return (None, None, *grads)


_STREAMS = {}


def _side_streams(device, n):
    """n CUDA streams of `device`, made once and reused."""
    key = (device.index if device.index is not None else torch.cuda.current_device(), n)
    if key not in _STREAMS:
        with torch.cuda.device(key[0]):
            _STREAMS[key] = [torch.cuda.Stream() for _ in range(n)]
    return _STREAMS[key]


def cp_values(dt: DeviceTensor, factors, rank=None):
    """CP model values at the nonzeros of `dt` (differentiable in `factors`)."""
    R = factors[0].shape[1] if rank is None else int(rank)
    return CPValues.apply(dt, R, *factors)


def cp_loss(dt: DeviceTensor, values: torch.Tensor, factors, rank=None):
    """0.5 * sum over nonzeros of (x - model)^2; `values` are the tensor's
    nonzero values in the same order as `dt` was built from."""
    model = cp_values(dt, factors, rank)
    r = values.to(torch.float32) - model
    return 0.5 * torch.dot(r, r)
