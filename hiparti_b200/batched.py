"""Batched CPD-ALS of many small 3-D tensors of uneven size and rank
(ptiB200BatchCreate / ptiB200BatchCpdAls / ptiB200BatchFree).

The reference factors one tensor per ptiCpdAls call (src/sptensor/cpd.c:32-208);
a batch runs the same ALS loop on every tensor, each iteration of the whole
batch being one persistent kernel launch replayed from a CUDA graph.
"""
from __future__ import annotations

import numpy as np

from ._ffi import check, ffi, lib

_PREC = {"fp32": 0, "bf16": 1}


def stride_for(rank: int) -> int:
    """Row stride of a factor matrix of the given rank (a multiple of 8)."""
    return ((int(rank) + 7) // 8) * 8


class Batch:
    """A batch of 3-D COO tensors resident on the GPU, converted to HiCOO with
    per-mode schedules.  tensors: list of (dims, inds, vals) with inds three
    arrays of nnz indices (numpy or CUDA tensors) and vals nnz float32 values;
    ranks: one rank in [1, 32] per tensor; tune: time the block size and the
    columns per lane on this batch (cached per batch shape)."""

    def __init__(self, tensors, ranks, tune=True):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dims = [[int(d) for d in t[0]] for t in tensors]
        self.ranks = [int(r) for r in ranks]
        if len(self.ranks) != len(self.dims):
            raise ValueError("one rank per tensor")
        keep = []
        ind_ptrs, val_ptrs, nnz = [], [], []
        for dims, inds, vals in tensors:
            if len(dims) != 3 or len(inds) != 3:
                raise ValueError("batched CPD takes 3-D tensors")
            di = [torch.as_tensor(np.asarray(i, dtype=np.uint32).view(np.int32)) if not torch.is_tensor(i) else i
                  for i in inds]
            di = [i.to(dev).to(torch.int32).contiguous() for i in di]
            dv = (torch.as_tensor(np.asarray(vals, dtype=np.float32)) if not torch.is_tensor(vals) else vals)
            dv = dv.to(dev).to(torch.float32).contiguous()
            keep += di + [dv]
            ind_ptrs += [ffi.cast("ptiIndex *", i.data_ptr()) for i in di]
            val_ptrs.append(ffi.cast("ptiValue *", dv.data_ptr()))
            nnz.append(dv.numel())
        B = len(self.dims)
        self.nnz = nnz
        d = ffi.new("ptiIndex[]", [x for dims in self.dims for x in dims])
        n = ffi.new("ptiNnzIndex[]", nnz)
        ip = ffi.new("ptiIndex *[]", ind_ptrs)
        vp = ffi.new("ptiValue *[]", val_ptrs)
        rk = ffi.new("ptiIndex[]", self.ranks)
        hp = ffi.new("ptiB200Batch **")
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200BatchCreate(hp, B, d, n, ip, vp, rk, 1 if tune else 0, stream), "ptiB200BatchCreate")
        self._h = hp[0]
        del keep  # the library copied the tensors

    def info(self):
        sb = ffi.new("int *")
        cpl = ffi.new("int *")
        tune = ffi.new("float *")
        setup = ffi.new("float *")
        nt = ffi.new("ptiNnzIndex *")
        check(lib().ptiB200BatchInfo(self._h, sb, cpl, tune, setup, nt), "ptiB200BatchInfo")
        return {"sb_bits": sb[0], "cols_per_lane": cpl[0], "tune_ms": tune[0], "setup_ms": setup[0],
                "ntasks": int(nt[0])}

    def cpd_als(self, factors, niters, precision="bf16", fp32_sweeps=2):
        """factors: per tensor a list of 3 float32 CUDA tensors (I_m, stride_for(R)),
        holding the initial factors; overwritten with the result.  Returns
        (lambdas, fits, ms_per_iter): lambdas a list of float32 CUDA tensors,
        fits a (ntensors, niters) numpy array of every tensor's fit after every
        iteration, ms_per_iter the device time of one iteration of the batch."""
        import torch
        B = len(self.dims)
        if len(factors) != B:
            raise ValueError("one factor set per tensor")
        fptr = []
        for b, fs in enumerate(factors):
            for m, f in enumerate(fs):
                if f.dtype != torch.float32 or not f.is_contiguous() or \
                        tuple(f.shape) != (self.dims[b][m], stride_for(self.ranks[b])):
                    raise ValueError(f"factor ({b}, {m}) must be a contiguous float32 "
                                     f"({self.dims[b][m]}, {stride_for(self.ranks[b])}) tensor")
                fptr.append(ffi.cast("float *", f.data_ptr()))
        dev = factors[0][0].device
        lams = [torch.empty(r, dtype=torch.float32, device=dev) for r in self.ranks]
        lp = ffi.new("float *[]", [ffi.cast("float *", l.data_ptr()) for l in lams])
        fp = ffi.new("float *[]", fptr)
        fits = ffi.new("double[]", B * int(niters))
        ms = ffi.new("float *")
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200BatchCpdAls(self._h, int(niters), _PREC[precision], int(fp32_sweeps), fp, lp, fits, ms,
                                       stream), "ptiB200BatchCpdAls")
        f = np.frombuffer(ffi.buffer(fits, B * int(niters) * 8), dtype=np.float64).reshape(B, int(niters)).copy()
        return lams, f, float(ms[0])

    def free(self):
        if getattr(self, "_h", None) is not None:
            lib().ptiB200BatchFree(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
