"""Benchmark: sparse HiCOO MTTKRP throughput on B200 (and CPD-ALS s/iter).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mttkrp|cpd]

Default workload (mttkrp): 3rd-order tensor 200,000 x 150,000 x 20,000 with
50M unique nonzeros, each mode's index Zipf(s=1.1) over a seeded permutation,
values U(0,1) FP32; HiCOO sb=7 (sk=10, sc=14); FP32 factors U(0,1), R=32.
One step = MTTKRP of all 3 modes.  The metric is algorithmic GB/s:
    B(mode) = nnz*(N + 4) + nb*(8 + 4N) + 4*R*sum_m I_m
(indices 1 B/mode + value, bptr + block indices, N-1 factor reads + 1 output).

The timed tensor (0.8 GB) is larger than the 126 MB L2, so steps are not
served from L2.  With --gpus N (torchrun) every rank runs its own replica of
the workload (the path does not shard; no collective), value = all ranks'
bytes / max time.

--impl reference times the reference's own OpenMP CPU code (oracle/_ref,
compiled from the reference sources) on the same 50M-nonzero tensor.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

C2_DIMS = (200_000, 150_000, 20_000)
C2_NNZ = 50_000_000
C2_R = 32
C2_SB, C2_SK, C2_SC = 7, 10, 14
C3_DIMS = (20_000, 20_000, 20_000, 500)
C3_NNZ = 40_000_000
C3_R = 32
C3_ITERS = 50
LOWRANK_R = 10  # rank of the C3-sized low-rank precision block (its planted rank)
SEED = 2024


def hicoo_bytes(nnz, nb, dims, R, N, fsize=4):
    return nnz * (N + 4) + nb * (8 + 4 * N) + fsize * R * sum(dims)


def factor_match_score(lam_a, facs_a, lam_b, facs_b):
    """Factor match score of two CP models (Acar et al.): the components are
    paired by the best assignment of the product over modes of the absolute
    column cosines; each pair scores that product times
    1 - |lambda_a - lambda_b| / max(lambda_a, lambda_b); the score is the mean
    over components (1 = the same model)."""
    from scipy.optimize import linear_sum_assignment
    R = len(lam_a)
    sim = np.ones((R, R))
    for A, B in zip(facs_a, facs_b):
        A = np.asarray(A, np.float64)[:, :R]
        B = np.asarray(B, np.float64)[:, :R]
        na = np.linalg.norm(A, axis=0)
        nb = np.linalg.norm(B, axis=0)
        sim *= np.abs(A.T @ B) / np.maximum(np.outer(na, nb), 1e-300)
    rows, cols = linear_sum_assignment(-sim)
    la, lb = np.abs(np.asarray(lam_a, np.float64)), np.abs(np.asarray(lam_b, np.float64))
    pen = 1.0 - np.abs(la[rows] - lb[cols]) / np.maximum(np.maximum(la[rows], lb[cols]), 1e-300)
    return float(np.mean(sim[rows, cols] * pen))


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch recorded from an ncu capture in profiles/<name>."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_full_size:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """Samples nvidia-smi every 200 ms while active."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    from hiparti_b200 import replicas
    return replicas.setup("nccl")


def barrier(world):
    from hiparti_b200 import replicas
    replicas.barrier(world)


def max_over_ranks(x, world):
    from hiparti_b200 import replicas
    return replicas.max_over_ranks(x, world)


def make_c2(device, seed, nnz=C2_NNZ):
    """C2 tensor on the device: torch COO -> device HiCOO (GPU conversion)."""
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.synth import coords_torch
    inds = coords_torch(C2_DIMS, nnz, seed, zipf_s=1.1, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1)
    vals = torch.rand(nnz, generator=g, device=device, dtype=torch.float32)
    coo = DeviceTensor.from_torch_coo(C2_DIMS, inds, vals)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = coo.to_hicoo(C2_SB, C2_SK, C2_SC)
    torch.cuda.synchronize()
    conv_s = time.perf_counter() - t0
    return coo, h, inds, vals, conv_s


def c2_factors(device, seed):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed + 2)
    stride = ((C2_R - 1) // 8 + 1) * 8
    return [torch.rand((d, stride), generator=g, device=device, dtype=torch.float32) for d in C2_DIMS]


def make_c3(device, seed):
    """C3: 4-D 20000^3 x 500, 40M unique uniform coordinates; values of a
    planted rank-10 Kruskal model (|N(0,1)| entries, unit-norm columns,
    weights U(1,10)) plus N(0, 0.01^2) noise (0.01 read as the standard
    deviation)."""
    import torch
    from hiparti_b200.synth import coords_torch
    inds = coords_torch(C3_DIMS, C3_NNZ, seed, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 3)
    rank = 10
    lam = torch.rand(rank, generator=g, device=device, dtype=torch.float64) * 9 + 1
    model = lam.expand(C3_NNZ, rank).clone()
    for d, ix in zip(C3_DIMS, inds):
        a = torch.randn((d, rank), generator=g, device=device, dtype=torch.float64).abs_()
        a /= a.norm(dim=0, keepdim=True)
        model *= a[ix.long()]
    noise = torch.randn(C3_NNZ, generator=g, device=device, dtype=torch.float64) * 0.01
    vals = (model.sum(1) + noise).float()
    del model, noise
    return inds, vals


def run_cpd(args):
    """C3 CPD-ALS: FP32 factors vs BF16 factors for the MTTKRP gathers (FP32
    accumulation, FP64 Grams/solves; the last fp32_sweeps iterations in FP32),
    same start; final fits against the FP64 oracle from the same start."""
    import torch
    from hiparti_b200 import DeviceTensor
    dev = torch.device("cuda", torch.cuda.current_device())
    inds, vals = make_c3(dev, SEED + 7)
    coo = DeviceTensor.from_torch_coo(C3_DIMS, inds, vals)
    t = coo.to_hicoo(7, 10, 14) if args.cpd_format == "hicoo" else coo
    t.prepare()
    stride = ((C3_R - 1) // 8 + 1) * 8
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 8)
    init = [torch.rand((d, stride), generator=g, device=dev, dtype=torch.float32) for d in C3_DIMS]
    for a in init:
        a[:, C3_R:] = 0
    out = {"workload": f"C3 CPD-ALS: 4-D 20000^3x500, 40M nnz planted rank-10 + N(0,0.01^2), R={C3_R}, "
                       f"{args.cpd_iters} iterations, {args.cpd_format.upper()} tensor",
           "iters": args.cpd_iters, "fp32_sweeps": args.fp32_sweeps}
    results = {}
    for prec in ["fp32", "bf16"]:
        # one warm-up iteration, then the timed run from the same start
        fac = [a.clone() for a in init]
        t.cpd_als(fac, 1, rank=C3_R, precision=prec, fp32_sweeps=1 if prec == "fp32" else 0)
        fac = [a.clone() for a in init]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam, fits = t.cpd_als(fac, args.cpd_iters, rank=C3_R, precision=prec,
                              fp32_sweeps=args.fp32_sweeps if prec == "bf16" else args.cpd_iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        results[prec] = (dt / args.cpd_iters, fits[-1], lam.cpu().numpy(), [f[:, :C3_R].cpu().numpy() for f in fac])
        out[f"s_per_iter_{prec}"] = round(dt / args.cpd_iters, 6)
        out[f"fit_{prec}"] = fits[-1]
    out["speedup_bf16_vs_fp32"] = round(results["fp32"][0] / results["bf16"][0], 3)
    if args.cpd_oracle:
        from oracle.oracle import Orc, ensure_built
        ensure_built(ref=False)
        orc = Orc()
        t0 = time.perf_counter()
        o = orc.cpd_als(list(C3_DIMS), [i.cpu().numpy().astype(np.uint32) for i in inds], vals.cpu().numpy(),
                        C3_R, args.cpd_iters, [a[:, :C3_R].cpu().numpy() for a in init])
        out["fit_fp64_oracle"] = o["fit"]
        out["oracle_s"] = round(time.perf_counter() - t0, 1)
        out["fit_diff_fp32"] = abs(results["fp32"][1] - o["fit"])
        out["fit_diff_bf16"] = abs(results["bf16"][1] - o["fit"])
        for prec in ["fp32", "bf16"]:
            out[f"fms_{prec}_vs_oracle"] = round(factor_match_score(results[prec][2], results[prec][3],
                                                                    o["lambda_"], o["factors"]), 6)
    coo.free()
    if t is not coo:
        t.free()
    return out


def run_cpd_lowrank(args):
    """BF16 precision at the C3 size on a tensor whose fit is far from 0: a
    4-D 20000^3x500 sparse tensor of exact CP rank 10 (each component on 45
    rows of every mode, so about 41M nonzeros) plus N(0, 0.1^2) on the
    nonzeros, R = 10 (the planted rank, where the ALS problem is well posed;
    with R = 32 the surplus components leave the normal equations so
    ill-conditioned that even FP32 and FP64 runs part ways), 50 iterations
    from the planted factors perturbed by 30%: FP32 factors, BF16 factors with
    closing FP32 sweeps,
    and the FP64 oracle; fit differences and factor match scores against the
    oracle.  (The C3 construction samples a dense model at random
    coordinates, which leaves a sparse tensor of high rank, so its fits are
    near 0.)"""
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.synth import sparse_lowrank_torch
    dev = torch.device("cuda", torch.cuda.current_device())
    inds, vals, (plam, pfacs) = sparse_lowrank_torch(C3_DIMS, 10, 45, noise=0.1, seed=SEED + 17, device=dev)
    nnz = vals.numel()
    coo = DeviceTensor.from_torch_coo(C3_DIMS, inds, vals)
    t = coo.to_hicoo(7, 10, 14)
    t.prepare()
    R = LOWRANK_R
    stride = ((R - 1) // 8 + 1) * 8
    # start near the planted model (its factors with 30% multiplicative noise
    # plus a little everywhere): the block measures precision, not how ALS
    # fares from a random start (from U(0,1) factors it stalls at a saddle
    # near fit 0.78, where the order of FP32 sums decides whether and when it
    # leaves it)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 18)
    init = []
    for f in pfacs:
        a = torch.zeros((f.shape[0], stride), device=dev, dtype=torch.float32)
        noise = 1 + 0.3 * torch.randn(f.shape, generator=g, device=dev, dtype=torch.float64)
        a[:, :R] = (f * noise + 0.01 * torch.rand(f.shape, generator=g, device=dev, dtype=torch.float64)).float()
        init.append(a)
    out = {"workload": f"4-D 20000^3x500 sparse tensor of CP rank 10 (45 rows per component and mode) + "
                       f"N(0,0.1^2), {nnz} nnz, R={R}, {args.cpd_iters} iterations from the planted factors with "
                       f"30% noise, HICOO tensor",
           "nnz": int(nnz), "iters": args.cpd_iters, "fp32_sweeps": args.fp32_sweeps}
    res = {}
    for prec in ["fp32", "bf16"]:
        fac = [a.clone() for a in init]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam, fits = t.cpd_als(fac, args.cpd_iters, rank=R, precision=prec,
                              fp32_sweeps=args.fp32_sweeps if prec == "bf16" else args.cpd_iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[prec] = (fits[-1], lam.cpu().numpy(), [f[:, :R].cpu().numpy() for f in fac])
        out[f"fit_{prec}"] = fits[-1]
        out[f"s_per_iter_{prec}"] = round(dt / args.cpd_iters, 6)
    out["fms_bf16_vs_fp32"] = round(factor_match_score(res["bf16"][1], res["bf16"][2], res["fp32"][1],
                                                       res["fp32"][2]), 6)
    if args.cpd_oracle:
        from oracle.oracle import Orc, ensure_built
        ensure_built(ref=False)
        orc = Orc()
        t0 = time.perf_counter()
        o = orc.cpd_als(list(C3_DIMS), [i.cpu().numpy().astype(np.uint32) for i in inds], vals.cpu().numpy(),
                        R, args.cpd_iters, [a[:, :R].cpu().numpy() for a in init])
        out["oracle_s"] = round(time.perf_counter() - t0, 1)
        out["fit_fp64_oracle"] = o["fit"]
        for prec in ["fp32", "bf16"]:
            out[f"fit_diff_{prec}"] = abs(res[prec][0] - o["fit"])
            out[f"fms_{prec}_vs_oracle"] = round(factor_match_score(res[prec][1], res[prec][2], o["lambda_"],
                                                                    o["factors"]), 6)
    coo.free()
    t.free()
    return out


C4_DIMS = (100_000, 100_000, 100_000)
C4_NNZ = 20_000_000
C4_R = 64


def run_gradcp(args):
    """C4 gradient CP: 100,000^3, 20M uniform nonzeros, values of a planted
    rank-16 model (|N(0,1)| entries, unit-norm columns, weights U(1,10)) plus
    N(0, 0.05^2) noise; R=64 FP32 factors N(0, 0.1).  One step = loss
    0.5*sum (x - model)^2 at the nonzeros + backward (3 residual MTTKRPs)."""
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.autograd import cp_loss
    from hiparti_b200.synth import coords_torch
    dev = torch.device("cuda", torch.cuda.current_device())
    inds = coords_torch(C4_DIMS, C4_NNZ, SEED + 11, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 12)
    lam = torch.rand(16, generator=g, device=dev, dtype=torch.float64) * 9 + 1
    model = lam.expand(C4_NNZ, 16).clone()
    for d, ix in zip(C4_DIMS, inds):
        a = torch.randn((d, 16), generator=g, device=dev, dtype=torch.float64).abs_()
        a /= a.norm(dim=0, keepdim=True)
        model *= a[ix.long()]
    vals = (model.sum(1) + 0.05 * torch.randn(C4_NNZ, generator=g, device=dev, dtype=torch.float64)).float()
    del model
    dt = DeviceTensor.from_torch_coo(C4_DIMS, inds, vals)
    dt.prepare()
    stride = C4_R
    facs = [(0.1 * torch.randn((d, stride), generator=g, device=dev)).requires_grad_(True) for d in C4_DIMS]

    def step():
        for f in facs:
            f.grad = None
        loss = cp_loss(dt, vals, facs, rank=C4_R)
        loss.backward()
        return loss
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k = 5
    e0.record()
    for _ in range(k):
        loss = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    dt.free()
    return {"workload": "C4 gradient CP: 100000^3, 20M nnz planted rank-16 + N(0,0.05^2), R=64 FP32, "
                        "loss + backward (model at nonzeros + 3 residual MTTKRPs)",
            "ms_per_gradient": round(ms, 3), "loss": float(loss.item())}


TTM_R = 16
TTM_REF_NNZ = 2_000_000


def run_ttm(args):
    """TTM of the C2 tensor (50M Zipf nonzeros) with an R = 16 matrix along
    every mode on the GPU (ptiB200TTM; fibers built once per mode, timed
    apart), against the reference's ptiOmpSparseTensorMulMatrix (oracle/_ref,
    all host threads) on a 2M-nonzero sample of the same construction."""
    import numpy as np
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    coo, h, inds, vals, _ = make_c2(dev, SEED + 41)
    h.free()
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 42)
    out = {"workload": f"TTM of the C2 tensor (3-D 200000x150000x20000, 50M Zipf(1.1) nnz), R={TTM_R} FP32, "
                       "each mode", "modes": []}
    peak, _ = measured_peak()
    for mode in range(3):
        U = torch.rand((C2_DIMS[mode], TTM_R), generator=g, device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        finds, Y = coo.ttm(U, mode)  # builds the fibers, then one TTM
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0
        nfib = Y.shape[0]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record()
        for _ in range(reps):
            coo.ttm(U, mode)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        # the kernel's bytes: mode index + value per nonzero, fiber pointers,
        # the factor once, Y written
        algo = C2_NNZ * 8 + (nfib + 1) * 8 + C2_DIMS[mode] * TTM_R * 4 + nfib * Y.shape[1] * 4
        out["modes"].append({"mode": mode, "fibers": int(nfib), "ms": round(ms, 3),
                             "fiber_build_plus_first_s": round(build_s, 3),
                             "algorithmic_GBps": round(algo / ms / 1e6, 1),
                             "frac_of_hbm": round(algo / ms / 1e6 / peak, 3)})
        del finds, Y, U
    out["note"] = ("timed region: ptiB200TTMFibers (cached) + ptiB200TTM per call, through the Python API "
                   "(allocates Y each call)")
    coo.free()
    try:
        from oracle.oracle import Ref
        ref = Ref() if Ref.available() else None
    except Exception:
        ref = None
    if ref is not None:
        sample = np.unique(np.stack([i[:TTM_REF_NNZ].cpu().numpy() for i in inds], 1), axis=0)
        sinds = [sample[:, m].astype(np.uint32) for m in range(3)]
        svals = np.random.default_rng(SEED + 43).random(sample.shape[0]).astype(np.float32)
        U = np.random.default_rng(SEED + 44).random((C2_DIMS[2], TTM_R)).astype(np.float32)
        import ctypes as C
        from oracle.oracle import _Matrix, _SemiSparse
        t, keep = ref._coo(C2_DIMS, sinds, svals)
        st = ((TTM_R - 1) // 8 + 1) * 8
        buf = np.zeros((C2_DIMS[2], st), np.float32)
        buf[:, :TTM_R] = U
        mtx = _Matrix(C2_DIMS[2], TTM_R, C2_DIMS[2], st, buf.ctypes.data)
        Y = _SemiSparse()
        devnull = os.open(os.devnull, os.O_WRONLY)
        saved = os.dup(1)
        os.dup2(devnull, 1)
        try:
            t0 = time.perf_counter()
            ref.L.ptiOmpSparseTensorMulMatrix(C.byref(Y), C.byref(t), C.byref(mtx), C.c_uint32(2))
            ref_s = time.perf_counter() - t0
        finally:
            os.dup2(saved, 1)
            os.close(devnull)
            os.close(saved)
        out["reference_cpu"] = {"kind": "reference", "cores": os.cpu_count(), "mode": 2,
                                "sample": f"{sample.shape[0]} unique nonzeros of the same construction, "
                                          "ptiOmpSparseTensorMulMatrix incl. its sort and fiber build",
                                "s": round(ref_s, 3), "Mnnz_per_s": round(sample.shape[0] / ref_s / 1e6, 2)}
    return out


def run_c2_sk20(args):
    """The C2 tensor converted with sk = 20 (one HiCOO kernel, the setting of
    the reference's single-kernel sweeps) instead of sk = 10: conversion time
    and the all-mode MTTKRP time.  The MTTKRP schedule is built from blocks,
    so sk should change the conversion's kernel pointers and schedule only."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    coo, h, inds, vals, conv10 = make_c2(dev, SEED)
    facs = c2_factors(dev, SEED)
    out = {"workload": "C2 HiCOO MTTKRP with sk=20 (single kernel) against sk=10, sb=7, R=32 FP32"}
    for sk, t in ((10, h), (20, None)):
        if t is None:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            t = coo.to_hicoo(C2_SB, 20, C2_SC)
            torch.cuda.synchronize()
            conv = time.perf_counter() - t0
        else:
            conv = conv10
        t.prepare()
        for m in range(3):
            t.mttkrp(facs, m, rank=C2_R)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            for m in range(3):
                t.mttkrp(facs, m, rank=C2_R)
        e1.record()
        torch.cuda.synchronize()
        out[f"sk{sk}"] = {"conversion_s": round(conv, 4), "mttkrp_ms_all_modes": round(e0.elapsed_time(e1) / 5, 3),
                          "nb": t.nb}
        t.free()
    coo.free()
    return out


RENUM_REF_NNZ = 200_000


def run_renumber(args):
    """Lexi-order renumbering (one iteration) of the C2 tensor on the GPU: the
    HiCOO block count and the all-mode MTTKRP time before and after, the
    renumbering time, and the reference's orderit (oracle/_ref, CPU) against
    the GPU on a 200k-nonzero sample of the same construction."""
    import numpy as np
    import torch
    from hiparti_b200 import COOTensor
    dev = torch.device("cuda", torch.cuda.current_device())
    coo, h, inds, vals, _ = make_c2(dev, SEED + 31)
    facs = c2_factors(dev, SEED + 31)

    def mttkrp_ms(t):
        for m in range(3):
            t.prepare(m)
        for m in range(3):
            t.mttkrp(facs, m, rank=C2_R)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            for m in range(3):
                t.mttkrp(facs, m, rank=C2_R)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 3

    out = {"workload": "Lexi-order renumbering, 1 iteration, of the C2 tensor (3-D 200000x150000x20000, 50M "
                       "Zipf(1.1) nnz); HiCOO sb=7; MTTKRP R=32 FP32, all 3 modes"}
    nb0, ms0 = h.nb, mttkrp_ms(h)
    h.free()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    coo.renumber(1, apply=True)
    torch.cuda.synchronize()
    ren_s = time.perf_counter() - t0
    h2 = coo.to_hicoo(C2_SB, C2_SK, C2_SC)
    nb1, ms1 = h2.nb, mttkrp_ms(h2)
    h2.free()
    coo.free()
    out.update({"s_renumber_gpu": round(ren_s, 3), "nb_before": nb0, "nb_after": nb1,
                "nnz_per_block_before": round(C2_NNZ / nb0, 2), "nnz_per_block_after": round(C2_NNZ / nb1, 2),
                "mttkrp_ms_all_modes_before": round(ms0, 3), "mttkrp_ms_all_modes_after": round(ms1, 3)})
    try:
        from oracle.oracle import Ref
        ref = Ref() if Ref.available() else None
    except Exception:
        ref = None
    if ref is not None:
        sample = [i[:RENUM_REF_NNZ].cpu().numpy() for i in inds]
        keys = np.unique(np.stack(sample, 1), axis=0)  # orderit wants unique coordinates
        sinds = [keys[:, m].astype(np.uint32) for m in range(3)]
        svals = np.ones(keys.shape[0], np.float32)
        import os as _os
        t0 = time.perf_counter()
        devnull = _os.open(_os.devnull, _os.O_WRONLY)
        saved = _os.dup(1)
        _os.dup2(devnull, 1)  # the reference prints per-mode timings
        try:
            want = ref.orderit(C2_DIMS, sinds, svals, 1)
        finally:
            _os.dup2(saved, 1)
            _os.close(devnull)
            _os.close(saved)
        ref_s = time.perf_counter() - t0
        small = COOTensor(C2_DIMS, sinds, svals)
        small.renumber(1)  # warm-up
        t0 = time.perf_counter()
        small.renumber(1)
        ours_s = time.perf_counter() - t0
        # (Zipf data has many indices with equal row lists, whose relative
        # order the reference leaves to its quicksort; parity is tested on
        # tensors where the order is unique.)
        del want
        out["sample"] = {"nnz": int(keys.shape[0]), "kind": "reference", "cores": 1,
                         "s_reference_orderit_cpu": round(ref_s, 3), "s_ours_gpu_incl_copies": round(ours_s, 4),
                         "speedup": round(ref_s / ours_s, 1)}
    out["bfs_like"] = run_bfs_like(inds, args.bfs_nnz)
    return out


def run_bfs_like(inds, nnz):
    """BFS-like renumbering (ptiIndexRenumber, renumber = 2) beside one
    Lexi-order pass on the first `nnz` nonzeros of the C2 tensor: HiCOO block
    counts (sb = 7) before and after each, and the time of each call.  The
    BFS-like walk is a priority queue whose every step depends on the last, so
    it runs on the host over vertex lists built on the GPU."""
    import numpy as np
    from hiparti_b200 import COOTensor, DeviceTensor
    part = [i[:nnz].cpu().numpy().view(np.uint32).copy() for i in inds]
    vals = np.ones(part[0].size, np.float32)
    t = COOTensor(C2_DIMS, part, vals)

    def nb_of(maps):
        u = t.shuffled(maps) if maps is not None else COOTensor(C2_DIMS, [p.copy() for p in part], vals.copy())
        d = DeviceTensor.from_coo(u)
        h = d.to_hicoo(C2_SB, C2_SK, C2_SC)
        nb = h.nb
        h.free()
        d.free()
        return nb

    t0 = time.perf_counter()
    bfs = t.renumber(method="bfs")
    bfs_s = time.perf_counter() - t0
    t.renumber(1)  # warm-up
    t0 = time.perf_counter()
    lexi = t.renumber(1)
    lexi_s = time.perf_counter() - t0
    nb0, nb_b, nb_l = nb_of(None), nb_of(bfs), nb_of(lexi)
    return {"workload": f"first {part[0].size} nonzeros of the C2 tensor, HiCOO sb=7", "nb_before": nb0,
            "nb_after_bfs_like": nb_b, "nb_after_lexi_1_iteration": nb_l,
            "nnz_per_block": {"before": round(part[0].size / nb0, 2), "bfs_like": round(part[0].size / nb_b, 2),
                              "lexi": round(part[0].size / nb_l, 2)},
            "s_bfs_like_incl_copies": round(bfs_s, 3), "s_lexi_gpu_incl_copies": round(lexi_s, 4)}


INGEST_NNZ = 10_000_000
INGEST_REF_NNZ = 1_000_000


def write_tns_fixed(path, dims, inds, vals_u6):
    """Writes a .tns file with fixed-width fields: 1-based indices zero-padded
    to the widest mode size and values "0.dddddd" (vals_u6 = int(v * 1e6)).
    fscanf reads leading zeros like any other digits."""
    import numpy as np
    cols = []
    for d, ix in zip(dims, inds):
        w = len(str(d))
        pw = 10 ** np.arange(w - 1, -1, -1, dtype=np.int64)
        cols.append((((ix.astype(np.int64) + 1)[:, None] // pw) % 10 + 48).astype(np.uint8))
        cols.append(np.full((ix.size, 1), 32, np.uint8))
    pw = 10 ** np.arange(5, -1, -1, dtype=np.int64)
    cols.append(np.tile(np.frombuffer(b"0.", np.uint8), (vals_u6.size, 1)))
    cols.append(((vals_u6.astype(np.int64)[:, None] // pw) % 10 + 48).astype(np.uint8))
    cols.append(np.full((vals_u6.size, 1), 10, np.uint8))
    body = np.concatenate(cols, axis=1)
    with open(path, "wb") as f:
        f.write(f"{len(dims)}\n{' '.join(map(str, dims))}\n".encode())
        f.write(body.tobytes())


def run_ingest(args):
    """GPU tensor ingest: a 10M-nonzero .tns file with the C2 construction's
    dims and Zipf(1.1) coordinates (fixed-width text, U(0,1) values with six
    decimals) loaded by ptiB200LoadSparseTensor from the page cache into device
    memory; the reference's fscanf loader (oracle/_ref, compiled from
    src/sptensor/load.c) timed on a 1M-nonzero file of the same construction."""
    import tempfile
    import time
    import numpy as np
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.synth import coords_torch
    dev = torch.device("cuda", torch.cuda.current_device())
    out = {"workload": f"ingest: .tns text, 3-D {C2_DIMS[0]}x{C2_DIMS[1]}x{C2_DIMS[2]}, Zipf(1.1) coordinates, "
                       f"{INGEST_NNZ} nnz, file in the page cache -> device COO tensor"}
    with tempfile.TemporaryDirectory() as tmp:
        inds = [i.cpu().numpy() for i in coords_torch(C2_DIMS, INGEST_NNZ, SEED + 21, zipf_s=1.1, device=dev)]
        rng = np.random.default_rng(SEED + 22)
        vals = rng.integers(0, 1_000_000, INGEST_NNZ)
        path = f"{tmp}/c2_10m.tns"
        write_tns_fixed(path, C2_DIMS, inds, vals)
        size = os.path.getsize(path)
        times = []
        for _ in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            t = DeviceTensor.load(path)
            times.append(time.perf_counter() - t0)
            t.free()
        sec = sorted(times[1:])[len(times[1:]) // 2]
        out.update({"file_bytes": size, "nnz": INGEST_NNZ, "s_load": round(sec, 4),
                    "GBps": round(size / sec / 1e9, 3), "Mnnz_per_s": round(INGEST_NNZ / sec / 1e6, 1)})
        t = DeviceTensor.load(path, dedupe=True)
        info_inds, _ = t.coo_arrays()
        out["unique_nnz"] = int(info_inds[0].size)
        t.free()
        try:
            from oracle.oracle import Ref
            ref = Ref() if Ref.available() else None
        except Exception:
            ref = None
        if ref is not None:
            rpath = f"{tmp}/c2_1m.tns"
            write_tns_fixed(rpath, C2_DIMS, [i[:INGEST_REF_NNZ] for i in inds], vals[:INGEST_REF_NNZ])
            rsize = os.path.getsize(rpath)
            t0 = time.perf_counter()
            rc, _, rinds, _ = ref.load(rpath, 1)
            rsec = time.perf_counter() - t0
            if rc == 0:
                out["reference_cpu"] = {"kind": "reference", "cores": 1, "sample": f"first {INGEST_REF_NNZ} nonzeros "
                                        "of the same file construction, ptiLoadSparseTensor (fscanf)",
                                        "file_bytes": rsize, "s_load": round(rsec, 3),
                                        "GBps": round(rsize / rsec / 1e9, 4)}
                out["speedup_vs_reference"] = round(out["GBps"] / out["reference_cpu"]["GBps"], 1)
    return out


C5_TENSORS = 256
C5_ITERS = 20


def make_c5(device, seed):
    """C5: 256 3-D tensors, each mode's size U{50..5000}, nnz log-uniform in
    [1e3, 1e6] (at most a quarter of the tensor's cells), unique uniform
    coordinates, values U(0,1); ranks drawn from {8, 16, 32}."""
    import torch
    from hiparti_b200.synth import coords_torch
    rng = np.random.default_rng(seed)
    tensors, ranks = [], []
    for b in range(C5_TENSORS):
        dims = tuple(int(x) for x in rng.integers(50, 5001, 3))
        nnz = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        nnz = min(nnz, int(np.prod(dims, dtype=np.float64)) // 4)
        inds = coords_torch(dims, nnz, seed * 1000 + b, device=device)
        g = torch.Generator(device=device)
        g.manual_seed(seed * 1000 + b + 500)
        vals = torch.rand(nnz, generator=g, device=device, dtype=torch.float32)
        tensors.append((dims, inds, vals))
        ranks.append(int(rng.choice([8, 16, 32])))
    return tensors, ranks


def run_batched(args):
    """C5 batched uneven CPD-ALS: 256 tensors factored together, one
    persistent launch per iteration of the whole batch replayed from a CUDA
    graph, block size and columns per lane autotuned; FP32 and BF16 (two
    closing FP32 sweeps) from the same U(0,1) start; fits of a sample of the
    tensors against the FP64 oracle from the same start; the same FP32 ALS
    run tensor by tensor through ptiB200CpdAls for comparison."""
    import torch
    from hiparti_b200 import DeviceTensor
    from hiparti_b200.batched import Batch, stride_for
    dev = torch.device("cuda", torch.cuda.current_device())
    iters = args.batched_iters
    tensors, ranks = make_c5(dev, SEED + 21)
    total_nnz = sum(int(v.numel()) for _, _, v in tensors)
    bt = Batch(tensors, ranks, tune=True)
    info = bt.info()
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 22)
    init = []
    for (dims, _, _), R in zip(tensors, ranks):
        fs = []
        for d in dims:
            a = torch.rand((d, stride_for(R)), generator=g, device=dev, dtype=torch.float32)
            a[:, R:] = 0
            fs.append(a)
        init.append(fs)
    out = {"workload": f"C5 batched CPD-ALS: {C5_TENSORS} 3-D tensors, dims U{{50..5000}}, nnz log-U[1e3,1e6] "
                       f"(total {total_nnz}), U(0,1) values, ranks from {{8,16,32}}, {iters} iterations",
           "total_nnz": total_nnz, "sb_bits": info["sb_bits"], "cols_per_lane_bf16": info["cols_per_lane"],
           "tasks_per_iter": info["ntasks"], "tune_s": round(info["tune_ms"] / 1e3, 3),
           "setup_s": round(info["setup_ms"] / 1e3, 3)}
    fits, models = {}, {}
    for prec in ["fp32", "bf16"]:
        facs = [[a.clone() for a in fs] for fs in init]
        bt.cpd_als(facs, 2, precision=prec, fp32_sweeps=1)  # warm-up
        facs = [[a.clone() for a in fs] for fs in init]
        lams, f, ms = bt.cpd_als(facs, iters, precision=prec, fp32_sweeps=2 if prec == "bf16" else iters)
        fits[prec] = f[:, -1]
        models[prec] = (lams, facs)
        out[f"ms_per_iter_{prec}"] = round(ms, 4)
        # MTTKRP work of one iteration: every nonzero of every tensor, 3 modes
        out[f"gnnz_modes_per_s_{prec}"] = round(3 * total_nnz / (ms * 1e-3) / 1e9, 2)
    out["speedup_bf16_vs_fp32"] = round(out["ms_per_iter_fp32"] / out["ms_per_iter_bf16"], 3)
    bt.free()
    if args.batched_sequential:
        # the same FP32 ALS, one ptiB200CpdAls call (HiCOO, sb 7) per tensor
        dts = [DeviceTensor.from_torch_coo(d, i, v).to_hicoo(7, 7, 7) for d, i, v in tensors]
        for t in dts:
            t.prepare()
        facs = [[a.clone() for a in fs] for fs in init]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t, fs, R in zip(dts, facs, ranks):
            t.cpd_als(fs, iters, rank=R)
        torch.cuda.synchronize()
        out["ms_per_iter_fp32_tensor_by_tensor"] = round((time.perf_counter() - t0) * 1e3 / iters, 3)
        for t in dts:
            t.free()
    if args.batched_oracle > 0:
        from oracle.oracle import Orc, ensure_built
        ensure_built(ref=False)
        orc = Orc()
        order = np.argsort([int(v.numel()) for _, _, v in tensors])
        pick = order[np.linspace(0, len(order) - 1, min(args.batched_oracle, len(order))).round().astype(int)]
        t0 = time.perf_counter()
        d32, d16, f32s, f16s = [], [], [], []
        for b in pick:
            dims, inds, vals = tensors[b]
            R = ranks[b]
            o = orc.cpd_als(list(dims), [i.cpu().numpy().astype(np.uint32) for i in inds], vals.cpu().numpy(), R,
                            iters, [a[:, :R].cpu().numpy() for a in init[b]])
            d32.append(abs(fits["fp32"][b] - o["fit"]))
            d16.append(abs(fits["bf16"][b] - o["fit"]))
            for prec, acc in (("fp32", f32s), ("bf16", f16s)):
                lams, facs = models[prec]
                acc.append(factor_match_score(lams[b].cpu().numpy(), [x[:, :R].cpu().numpy() for x in facs[b]],
                                              o["lambda_"], o["factors"]))
        out["oracle_tensors"] = int(len(pick))
        out["oracle_s"] = round(time.perf_counter() - t0, 1)
        out["max_fit_diff_fp32"] = float(max(d32))
        out["max_fit_diff_bf16"] = float(max(d16))
        out["min_fms_fp32_vs_oracle"] = round(float(min(f32s)), 6)
        out["min_fms_bf16_vs_oracle"] = round(float(min(f16s)), 6)
    out["fit_bf16_min_max"] = [float(fits["bf16"].min()), float(fits["bf16"].max())]
    return out


def pool_used_bytes():
    """Bytes in use in the current device's default memory pool (the pool the
    library's cudaMallocAsync draws from), or None where it cannot be read."""
    import torch
    try:
        from cuda.bindings import driver as drv
        err, pool = drv.cuDeviceGetDefaultMemPool(torch.cuda.current_device())
        if err != drv.CUresult.CUDA_SUCCESS:
            return None
        err, v = drv.cuMemPoolGetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
        return int(v) if err == drv.CUresult.CUDA_SUCCESS else None
    except Exception:
        return None


def run_ours_mttkrp(args, rank, world):
    import torch
    from hiparti_b200 import HiCOOTensor, ffi, lib
    dev = torch.device("cuda", torch.cuda.current_device())
    nnz = args.nnz
    coo, h, inds, vals, conv_s = make_c2(dev, SEED + rank, nnz)
    nb = h.nb
    mats = c2_factors(dev, SEED + rank)
    stride = mats[0].shape[1]
    N = 3
    # per-mode schedules (built once per tensor, reused by every MTTKRP)
    torch.cuda.synchronize()
    used_before = pool_used_bytes()
    t0 = time.perf_counter()
    h.prepare()
    torch.cuda.synchronize()
    prep_s = time.perf_counter() - t0
    used_after = pool_used_bytes()
    # device memory the three schedules hold (the library allocates from the
    # device's default memory pool; freed temporaries do not count)
    schedule_bytes = used_after - used_before if used_before is not None and used_after is not None else None
    outs = [torch.empty((d, stride), dtype=torch.float32, device=dev) for d in C2_DIMS]
    bytes_mode = [hicoo_bytes(nnz, nb, C2_DIMS, C2_R, N) for _ in range(N)]
    step_bytes = sum(bytes_mode)
    stream = torch.cuda.current_stream()

    def step(ev=None):
        for m in range(N):
            if ev is not None:
                ev[m][0].record(stream)
            h.mttkrp(mats, m, rank=C2_R, out=outs[m])
            if ev is not None:
                ev[m][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    ev = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(N)] for _ in range(args.steps)]
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        step(ev[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms_total = t_start.elapsed_time(t_end)
    ms_total = max_over_ranks(ms_total, world)
    ms_step = ms_total / args.steps
    per_mode_ms = [statistics.mean(ev[k][m][0].elapsed_time(ev[k][m][1]) for k in range(args.steps))
                   for m in range(N)]
    value = step_bytes * world * args.steps / (ms_total * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    mean_launch_ms = statistics.mean(per_mode_ms)
    achieved = statistics.mean(bytes_mode[m] / (per_mode_ms[m] * 1e-3) / 1e9 for m in range(N))
    traffic = profile_traffic("hicoo_mttkrp_c2.txt")

    # ---- the gathers against the L2 read bandwidth measured here ----
    gather = None
    try:
        gb = ffi.new("double *")
        if lib().ptiB200ProbeL2ReadBandwidth(64 << 20, 50, gb) == 0:
            gathered = (N - 1) * C2_R * 4 * nnz  # two factor rows of R FP32 values per nonzero
            g_achieved = gathered / (mean_launch_ms * 1e-3) / 1e9
            gather = {"bound": "l2", "gathered_bytes_per_launch": gathered, "achieved": round(g_achieved, 1),
                      "peak": round(gb[0], 1), "unit": "GB/s", "frac": round(g_achieved / gb[0], 4),
                      "peak_source": "ptiB200ProbeL2ReadBandwidth: 64 MiB streamed 50 times with 16-byte L2-only "
                                     "loads, eight in flight per thread, 2048 threads per SM (this run)",
                      "note": "gathers hit L1 too, so the fraction can exceed 1"}
    except Exception as exc:  # the probe is a side figure; the bench line stands without it
        gather = {"unavailable": str(exc)}

    # ---- end to end through the reference-facing C ABI (host buffers) ----
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(h, inds, vals, mats, nb, args)

    result = {
        "metric": "hicoo_mttkrp_GBps", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Zipf(1.1) coordinates, U(0,1) values and factors)",
        "config": {"workload": f"C2 HiCOO MTTKRP, 3-D 200000x150000x20000, {nnz // 1000000}M nnz Zipf(1.1), "
                               "R=32, sb=7 sk=10 sc=14, FP32, all 3 modes per step",
                   "nnz": nnz, "nb": nb, "prepare_s": round(prep_s, 3), "schedule_device_bytes": schedule_bytes,
                   "rank": C2_R, "modes_per_step": N,
                   "algorithmic_bytes_per_step": step_bytes,
                   "l2": "inputs larger than L2 (tensor 0.8 GB vs 126 MB L2)",
                   "parallelism": f"replicas x{world}", "conversion_s": round(conv_s, 3),
                   "per_mode_ms": [round(x, 4) for x in per_mode_ms]},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs", "kernel": "hicoo_sched_kernel (one launch per mode)",
                     "mean_launch_ms": round(mean_launch_ms, 4)},
        "gather_roofline": gather,
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": N * args.steps,
    }
    return result


def pinned_numpy(arr):
    import torch
    t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype)) if arr.dtype != np.uint32 else torch.int32,
                    pin_memory=True)
    out = t.numpy().view(arr.dtype)
    out[...] = arr
    return out, t


def run_e2e(h_dev, inds, vals, mats, nb, args):
    """The drop-in call ptiMTTKRPHiCOO with host (pinned) buffers: every call
    copies the HiCOO tensor and factors to the device and the result back."""
    import torch
    from hiparti_b200 import COOTensor, HiCOOTensor
    from hiparti_b200.api import _MatrixSet
    from hiparti_b200._ffi import ffi, lib, check
    # HiCOO arrays on the host: bring the device conversion's result back
    host = download_hicoo(h_dev)
    keep = []
    def pin(a):
        p, t = pinned_numpy(a)
        keep.append(t)
        return p
    hh = HiCOOTensor(C2_DIMS, C2_SB, C2_SK, C2_SC, pin(host["bptr"]), [pin(b) for b in host["binds"]],
                     [pin(e) for e in host["einds"]], pin(host["vals"]))
    hmats = [pin(m.cpu().numpy()) for m in mats]
    stride = hmats[0].shape[1]
    out = pin(np.zeros((max(C2_DIMS), stride), np.float32))
    ms = _MatrixSet(hmats + [out], C2_R)
    N = 3
    orders = [ffi.new("ptiIndex[]", [(m + i) % N for i in range(N)]) for m in range(N)]
    L = lib()

    def step():
        for m in range(N):
            check(L.ptiMTTKRPHiCOO(hh.c, ms.ptrs, orders[m], m), "ptiMTTKRPHiCOO")

    for _ in range(max(1, min(args.warmup, 2))):
        step()
    ksteps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(ksteps):
        step()
    dt = (time.perf_counter() - t0) / ksteps
    tensor_bytes = host["bptr"].nbytes + sum(b.nbytes for b in host["binds"]) + \
        sum(e.nbytes for e in host["einds"]) + host["vals"].nbytes
    fac_bytes = [m.nbytes for m in hmats]
    h2d = sum(tensor_bytes + sum(fac_bytes) - fac_bytes[m] for m in range(N))
    d2h = sum(C2_DIMS[m] * stride * 4 for m in range(N))
    step_bytes = N * hicoo_bytes(host["vals"].size, nb, C2_DIMS, C2_R, N)
    # the host link on this box: one pinned host->device copy of the HiCOO
    # value array's size, for reading the e2e figure against
    src = torch.empty(host["vals"].nbytes, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(host["vals"].nbytes, dtype=torch.uint8, device="cuda")
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    link = host["vals"].nbytes / (time.perf_counter() - t1) / 1e9
    del src, dst
    return {"value": round(step_bytes / dt / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": round(dt * 1e3, 3), "steps": ksteps,
            "h2d_link_GBps_measured": round(link, 1),
            "api": "ptiMTTKRPHiCOO (C ABI, host pinned buffers, tensor + factors copied in per call)"}


def download_hicoo(h):
    """Host copies of a device HiCOO tensor's arrays (bptr, binds, einds, vals)."""
    from hiparti_b200._ffi import ffi, lib, check
    info = h.info()
    N, nnz, nb = info["nmodes"], info["nnz"], info["nb"]
    bptr = np.empty(nb + 1, np.uint64)
    binds = [np.empty(nb, np.uint32) for _ in range(N)]
    einds = [np.empty(nnz, np.uint8) for _ in range(N)]
    vals = np.empty(nnz, np.float32)
    bp = ffi.new("ptiNnzIndex **")
    args = ffi.new("void *[]", [ffi.cast("void *", binds[m].ctypes.data) for m in range(N)])
    eargs = ffi.new("void *[]", [ffi.cast("void *", einds[m].ctypes.data) for m in range(N)])
    check(lib().ptiB200DownloadHiCOO(h._h, ffi.cast("ptiNnzIndex *", bptr.ctypes.data), args, eargs,
                                     ffi.cast("ptiValue *", vals.ctypes.data)), "ptiB200DownloadHiCOO")
    return {"bptr": bptr, "binds": binds, "einds": einds, "vals": vals}


def c2_host_tensor(seed=SEED, nnz=C2_NNZ):
    """The C2 tensor and factors exactly as run_ours_mttkrp builds them (same
    generator, same seeds), brought to host memory.  Generation runs on the
    GPU with torch when one is present (de-duplicating 65M coordinates takes
    milliseconds there and minutes with numpy); this is data generation only,
    outside every timed region."""
    import torch
    from hiparti_b200.synth import coords_torch
    dev = torch.device("cuda", torch.cuda.current_device())
    ti = coords_torch(C2_DIMS, nnz, seed, zipf_s=1.1, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    tv = torch.rand(nnz, generator=g, device=dev, dtype=torch.float32)
    inds = [t.cpu().numpy().view(np.uint32) for t in ti]
    vals = tv.cpu().numpy()
    mats = [m.cpu().numpy() for m in c2_factors(dev, seed)]
    del ti, tv
    torch.cuda.empty_cache()
    return inds, vals, mats


def run_reference_arm(args, rank, world):
    """Times the reference's own CPU code (oracle/_ref/libHiParTI.so, built
    from its sources) on the benchmark workload itself: the 50M-nonzero C2
    tensor of run_ours_mttkrp (same seeds), converted by the reference's
    ptiSparseTensorToHiCOO(tk=1) (untimed, as the reference's driver
    benchmark/tensor/mttkrp_hicoo.c converts before its timed loop), then
    ptiOmpMTTKRPHiCOO with every host thread, 3 modes per step.  Under torchrun
    rank 0 alone runs; the other ranks return without work."""
    if rank != 0:
        return None
    from oracle.oracle import Ref, ensure_built
    try:
        ensure_built(ref=True)
    except Exception:
        pass
    if not Ref.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref not built (needs its sources)"}
    import torch
    if not torch.cuda.is_available():
        return {"impl": "reference", "unavailable": "the C2 tensor is generated on a CUDA device; none present"}
    ref = Ref()
    threads = os.cpu_count() or 1
    nnz = args.nnz
    t0 = time.perf_counter()
    inds, vals, mats = c2_host_tensor(SEED, nnz)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    h = ref.to_hicoo(list(C2_DIMS), inds, vals, C2_SB, C2_SK, C2_SC)
    conv_s = time.perf_counter() - t0
    del inds, vals
    nb = h["bptr"].size - 1
    run = ref.omp_hicoo_mttkrp_runner(list(C2_DIMS), h, mats, C2_R, threads)
    N = 3
    for _ in range(args.warmup):
        for m in range(N):
            run(m)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for m in range(N):
            run(m)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    step_bytes = N * hicoo_bytes(nnz, nb, C2_DIMS, C2_R, N)
    value = step_bytes / dt / 1e9
    sample_desc = (f"the full workload: {nnz} unique nonzeros of the C2 construction (seed {SEED}, the tensor "
                   f"--impl ours times), nb={nb}; HiCOO built by the reference's ptiSparseTensorToHiCOO(tk=1) "
                   f"in {conv_s:.1f} s, untimed; one step = ptiOmpMTTKRPHiCOO(tk={threads}, tb=1) for modes 0,1,2")
    return {"metric": "hicoo_mttkrp_GBps", "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Zipf(1.1) coordinates, U(0,1) values and factors)", "impl": "reference",
            "config": {"workload": f"C2 HiCOO MTTKRP, 3-D 200000x150000x20000, {nnz // 1000000}M nnz Zipf(1.1), "
                                   "R=32, sb=7 sk=10 sc=14, FP32, all 3 modes per step",
                       "nnz": nnz, "nb": nb, "rank": C2_R, "modes_per_step": N,
                       "algorithmic_bytes_per_step": step_bytes, "generation_s": round(gen_s, 1),
                       "reference_conversion_s": round(conv_s, 2), "parallelism": "reference OpenMP, rank 0"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
                             "sample": sample_desc},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_sample(args):
    """cpu_baseline of our own line: the reference's ptiOmpMTTKRPHiCOO on a
    bounded sample of the C2 construction (rank 0, N = 1), so that the default
    run stays within minutes; the full-size reference run is --impl reference."""
    from oracle.oracle import Ref, ensure_built
    from hiparti_b200.synth import coords_numpy
    try:
        ensure_built(ref=True)
    except Exception:
        pass
    if not Ref.available():
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference library oracle/_ref not built (needs its sources)"}
    ref = Ref()
    threads = os.cpu_count() or 1
    sample = args.ref_sample
    inds = coords_numpy(C2_DIMS, sample, SEED, zipf_s=1.1)
    vals = np.random.default_rng(SEED + 1).random(sample, dtype=np.float32)
    h = ref.to_hicoo(list(C2_DIMS), inds, vals, C2_SB, C2_SK, C2_SC)
    nb = h["bptr"].size - 1
    rng = np.random.default_rng(SEED + 2)
    stride = ((C2_R - 1) // 8 + 1) * 8
    mats = [rng.random((d, stride), dtype=np.float32) for d in C2_DIMS]
    run = ref.omp_hicoo_mttkrp_runner(list(C2_DIMS), h, mats, C2_R, threads)
    N = 3
    for m in range(N):
        run(m)
    t0 = time.perf_counter()
    for m in range(N):
        run(m)
    dt = time.perf_counter() - t0
    value = N * hicoo_bytes(sample, nb, C2_DIMS, C2_R, N) / dt / 1e9
    return {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": (f"{sample} unique nonzeros drawn by the C2 construction (same dims, Zipf(1.1) per mode, "
                       f"U(0,1) values), nb={nb}; HiCOO built by the reference's ptiSparseTensorToHiCOO(tk=1), "
                       f"untimed; one step = ptiOmpMTTKRPHiCOO(tk={threads}, tb=1) for modes 0,1,2")}


C1_DIMS = (1000, 1000, 1000)
C1_NNZ = 1_000_000
C1_R = 16
CPD_SAMPLE_NNZ = 2_000_000


def run_cpu_paths(args):
    """The reference's other CPU paths beside ours on the same bounded inputs
    (rank 0, N = 1): COO->HiCOO conversion of the 4M-nonzero C2 sample
    (ptiSparseTensorToHiCOO(tk=1) against the GPU conversion), the C1 COO
    MTTKRP (ptiOmpMTTKRP with atomics and ptiOmpMTTKRP_Reduce against the
    device COO kernel), and CPD-ALS iterations on a 2M-nonzero sample of the
    C3 construction (OmpCpdAlsStep against ptiB200CpdAls, R = 32)."""
    import numpy as np
    import torch
    from oracle.oracle import Ref
    from hiparti_b200 import COOTensor, DeviceTensor
    from hiparti_b200.synth import coords_numpy, planted_tensor
    if not Ref.available():
        return {"unavailable": "reference library oracle/_ref not built"}
    ref = Ref()
    threads = os.cpu_count() or 1
    out = {"threads": threads}
    dev = torch.device("cuda", torch.cuda.current_device())

    # conversion
    inds = coords_numpy(C2_DIMS, args.ref_sample, SEED, zipf_s=1.1)
    vals = np.random.default_rng(SEED + 1).random(args.ref_sample, dtype=np.float32)
    t0 = time.perf_counter()
    ref.to_hicoo(list(C2_DIMS), inds, vals, C2_SB, C2_SK, C2_SC)
    ref_conv = time.perf_counter() - t0
    coo = DeviceTensor.from_coo(COOTensor(C2_DIMS, inds, vals))
    h = coo.to_hicoo(C2_SB, C2_SK, C2_SC)  # warm-up
    h.free()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = coo.to_hicoo(C2_SB, C2_SK, C2_SC)
    torch.cuda.synchronize()
    ours_conv = time.perf_counter() - t0
    h.free()
    coo.free()
    out["conversion"] = {"sample_nnz": args.ref_sample, "s_reference_tk1": round(ref_conv, 3),
                         "s_ours_gpu_device_resident": round(ours_conv, 4), "speedup": round(ref_conv / ours_conv, 1)}

    # C1 COO MTTKRP, 3 modes
    inds = coords_numpy(C1_DIMS, C1_NNZ, SEED + 51)
    vals = np.random.default_rng(SEED + 52).random(C1_NNZ, dtype=np.float32)
    stride = ((C1_R - 1) // 8 + 1) * 8
    mats = [np.random.default_rng(SEED + 53 + m).random((d, stride), dtype=np.float32) for m, d in enumerate(C1_DIMS)]
    step_bytes = 3 * (C1_NNZ * (3 * 4 + 4) + 4 * C1_R * sum(C1_DIMS))
    res = {}
    for variant in ("omp", "omp_reduce"):
        for m in range(3):  # warm-up
            ref.mttkrp_coo(list(C1_DIMS), inds, vals, mats, C1_R, m, variant=variant, tk=threads)
        t0 = time.perf_counter()
        for m in range(3):
            ref.mttkrp_coo(list(C1_DIMS), inds, vals, mats, C1_R, m, variant=variant, tk=threads)
        res[variant] = time.perf_counter() - t0
    dt = DeviceTensor.from_coo(COOTensor(C1_DIMS, inds, vals))
    facs = [torch.from_numpy(a).to(dev) for a in mats]
    for m in range(3):
        dt.prepare(m)
        dt.mttkrp(facs, m, rank=C1_R)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        for m in range(3):
            dt.mttkrp(facs, m, rank=C1_R)
    e1.record()
    torch.cuda.synchronize()
    ours_ms = e0.elapsed_time(e1) / 10
    dt.free()
    out["coo_mttkrp_c1"] = {"workload": "C1: 3-D 1000^3, 1M uniform nnz, R=16, 3 modes per step",
                            "GBps_reference_omp_atomic": round(step_bytes / res["omp"] / 1e9, 3),
                            "GBps_reference_omp_reduce": round(step_bytes / res["omp_reduce"] / 1e9, 3),
                            "GBps_ours_device": round(step_bytes / ours_ms / 1e6, 1),
                            "ms_ours_per_step": round(ours_ms, 4)}

    # CPD iterations on a C3-construction sample
    dims = C3_DIMS
    inds, vals, _ = planted_tensor(dims, CPD_SAMPLE_NNZ, 10, 0.01, seed=SEED + 61)
    R = C3_R
    rng = np.random.default_rng(SEED + 62)
    init = [rng.random((d, R)).astype(np.float32) for d in dims]
    iters = 3
    t0 = time.perf_counter()
    ref.cpd_als_step(list(dims), inds, vals, R, iters, init, tk=threads)
    ref_iter = (time.perf_counter() - t0) / iters
    dtc = DeviceTensor.from_hicoo(COOTensor(dims, inds, vals).to_hicoo(C2_SB, C2_SK, C2_SC))
    stride = ((R - 1) // 8 + 1) * 8

    def dev_factors():
        fs = []
        for a in init:
            f = torch.zeros((a.shape[0], stride), dtype=torch.float32)
            f[:, :R] = torch.from_numpy(a)
            fs.append(f.to(dev))
        return fs
    dtc.cpd_als(dev_factors(), 2, rank=R)  # warm-up (schedules)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dtc.cpd_als(dev_factors(), 10, rank=R)
    torch.cuda.synchronize()
    ours_iter = (time.perf_counter() - t0) / 10
    dtc.free()
    out["cpd_c3_sample"] = {"workload": f"C3 construction, {CPD_SAMPLE_NNZ} nnz, R={R}",
                            "s_per_iter_reference_OmpCpdAlsStep": round(ref_iter, 4),
                            "s_per_iter_ours_hicoo_fp32": round(ours_iter, 5),
                            "speedup": round(ref_iter / ours_iter, 1)}
    return out


def cpu_baseline_block(args):
    """Reference OpenMP HiCOO MTTKRP on a bounded sample (rank 0, N=1)."""
    return run_reference_sample(args)


def summary_of(res):
    """The headline figures of every block, compact."""
    def pick(block, keys):
        b = res.get(block) or {}
        return {k: b[k] for k in keys if k in b}
    out = {"c2_GBps": res.get("value"), "c2_ms_per_step": res.get("ms_per_step"),
           "c2_per_mode_ms": (res.get("config") or {}).get("per_mode_ms"),
           "roofline_frac": (res.get("roofline") or {}).get("frac"), "e2e_GBps": (res.get("e2e") or {}).get("value"),
           "gather_frac_of_l2": (res.get("gather_roofline") or {}).get("frac")}
    c3 = res.get("cpd") or {}
    if c3:
        out["c3"] = {"ms_per_iter_fp32": round(1e3 * c3.get("s_per_iter_fp32", 0), 3),
                     "ms_per_iter_bf16": round(1e3 * c3.get("s_per_iter_bf16", 0), 3),
                     "speedup_bf16": c3.get("speedup_bf16_vs_fp32"),
                     **{k: c3[k] for k in ("fit_fp64_oracle", "fit_diff_fp32", "fit_diff_bf16", "fms_fp32_vs_oracle",
                                           "fms_bf16_vs_oracle") if k in c3}}
    lr = res.get("cpd_lowrank") or {}
    if lr:
        out["c3_lowrank"] = {"ms_per_iter_fp32": round(1e3 * lr.get("s_per_iter_fp32", 0), 3),
                             "ms_per_iter_bf16": round(1e3 * lr.get("s_per_iter_bf16", 0), 3),
                             **{k: lr[k] for k in ("fit_fp64_oracle", "fit_fp32", "fit_bf16", "fit_diff_fp32",
                                                   "fit_diff_bf16", "fms_fp32_vs_oracle", "fms_bf16_vs_oracle",
                                                   "fms_bf16_vs_fp32") if k in lr}}
    out["c4"] = pick("gradcp", ["ms_per_gradient"])
    out["c5"] = pick("batched", ["ms_per_iter_fp32", "ms_per_iter_bf16", "ms_per_iter_fp32_tensor_by_tensor",
                                 "max_fit_diff_fp32", "max_fit_diff_bf16"])
    rn = res.get("renumber") or {}
    if rn:
        out["renumber"] = {k: rn.get(k) for k in ("nb_before", "nb_after")}
        if "bfs_like" in rn:
            out["renumber"]["bfs_like"] = {k: rn["bfs_like"].get(k) for k in ("nb_before", "nb_after_bfs_like",
                                                                             "nb_after_lexi_1_iteration")}
    return {k: v for k, v in out.items() if v not in (None, {}, [])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mttkrp", choices=["mttkrp"])
    ap.add_argument("--ref-sample", type=int, default=4_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpd", action="store_true", help="skip the CPD-ALS (C3) block")
    ap.add_argument("--no-cpd-lowrank", action="store_true",
                    help="skip the C3-sized low-rank CPD-ALS precision block")
    ap.add_argument("--no-gradcp", action="store_true", help="skip the gradient-CP (C4) block")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched CPD-ALS (C5) block")
    ap.add_argument("--batched-iters", type=int, default=C5_ITERS)
    ap.add_argument("--no-ingest", action="store_true", help="skip the tensor-ingest block")
    ap.add_argument("--no-renumber", action="store_true", help="skip the renumbering block")
    ap.add_argument("--bfs-nnz", type=int, default=5_000_000,
                    help="nonzeros of the C2 tensor the BFS-like renumbering block runs on")
    ap.add_argument("--no-ttm", action="store_true", help="skip the TTM block")
    ap.add_argument("--no-sk20", action="store_true", help="skip the C2 sk=20 block")
    ap.add_argument("--only", choices=["cpd", "cpd_lowrank", "gradcp", "batched", "ingest", "renumber", "ttm",
                                       "cpu_paths", "sk20"],
                    default=None,
                    help="run one of the CPD blocks alone and print its JSON (for profiling captures)")
    ap.add_argument("--batched-oracle", type=int, default=16,
                    help="C5 tensors (spread over the size range) checked against the FP64 oracle")
    ap.add_argument("--batched-sequential", type=int, default=1,
                    help="also time the C5 ALS tensor by tensor through ptiB200CpdAls")
    ap.add_argument("--cpd-iters", type=int, default=C3_ITERS)
    ap.add_argument("--cpd-format", default="hicoo", choices=["hicoo", "coo"])
    ap.add_argument("--fp32-sweeps", type=int, default=2)
    ap.add_argument("--cpd-oracle", type=int, default=1)
    ap.add_argument("--nnz", type=int, default=C2_NNZ,
                    help="nonzeros of the C2 construction (smaller only for profiling captures)")
    args = ap.parse_args()

    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        res = run_reference_arm(args, rank, world)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
        return

    from hiparti_b200 import build
    build.build()
    if args.only:
        import torch
        torch.cuda.set_device(0)
        block = {"cpd": run_cpd, "cpd_lowrank": run_cpd_lowrank, "gradcp": run_gradcp, "batched": run_batched, "ingest": run_ingest,
                 "renumber": run_renumber, "ttm": run_ttm, "cpu_paths": run_cpu_paths,
                 "sk20": run_c2_sk20}[args.only]
        print(json.dumps({"only": args.only, **block(args)}), flush=True)
        return
    rank, world, _ = dist_setup(args.gpus)
    res = run_ours_mttkrp(args, rank, world)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline_block(args)
            res["reference_cpu_paths"] = run_cpu_paths(args)
        if world == 1 and not args.no_cpd:
            import torch
            torch.cuda.empty_cache()
            res["cpd"] = run_cpd(args)
        if world == 1 and not args.no_cpd_lowrank:
            import torch
            torch.cuda.empty_cache()
            res["cpd_lowrank"] = run_cpd_lowrank(args)
        if world == 1 and not args.no_gradcp:
            import torch
            torch.cuda.empty_cache()
            res["gradcp"] = run_gradcp(args)
        if world == 1 and not args.no_batched:
            import torch
            torch.cuda.empty_cache()
            res["batched"] = run_batched(args)
        if world == 1 and not args.no_ingest:
            import torch
            torch.cuda.empty_cache()
            res["ingest"] = run_ingest(args)
        if world == 1 and not args.no_renumber:
            import torch
            torch.cuda.empty_cache()
            res["renumber"] = run_renumber(args)
        if world == 1 and not args.no_ttm:
            import torch
            torch.cuda.empty_cache()
            res["ttm"] = run_ttm(args)
        if world == 1 and not args.no_sk20:
            import torch
            torch.cuda.empty_cache()
            res["c2_sk20"] = run_c2_sk20(args)
        # the CPD blocks, then a compact summary of every block, last on the
        # line (a reader that keeps only the end of stdout still sees them)
        for k in ("cpd", "cpd_lowrank"):
            if k in res:
                res[k] = res.pop(k)
        res["summary"] = summary_of(res)
        print(json.dumps(res), flush=True)
    from hiparti_b200 import replicas
    replicas.shutdown(world)


if __name__ == "__main__":
    main()
