"""Seeded synthetic sparse tensors with the shapes and value distributions of the
benchmark workloads (no public dataset is involved).

Coordinates are unique: draws that repeat an existing coordinate are rejected
and re-drawn, so the HiCOO ordering is fully defined and values keep their
stated distribution.  Small tensors are generated with numpy on the host; the
large workloads (tens of millions of nonzeros) with torch on a CUDA device,
where de-duplication by sorting takes milliseconds instead of minutes.
"""
from __future__ import annotations

import numpy as np


def _linear(cols, dims):
    key = np.zeros_like(cols[0], dtype=np.uint64)
    for c, d in zip(cols, dims):
        key = key * np.uint64(d) + c.astype(np.uint64)
    return key


def _delinear(keys, dims):
    out = []
    k = keys.copy()
    for d in reversed(dims):
        out.append((k % np.uint64(d)).astype(np.uint32))
        k //= np.uint64(d)
    return out[::-1]


def _zipf_sampler(rng, I, s):
    w = np.arange(1, I + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    perm = rng.permutation(I).astype(np.uint32)

    def draw(n):
        r = np.searchsorted(cdf, rng.random(n), side="right")
        return perm[np.minimum(r, I - 1)]
    return draw


def coords_numpy(dims, nnz, seed, zipf_s=None):
    """Unique coordinates, uniform per mode or Zipf(s) over a seeded permutation
    of each mode.  Returns a list of uint32 arrays in random order."""
    rng = np.random.default_rng(seed)
    dims = [int(d) for d in dims]
    total = 1
    for d in dims:
        total *= d
    if nnz > total:
        raise ValueError("more nonzeros than cells")
    if zipf_s is None:
        draws = [lambda n, d=d: rng.integers(0, d, n, dtype=np.uint32) for d in dims]
    else:
        draws = [_zipf_sampler(rng, d, zipf_s) for d in dims]
    keys = np.empty(0, np.uint64)
    while keys.size < nnz:
        need = nnz - keys.size
        cand = _linear([dr(int(need * 1.3) + 64) for dr in draws], dims)
        keys = np.unique(np.concatenate([keys, cand]))
    keys = rng.permutation(keys)[:nnz]
    return _delinear(keys, dims)


def uniform_tensor(dims, nnz, seed=0):
    """Uniform unique coordinates, values U(0,1) FP32."""
    inds = coords_numpy(dims, nnz, seed)
    vals = np.random.default_rng(seed + 1).random(nnz, dtype=np.float32)
    return inds, vals


def zipf_tensor(dims, nnz, s=1.1, seed=0):
    inds = coords_numpy(dims, nnz, seed, zipf_s=s)
    vals = np.random.default_rng(seed + 1).random(nnz, dtype=np.float32)
    return inds, vals


def planted_tensor(dims, nnz, rank, noise, seed=0):
    """Uniform unique coordinates; values of a planted rank-`rank` Kruskal
    model (factor entries |N(0,1)|, unit-norm columns, weights U(1,10)) plus
    N(0, noise^2) noise.  Returns (inds, vals, (lambda, factors))."""
    inds = coords_numpy(dims, nnz, seed)
    rng = np.random.default_rng(seed + 7)
    facs = []
    for d in dims:
        a = np.abs(rng.standard_normal((d, rank)))
        a /= np.linalg.norm(a, axis=0, keepdims=True)
        facs.append(a)
    lam = rng.uniform(1, 10, rank)
    model = np.tile(lam, (nnz, 1))
    for a, ix in zip(facs, inds):
        model *= a[ix]
    vals = (model.sum(1) + noise * rng.standard_normal(nnz)).astype(np.float32)
    return inds, vals, (lam, facs)


def sparse_lowrank_tensor(dims, rank, support, noise=0.0, seed=0):
    """A sparse tensor of exact CP rank `rank` (plus N(0, noise^2) on its
    nonzeros).  Component r has entries |N(0,1)| + 0.1 on `support` random rows
    of every mode and zeros elsewhere, with weight U(1,10); the nonzeros are
    the union of the components' support blocks, so about rank * support^N of
    them.  Unlike values of a dense model sampled at random coordinates (which
    leave the unsampled cells zero and make the sparse tensor high-rank), this
    tensor is low-rank, so CPD-ALS converges to a fit near 1.
    Returns (inds, vals, (lambda, factors))."""
    rng = np.random.default_rng(seed)
    facs = [np.zeros((d, rank)) for d in dims]
    cells = []
    for r in range(rank):
        rows = []
        for m, d in enumerate(dims):
            s = min(support, d)
            idx = rng.choice(d, s, replace=False)
            facs[m][idx, r] = np.abs(rng.standard_normal(s)) + 0.1
            rows.append(idx)
        grid = np.meshgrid(*rows, indexing="ij")
        cells.append(np.stack([g.ravel() for g in grid], 1))
    coords = np.unique(np.concatenate(cells), axis=0)
    inds = [coords[:, m].astype(np.uint32) for m in range(len(dims))]
    lam = rng.uniform(1, 10, rank)
    model = np.tile(lam, (coords.shape[0], 1))
    for a, ix in zip(facs, inds):
        model *= a[ix]
    vals = (model.sum(1) + noise * rng.standard_normal(coords.shape[0])).astype(np.float32)
    return inds, vals, (lam, facs)


def factor_matrices(dims, R, seed=0, dist="uniform"):
    """Row-major factors with the reference's stride (R rounded up to 8); pad
    columns are zero."""
    rng = np.random.default_rng(seed)
    stride = ((R - 1) // 8 + 1) * 8
    mats = []
    for d in dims:
        a = np.zeros((d, stride), np.float32)
        if dist == "uniform":
            a[:, :R] = rng.random((d, R), dtype=np.float32)
        else:
            a[:, :R] = rng.standard_normal((d, R)).astype(np.float32)
        mats.append(a)
    return mats


# ----------------------------------------------------------------------------
# Large tensors on the GPU
# ----------------------------------------------------------------------------
def coords_torch(dims, nnz, seed, zipf_s=None, device="cuda"):
    """Same construction as coords_numpy on a CUDA device with torch (Philox
    generator).  Returns a list of uint32-valued int64 torch tensors... as
    int32 tensors holding the unsigned coordinates (all < 2^31 here)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    dims = [int(d) for d in dims]
    samplers = []
    for d in dims:
        if zipf_s is None:
            samplers.append(lambda n, d=d: torch.randint(0, d, (n,), generator=g, device=device))
        else:
            w = torch.arange(1, d + 1, device=device, dtype=torch.float64) ** (-zipf_s)
            cdf = torch.cumsum(w, 0)
            cdf /= cdf[-1].clone()
            perm = torch.randperm(d, generator=g, device=device)

            def draw(n, cdf=cdf, perm=perm, d=d):
                u = torch.rand(n, generator=g, device=device, dtype=torch.float64)
                r = torch.searchsorted(cdf, u, right=True).clamp_(max=d - 1)
                return perm[r]
            samplers.append(draw)

    def linear(cols):
        key = torch.zeros_like(cols[0])
        for c, d in zip(cols, dims):
            key = key * d + c
        return key

    keys = torch.empty(0, dtype=torch.int64, device=device)
    while keys.numel() < nnz:
        need = nnz - keys.numel()
        cand = linear([s(int(need * 1.3) + 1024) for s in samplers])
        keys = torch.unique(torch.cat([keys, cand]))
    keys = keys[torch.randperm(keys.numel(), generator=g, device=device)[:nnz]]
    cols = []
    for d in reversed(dims):
        cols.append((keys % d).to(torch.int32))
        keys = keys // d
    return cols[::-1]


def sparse_lowrank_torch(dims, rank, support, noise=0.0, seed=0, device="cuda"):
    """sparse_lowrank_tensor on a CUDA device with torch, for tens of millions
    of nonzeros: component r has entries |N(0,1)| + 0.1 on `support` random
    rows of every mode (zeros elsewhere) and weight U(1,10); the nonzeros are
    the union of the components' support blocks (rank * support^N coordinates
    before the rare overlaps merge), with values sum_r lambda_r prod_m
    A_m[i_m, r] + N(0, noise^2).  Returns (inds as int32 tensors, FP32 values,
    (lambda, factors) as FP64 tensors)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    dims = [int(d) for d in dims]
    N = len(dims)
    facs = [torch.zeros((d, rank), dtype=torch.float64, device=device) for d in dims]
    keys = []
    for r in range(rank):
        rows = []
        for m, d in enumerate(dims):
            s = min(support, d)
            idx = torch.randperm(d, generator=g, device=device)[:s]
            facs[m][idx, r] = torch.randn(s, generator=g, device=device, dtype=torch.float64).abs_() + 0.1
            rows.append(idx)
        grid = torch.meshgrid(*rows, indexing="ij")
        key = torch.zeros_like(grid[0].reshape(-1))
        for gm, d in zip(grid, dims):
            key = key * d + gm.reshape(-1)
        keys.append(key)
    keys = torch.unique(torch.cat(keys))
    cols = []
    k = keys.clone()
    for d in reversed(dims):
        cols.append(k % d)
        k = k // d
    cols = cols[::-1]
    lam = torch.rand(rank, generator=g, device=device, dtype=torch.float64) * 9 + 1
    vals = torch.zeros(keys.numel(), dtype=torch.float64, device=device)
    step = 1 << 22
    for z0 in range(0, keys.numel(), step):
        model = lam.expand(min(step, keys.numel() - z0), rank).clone()
        for a, c in zip(facs, cols):
            model *= a[c[z0:z0 + step]]
        vals[z0:z0 + step] = model.sum(1)
    if noise:
        vals += torch.randn(vals.numel(), generator=g, device=device, dtype=torch.float64) * noise
    inds = [c.to(torch.int32) for c in cols]
    return inds, vals.float(), (lam, facs)
