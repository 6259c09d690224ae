"""GPU parity at the benchmark configurations' full sizes, against the
reference library compiled from its sources (oracle/_ref), on the same seeded
inputs:

* C1: 3-D 1000^3, 1,000,000 coordinates drawn uniformly (duplicates merged by
  summing their values), U(0,1) values, 1000x16 U(0,1) factors, R = 16: the
  drop-in ptiMTTKRP / ptiOmpMTTKRP (GPU) against the reference's ptiMTTKRP
  (src/sptensor/mttkrp.c:39-163) and ptiOmpMTTKRP_Reduce
  (src/sptensor/mttkrp_omp.c:401-493), every mode, normwise relative 1e-5.
* C2: 3-D 200,000 x 150,000 x 20,000 with 50M unique Zipf(1.1) coordinates
  (the benchmark tensor itself: same generator and seed), sb = 7, sk = 10,
  sc = 14:
    - the drop-in ptiSparseTensorToHiCOO (GPU) bit for bit against the
      reference's ptiSparseTensorToHiCOO(tk=1)
      (src/sptensor/hicoo/convert.c:646-860): bptr, binds, einds, values,
      kptr, cptr, knnzs, nkiters, max_nnzb, the kernel schedule kschr, the
      balanced scheduler and the caller's COO left sorted;
    - the drop-in ptiOmpMTTKRPHiCOO (GPU) against the reference's
      ptiOmpMTTKRPHiCOO (src/sptensor/hicoo/mttkrp_omp.c:184) on that HiCOO
      tensor with R = 32 U(0,1) factors, every mode: ours within normwise
      relative 1e-5 of an FP64 sum, and apart from the reference by no more
      than the reference's own FP32 error (see the test).
"""
import os

import numpy as np
import pytest

from conftest import rel_err
from hiparti_b200 import COOTensor, synth

pytestmark = pytest.mark.gpu
TOL = 1e-5
THREADS = os.cpu_count() or 1


def c1_tensor(seed=2024):
    """C1: 1,000,000 uniform draws over 1000^3, duplicates merged (values
    summed), nonzeros in random order."""
    dims = (1000, 1000, 1000)
    n = 1_000_000
    rng = np.random.default_rng(seed)
    cols = [rng.integers(0, d, n, dtype=np.uint64) for d in dims]
    vals = rng.random(n, dtype=np.float32)
    key = (cols[0] * np.uint64(dims[1]) + cols[1]) * np.uint64(dims[2]) + cols[2]
    uniq, inv = np.unique(key, return_inverse=True)
    merged = np.bincount(inv, weights=vals.astype(np.float64)).astype(np.float32)
    order = rng.permutation(uniq.size)
    uniq, merged = uniq[order], merged[order]
    inds = [(uniq // np.uint64(dims[1] * dims[2])).astype(np.uint32),
            ((uniq // np.uint64(dims[2])) % np.uint64(dims[1])).astype(np.uint32),
            (uniq % np.uint64(dims[2])).astype(np.uint32)]
    return dims, inds, merged


def test_c1_coo_mttkrp_vs_reference(lib, cuda, ref):
    dims, inds, vals = c1_tensor()
    assert 999_000 < vals.size <= 1_000_000
    R = 16
    mats = synth.factor_matrices(dims, R, seed=2025)
    coo = COOTensor(dims, inds, vals)
    for mode in range(3):
        want_seq = ref.mttkrp_coo(dims, inds, vals, mats, R, mode, variant="seq")
        want_red = ref.mttkrp_coo(dims, inds, vals, mats, R, mode, variant="omp_reduce", tk=THREADS)
        assert rel_err(want_red, want_seq) < TOL  # the reference agrees with itself
        for variant in ("seq", "omp"):
            got = coo.mttkrp(mats, R, mode, variant=variant)
            assert rel_err(got[:, :R], want_seq[:, :R]) < TOL, (mode, variant)
            assert rel_err(got[:, :R], want_red[:, :R]) < TOL, (mode, variant)
            assert np.all(got[:, R:] == 0)


@pytest.fixture(scope="module")
def c2(lib, cuda, ref):
    """The 50M-nonzero benchmark tensor on the host, converted by both
    libraries."""
    import torch
    from bench import C2_DIMS, C2_SB, C2_SC, C2_SK, SEED, c2_factors
    from hiparti_b200.synth import coords_torch
    ti = coords_torch(C2_DIMS, 50_000_000, SEED, zipf_s=1.1, device=cuda)
    g = torch.Generator(device=cuda)
    g.manual_seed(SEED + 1)
    tv = torch.rand(50_000_000, generator=g, device=cuda, dtype=torch.float32)
    inds = [t.cpu().numpy().view(np.uint32) for t in ti]
    vals = tv.cpu().numpy()
    mats = [m.cpu().numpy() for m in c2_factors(cuda, SEED)]
    del ti, tv
    torch.cuda.empty_cache()
    coo = COOTensor(C2_DIMS, [i.copy() for i in inds], vals.copy())
    ours = coo.to_hicoo(C2_SB, C2_SK, C2_SC)
    theirs = ref.to_hicoo(list(C2_DIMS), inds, vals, C2_SB, C2_SK, C2_SC)
    return {"dims": C2_DIMS, "coo": coo, "ours": ours, "ref": theirs, "mats": mats}


def test_c2_conversion_bit_exact_vs_reference(c2):
    h, r, coo = c2["ours"], c2["ref"], c2["coo"]
    assert h.nnz == 50_000_000 and h.nb == r["bptr"].size - 1
    np.testing.assert_array_equal(h.bptr, r["bptr"])
    np.testing.assert_array_equal(h.vals, r["vals"])
    np.testing.assert_array_equal(h.kptr, r["kptr"])
    np.testing.assert_array_equal(h.cptr, r["cptr"])
    np.testing.assert_array_equal(h.knnzs, r["knnzs"])
    np.testing.assert_array_equal(h.nkiters, r["nkiters"])
    assert h.max_nnzb == r["max_nnzb"]
    for m in range(3):
        np.testing.assert_array_equal(h.binds[m], r["binds"][m])
        np.testing.assert_array_equal(h.einds[m], r["einds"][m])
        # the caller's COO is left sorted in HiCOO order, as the reference leaves it
        np.testing.assert_array_equal(coo.inds[m], r["sorted_inds"][m])
    np.testing.assert_array_equal(coo.vals, r["sorted_vals"])
    assert len(h.kschr_rows) == len(r["kschr_rows"])
    for a, b in zip(h.kschr_rows, r["kschr_rows"]):
        np.testing.assert_array_equal(a, b)
    for key, rk in [("rows", "kschr_balanced_rows"), ("pos_rows", "kschr_balanced_pos_rows"),
                    ("rest", "kschr_rest")]:
        assert len(h.balanced[key]) == len(r[rk])
        for a, b in zip(h.balanced[key], r[rk]):
            np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(h.balanced["nkpars"], r["nkpars"])


def _fp64_mttkrp(coo, mats, R, mode, cuda):
    """MTTKRP of a host COO tensor in FP64 with torch on the GPU (chunks of
    nonzeros, index_add_ into an FP64 output)."""
    import torch
    inds = [torch.from_numpy(i.view(np.int32)).to(cuda).long() for i in coo.inds]
    vals = torch.from_numpy(coo.vals).to(cuda).double()
    facs = [torch.from_numpy(m[:, :R]).to(cuda).double() for m in mats]
    out = torch.zeros((coo.dims[mode], R), dtype=torch.float64, device=cuda)
    step = 4_000_000
    for z0 in range(0, vals.numel(), step):
        sl = slice(z0, z0 + step)
        p = vals[sl][:, None]
        for k in range(len(mats)):
            if k != mode:
                p = p * facs[k][inds[k][sl]]
        out.index_add_(0, inds[mode][sl], p)
    res = out.cpu().numpy()
    del inds, vals, facs, out
    torch.cuda.empty_cache()
    return res


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_c2_hicoo_mttkrp_vs_reference_omp(c2, ref, cuda, mode):
    """Both results against an FP64 sum of the same products.  The reference
    adds every product into its output row with an FP32 atomic, one after
    another (hicoo/mttkrp_omp.c:400-467), and the head rows of a Zipf(1.1)
    mode hold millions of nonzeros, so its own error can exceed 1e-5; ours
    sums per thread group and per tile before the row adds.  Required: ours
    within 1e-5 of FP64, and ours and the reference apart by no more than the
    reference's own error explains."""
    R = 32
    dims, mats = c2["dims"], c2["mats"]
    want = ref.mttkrp_hicoo(list(dims), c2["ref"], mats, R, mode, variant="omp", tk=THREADS)[:, :R]
    got = c2["ours"].mttkrp(mats, R, mode, variant="omp")
    assert np.all(got[:, R:] == 0)
    got = got[:, :R]
    exact = _fp64_mttkrp(c2["coo"], mats, R, mode, cuda)
    e_ours, e_ref, e_diff = rel_err(got, exact), rel_err(want, exact), rel_err(got, want)
    print(f"mode {mode}: ours vs FP64 {e_ours:.2e}, reference vs FP64 {e_ref:.2e}, ours vs reference {e_diff:.2e}")
    assert e_ours < TOL
    assert e_diff < max(TOL, 1.5 * e_ref)
    # rows of at most 1000 nonzeros, where the reference's serial FP32 sums
    # are short: the two libraries agree to 1e-5 there directly
    counts = np.bincount(c2["coo"].inds[mode], minlength=dims[mode])
    light = counts <= 1000
    assert light.sum() > 0.5 * dims[mode]
    assert rel_err(got[light], want[light]) < TOL
