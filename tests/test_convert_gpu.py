"""GPU COO->HiCOO conversion: bit-identical to the reference (golden fixtures
made by the reference library, the reference library itself where built, and
the oracle restatement), and size-independent properties at larger sizes."""
import numpy as np
import pytest

from conftest import load_golden
from hiparti_b200 import COOTensor, DeviceTensor, synth

pytestmark = pytest.mark.gpu


def _same_hicoo(h, ref, N):
    np.testing.assert_array_equal(h.bptr, ref["bptr"])
    np.testing.assert_array_equal(h.vals, ref["vals"])
    np.testing.assert_array_equal(h.kptr, ref["kptr"])
    np.testing.assert_array_equal(h.cptr, ref["cptr"])
    np.testing.assert_array_equal(h.knnzs, ref["knnzs"])
    np.testing.assert_array_equal(h.nkiters, ref["nkiters"])
    for m in range(N):
        np.testing.assert_array_equal(h.binds[m], ref["binds"][m])
        np.testing.assert_array_equal(h.einds[m], ref["einds"][m])


@pytest.mark.parametrize("case", ["coo3_uniform.npz", "coo4_uniform.npz", "coo3_zipf.npz"])
def test_golden_conversion(lib, cuda, case):
    g = load_golden(case)
    dims = [int(x) for x in g["dims"]]
    N = len(dims)
    coo = COOTensor(dims, [g[f"ind{m}"].copy() for m in range(N)], g["vals"].copy())
    h = coo.to_hicoo(int(g["sb"]), int(g["sk"]), int(g["sc"]))
    ref = {k: g[f"h_{k}"] for k in ["bptr", "vals", "kptr", "cptr", "knnzs", "nkiters"]}
    ref["binds"] = [g[f"h_binds{m}"] for m in range(N)]
    ref["einds"] = [g[f"h_einds{m}"] for m in range(N)]
    _same_hicoo(h, ref, N)
    assert h.max_nnzb == int(g["h_max_nnzb"])
    flat = np.concatenate(h.kschr_rows) if h.kschr_rows else np.empty(0, np.uint32)
    np.testing.assert_array_equal(flat, g["h_kschr_flat"])
    # the caller's COO is left sorted, as the reference leaves it
    for m in range(N):
        np.testing.assert_array_equal(coo.inds[m], g[f"h_sorted_ind{m}"])
    np.testing.assert_array_equal(coo.vals, g["h_sorted_vals"])


CASES = [
    ((300, 200, 100), 20000, 3, 5, 6, None),
    ((300, 200, 100), 20000, 2, 2, 2, None),      # sk == sb == sc
    ((300, 200, 100), 20000, 4, 12, 20, None),    # one kernel, one chunk
    ((5000, 4000, 3000), 60000, 7, 10, 14, 1.1),  # Zipf, the benchmark's block sizes
    ((90, 80, 70, 60), 30000, 3, 4, 5, None),     # 4-D
    ((1 << 20, 1 << 19, 3000), 50000, 5, 9, 9, 1.1),
    ((40000, 30000, 20000, 500), 80000, 7, 10, 14, None),
]


@pytest.mark.parametrize("dims,nnz,sb,sk,sc,zipf", CASES)
def test_conversion_vs_reference(lib, cuda, orc, ref, dims, nnz, sb, sk, sc, zipf):
    if zipf:
        inds, vals = synth.zipf_tensor(dims, nnz, s=zipf, seed=nnz)
    else:
        inds, vals = synth.uniform_tensor(dims, nnz, seed=nnz + sb)
    N = len(dims)
    h = COOTensor(dims, [i.copy() for i in inds], vals.copy()).to_hicoo(sb, sk, sc)
    r = ref.to_hicoo(dims, inds, vals, sb, sk, sc)
    _same_hicoo(h, r, N)
    assert h.max_nnzb == r["max_nnzb"]
    assert len(h.kschr_rows) == len(r["kschr_rows"])
    for a, b in zip(h.kschr_rows, r["kschr_rows"]):
        np.testing.assert_array_equal(a, b)
    for key, rk in [("rows", "kschr_balanced_rows"), ("pos_rows", "kschr_balanced_pos_rows"), ("rest", "kschr_rest")]:
        assert len(h.balanced[key]) == len(r[rk])
        for a, b in zip(h.balanced[key], r[rk]):
            np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(h.balanced["nkpars"], r["nkpars"])


def test_conversion_vs_oracle_medium(lib, cuda, orc):
    dims = (200_000, 150_000, 20_000)
    inds, vals = synth.zipf_tensor(dims, 1_000_000, s=1.1, seed=77)
    h = COOTensor(dims, [i.copy() for i in inds], vals.copy()).to_hicoo(7, 10, 14)
    o = orc.hicoo_build(dims, inds, vals, 7, 10, 14)
    _same_hicoo(h, o, 3)


def test_device_conversion_properties(lib, cuda):
    """Device path at 8M nonzeros: the HiCOO arrays reproduce the COO
    nonzeros, blocks are contiguous, and nonzeros are in (kernel, Morton) order."""
    import torch
    from hiparti_b200.synth import coords_torch
    dims = (200_000, 150_000, 20_000)
    n = 8_000_000
    inds = coords_torch(dims, n, 5, zipf_s=1.1, device="cuda")
    vals = torch.rand(n, device="cuda")
    coo = DeviceTensor.from_torch_coo(dims, inds, vals)
    h = coo.to_hicoo(7, 10, 14)
    from bench import download_hicoo
    host = download_hicoo(h)
    bptr = host["bptr"].astype(np.int64)
    assert bptr[0] == 0 and bptr[-1] == n and np.all(np.diff(bptr) > 0)
    blk = np.repeat(np.arange(bptr.size - 1), np.diff(bptr))
    coords = [(host["binds"][m][blk].astype(np.uint64) << np.uint64(7)) + host["einds"][m] for m in range(3)]
    # same multiset of (coordinate, value) as the input
    key_in = ((inds[0].long() * dims[1] + inds[1].long()) * dims[2] + inds[2].long()).cpu().numpy()
    key_out = (coords[0] * np.uint64(dims[1]) + coords[1]) * np.uint64(dims[2]) + coords[2]
    order_in = np.argsort(key_in)
    order_out = np.argsort(key_out.astype(np.int64))
    np.testing.assert_array_equal(key_in[order_in], key_out.astype(np.int64)[order_out])
    np.testing.assert_array_equal(vals.cpu().numpy()[order_in], host["vals"][order_out])
    # kernels in lexicographic order of (i >> sk)
    kc = [(c >> np.uint64(10)).astype(np.int64) for c in coords]
    kkey = (kc[0] * 1000 + kc[1]) * 1000 + kc[2]
    assert np.all(np.diff(kkey) >= 0)
    # inside a kernel, Morton order of the low 10 bits (mode 0 most significant)
    def spread(x):
        out = np.zeros_like(x, dtype=np.uint64)
        for b in range(10):
            out |= ((x >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b)
        return out
    low = [c & np.uint64(1023) for c in coords]
    mort = (spread(low[0]) << np.uint64(2)) | (spread(low[1]) << np.uint64(1)) | spread(low[2])
    same_kernel = np.diff(kkey) == 0
    assert np.all(np.diff(mort.astype(np.int64))[same_kernel] > 0)
    coo.free()
    h.free()
