"""CPU: pins the oracle (our C restatement) to the reference -- against the
committed golden fixtures made by the reference library, and against the
reference library itself where it has been built."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from hiparti_b200 import synth

CASES = ["coo3_uniform.npz", "coo4_uniform.npz", "coo3_zipf.npz"]


def _unpack(g):
    dims = [int(x) for x in g["dims"]]
    N = len(dims)
    inds = [g[f"ind{m}"] for m in range(N)]
    mats = [g[f"mat{m}"] for m in range(N)]
    return dims, inds, g["vals"], mats, int(g["R"])


@pytest.mark.parametrize("case", CASES)
def test_orc_coo_mttkrp_matches_golden(orc, case):
    g = load_golden(case)
    dims, inds, vals, mats, R = _unpack(g)
    for m in range(len(dims)):
        out = orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]]
        # same summation order as the sequential reference: bit-identical
        np.testing.assert_array_equal(out, g[f"coo_out{m}"])


@pytest.mark.parametrize("case", CASES)
def test_orc_hicoo_conversion_matches_golden(orc, case):
    g = load_golden(case)
    dims, inds, vals, mats, R = _unpack(g)
    N = len(dims)
    h = orc.hicoo_build(dims, inds, vals, int(g["sb"]), int(g["sk"]), int(g["sc"]))
    for key in ["bptr", "vals", "kptr", "cptr", "knnzs", "nkiters"]:
        np.testing.assert_array_equal(h[key], g[f"h_{key}"], err_msg=key)
    for m in range(N):
        np.testing.assert_array_equal(h["binds"][m], g[f"h_binds{m}"])
        np.testing.assert_array_equal(h["einds"][m], g[f"h_einds{m}"])
        # the COO order the reference leaves behind
        np.testing.assert_array_equal(inds[m][h["perm"]], g[f"h_sorted_ind{m}"])
    assert h["max_nnzb"] == int(g["h_max_nnzb"])
    np.testing.assert_array_equal(h["kschr"], g["h_kschr_flat"])
    np.testing.assert_array_equal(h["kschr_rowptr"], g["h_kschr_rowptr"])
    for m in range(N):
        out = orc.mttkrp_hicoo(h, mats, R, m)[: dims[m]]
        np.testing.assert_array_equal(out, g[f"hicoo_out{m}"])


def test_orc_cpd_matches_golden(orc):
    g = load_golden("cpd3_planted.npz")
    dims = [int(x) for x in g["dims"]]
    inds = [g[f"ind{m}"] for m in range(3)]
    init = [g[f"init{m}"] for m in range(3)]
    R, iters = int(g["R"]), int(g["iters"])
    o = orc.cpd_als(dims, inds, g["vals"], R, iters, init)
    # FP64 restatement vs the FP32 reference from the same start
    for m in range(3):
        assert rel_err(o["factors"][m], g[f"ref_factor{m}"]) < 1e-5
    assert rel_err(o["lambda_"], g["ref_lambda"]) < 1e-5
    # The fit computed from Grams agrees with the fit evaluated directly at the
    # nonzeros (the reference's reported fit does not: it reads the Gram
    # triangle its ssyrk_ call leaves unwritten).
    direct = orc.kruskal_fit(dims, inds, g["vals"], o["lambda_"], o["factors"])
    assert abs(direct - o["fit"]) < 1e-9


def test_orc_closed_form_all_ones(orc):
    # With all-ones factors MTTKRP(X, n)[i, r] is the sum of slice i's values.
    dims = (30, 20, 10)
    inds, vals = synth.uniform_tensor(dims, 2000, seed=5)
    mats = [np.ones((d, 8), np.float32) for d in dims]
    for m in range(3):
        out = orc.mttkrp_coo(inds, vals, mats, 8, m)
        slice_sum = np.bincount(inds[m], weights=vals.astype(np.float64), minlength=dims[m])
        np.testing.assert_allclose(out[:, 0], slice_sum, rtol=1e-5)
        assert np.all(out == out[:, :1])


def test_orc_vs_reference_library_random(orc, ref):
    rng = np.random.default_rng(9)
    for trial in range(3):
        N = 3 + trial % 2
        dims = tuple(int(x) for x in rng.integers(5, 70, N))
        nnz = int(min(np.prod(dims) // 3, 3000))
        inds, vals = synth.uniform_tensor(dims, nnz, seed=200 + trial)
        sb, sk, sc = 2, 4, 5
        h = orc.hicoo_build(dims, inds, vals, sb, sk, sc)
        r = ref.to_hicoo(dims, inds, vals, sb, sk, sc)
        for key in ["bptr", "vals", "kptr", "cptr", "knnzs", "nkiters"]:
            np.testing.assert_array_equal(h[key], r[key])
        R = int(rng.integers(1, 20))
        mats = synth.factor_matrices(dims, R, seed=trial)
        for m in range(N):
            np.testing.assert_array_equal(orc.mttkrp_coo(inds, vals, mats, R, m)[: dims[m]],
                                          ref.mttkrp_coo(dims, inds, vals, mats, R, m))


def test_orc_cpd_vs_reference_library(orc, ref):
    dims = (20, 18, 16, 6)
    inds, vals, _ = synth.planted_tensor(dims, 1500, 3, 0.01, seed=31)
    R = 3
    rng = np.random.default_rng(32)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    o = orc.cpd_als(dims, inds, vals, R, 3, init)
    _, lam, facs = ref.cpd_als_step(dims, inds, vals, R, 3, init)
    for m in range(4):
        assert rel_err(o["factors"][m], facs[m]) < 1e-4
    assert rel_err(o["lambda_"], lam) < 1e-4


def test_sparse_lowrank_generator_is_exactly_low_rank(orc):
    # the generating model reproduces every nonzero: fit 1 with no noise
    dims = (40, 30, 20)
    inds, vals, (lam, facs) = synth.sparse_lowrank_tensor(dims, 4, 5, 0.0, seed=3)
    assert vals.size > 200 and np.all(vals > 0)
    fit = orc.kruskal_fit(dims, inds, vals, lam, facs)
    assert abs(fit - 1.0) < 1e-6
