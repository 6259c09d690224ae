"""Generates the golden fixtures in this directory from the REFERENCE library
(oracle/_ref/libHiParTI.so, compiled from the reference's own sources by
`make -C oracle ref`).  Inputs are seeded synthetic tensors; outputs are what
the reference's ptiMTTKRP, ptiSparseTensorToHiCOO, ptiMTTKRPHiCOO and
CpdAlsStep return for them.

    python tests/golden/make_golden.py

Run only where the reference sources exist; the .npz files are committed.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from hiparti_b200 import synth  # noqa: E402
from oracle.oracle import Ref, ensure_built  # noqa: E402

OUT = Path(__file__).resolve().parent


def conversion_case(ref, name, dims, inds, vals, R, sb, sk, sc, fseed):
    mats = synth.factor_matrices(dims, R, seed=fseed)
    d = {"dims": np.asarray(dims, np.uint32), "vals": vals, "R": np.uint32(R),
         "sb": np.uint8(sb), "sk": np.uint8(sk), "sc": np.uint8(sc)}
    N = len(dims)
    for m in range(N):
        d[f"ind{m}"] = inds[m]
        d[f"mat{m}"] = mats[m]
    for m in range(N):
        d[f"coo_out{m}"] = ref.mttkrp_coo(dims, inds, vals, mats, R, m)
    h = ref.to_hicoo(dims, inds, vals, sb, sk, sc)
    d["h_bptr"] = h["bptr"]
    d["h_vals"] = h["vals"]
    d["h_kptr"] = h["kptr"]
    d["h_cptr"] = h["cptr"]
    d["h_knnzs"] = h["knnzs"]
    d["h_nkiters"] = h["nkiters"]
    d["h_max_nnzb"] = np.uint64(h["max_nnzb"])
    rows = h["kschr_rows"]
    d["h_kschr_flat"] = np.concatenate(rows) if rows else np.empty(0, np.uint32)
    d["h_kschr_rowptr"] = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.uint64)
    for m in range(N):
        d[f"h_binds{m}"] = h["binds"][m]
        d[f"h_einds{m}"] = h["einds"][m]
        d[f"h_sorted_ind{m}"] = h["sorted_inds"][m]
    d["h_sorted_vals"] = h["sorted_vals"]
    for m in range(N):
        d[f"hicoo_out{m}"] = ref.mttkrp_hicoo(dims, h, mats, R, m)
    np.savez_compressed(OUT / name, **d)
    print(name, "nnz", vals.size, "nb", h["bptr"].size - 1, "nk", h["kptr"].size - 1, "nc", h["cptr"].size)


def main():
    ensure_built(ref=True)
    ref = Ref()
    dims = (64, 48, 40)
    inds, vals = synth.uniform_tensor(dims, 5000, seed=101)
    conversion_case(ref, "coo3_uniform.npz", dims, inds, vals, 16, 3, 5, 6, 102)

    dims = (24, 20, 18, 16)
    inds, vals = synth.uniform_tensor(dims, 4000, seed=103)
    conversion_case(ref, "coo4_uniform.npz", dims, inds, vals, 8, 2, 4, 5, 104)

    dims = (500, 400, 300)
    inds, vals = synth.zipf_tensor(dims, 20000, s=1.1, seed=105)
    conversion_case(ref, "coo3_zipf.npz", dims, inds, vals, 32, 4, 6, 8, 106)

    # CPD: planted rank-3 model, R=4, 5 iterations from |N(0,1)| factors.
    dims = (30, 25, 20)
    inds, vals, _ = synth.planted_tensor(dims, 3000, 3, 0.01, seed=107)
    R, iters = 4, 5
    rng = np.random.default_rng(108)
    init = [np.abs(rng.standard_normal((d, R))).astype(np.float32) for d in dims]
    fit, lam, facs = ref.cpd_als_step(dims, inds, vals, R, iters, init)
    d = {"dims": np.asarray(dims, np.uint32), "vals": vals, "R": np.uint32(R), "iters": np.uint32(iters),
         "ref_fit": np.float64(fit), "ref_lambda": lam}
    for m in range(3):
        d[f"ind{m}"] = inds[m]
        d[f"init{m}"] = init[m]
        d[f"ref_factor{m}"] = facs[m]
    np.savez_compressed(OUT / "cpd3_planted.npz", **d)
    print("cpd3_planted.npz fit(reference-reported)", fit)


if __name__ == "__main__":
    main()
