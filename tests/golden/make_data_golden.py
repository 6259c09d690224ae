"""Generates golden fixtures from the reference's own example tensors
(data/tensors/*.tns of the reference tree) with the REFERENCE library
(oracle/_ref/libHiParTI.so, compiled from the reference's sources by
`make -C oracle ref`).

For every example file it stores the file's bytes and what the reference's
ptiLoadSparseTensor returns for them (return code, mode sizes, coordinates,
values).  For the files that load as 3-D tensors with unique coordinates it
also stores seeded factor matrices and the reference's ptiMTTKRP output, its
ptiSparseTensorToHiCOO arrays and its ptiMTTKRPHiCOO output for every mode.

    python tests/golden/make_data_golden.py

Run only where the reference tree exists; the .npz files are committed.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from hiparti_b200 import synth  # noqa: E402
from oracle.oracle import REF_SRC, Ref, ensure_built  # noqa: E402

OUT = Path(__file__).resolve().parent
DATA = REF_SRC / "data" / "tensors"  # the reference checkout ($HIPARTI_REF)
# (file, rank, sb, sk, sc) -- block sizes small enough that the tiny examples span several blocks
FILES = [("3d_7.tns", 4, 1, 2, 3), ("3d-24.tns", 8, 1, 2, 3), ("3d_dense.tns", 8, 1, 2, 3),
         ("3D_12031.tns", 16, 3, 4, 6), ("4d_3_16.tns", 8, 1, 2, 3)]


def main():
    ensure_built(ref=True)
    ref = Ref()
    for fname, R, sb, sk, sc in FILES:
        raw = (DATA / fname).read_bytes()
        d = {"file_bytes": np.frombuffer(raw, np.uint8).copy(), "R": np.uint32(R),
             "sb": np.uint8(sb), "sk": np.uint8(sk), "sc": np.uint8(sc)}
        rc, dims, inds, vals = ref.load(DATA / fname, 1)
        d["load_rc"] = np.int32(rc)
        note = f"rc {rc}"
        if rc == 0:
            N = len(dims)
            d["dims"] = np.asarray(dims, np.uint32)
            d["vals"] = vals
            for m in range(N):
                d[f"ind{m}"] = inds[m]
            lin = np.zeros(vals.size, np.int64)
            for m in range(N):
                lin = lin * int(dims[m]) + inds[m].astype(np.int64)
            unique = np.unique(lin).size == vals.size
            in_range = all(int(inds[m].max(initial=0)) < int(dims[m]) for m in range(N)) and vals.size > 0
            d["unique"] = np.bool_(unique)
            note += f" N {N} dims {dims} nnz {vals.size} unique {unique} in_range {in_range}"
            if N == 3 and unique and in_range:
                mats = synth.factor_matrices(dims, R, seed=len(raw))
                for m in range(N):
                    d[f"mat{m}"] = mats[m]
                    d[f"coo_out{m}"] = ref.mttkrp_coo(dims, inds, vals, mats, R, m)
                h = ref.to_hicoo(dims, inds, vals, sb, sk, sc)
                d["h_bptr"] = h["bptr"]
                d["h_vals"] = h["vals"]
                d["h_kptr"] = h["kptr"]
                d["h_cptr"] = h["cptr"]
                for m in range(N):
                    d[f"h_binds{m}"] = h["binds"][m]
                    d[f"h_einds{m}"] = h["einds"][m]
                    d[f"hicoo_out{m}"] = ref.mttkrp_hicoo(dims, h, mats, R, m)
                note += f" nb {h['bptr'].size - 1}"
        name = "data_" + fname.replace(".tns", "").replace("-", "_") + ".npz"
        np.savez_compressed(OUT / name, **d)
        print(name, note)


if __name__ == "__main__":
    main()
