"""Generates tests/golden/bfs_like.npz: BFS-like renumberings (ptiBFSLike,
src/sptensor/renumber.c:794-839) computed by the reference's own source,
compiled with an allocator that fills fresh memory with 0xFF bytes
(oracle/ff_malloc.c, `make -C oracle ref`), so that the visit marks it reads
before writing are "not visited" and the result is reproducible.

    python tests/golden/make_bfs_golden.py      (needs the reference checkout)
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from hiparti_b200 import synth  # noqa: E402
from oracle.oracle import Ref, ensure_built  # noqa: E402

OUT = Path(__file__).resolve().parent / "bfs_like.npz"
CASES = [((30, 20, 10), 300, 1), ((200, 150, 100), 3000, 2), ((40, 30, 20, 10), 2000, 4), ((500, 3, 7), 1000, 5),
         ((60, 50, 40), 4000, 6)]


def main():
    ensure_built(ref=True)
    ref = Ref()
    d = {"ncases": np.uint32(len(CASES))}
    for c, (dims, nnz, seed) in enumerate(CASES):
        inds, vals = synth.zipf_tensor(dims, nnz, s=1.1, seed=seed) if c % 2 else synth.uniform_tensor(dims, nnz, seed)
        maps = ref.bfs_like(list(dims), inds, vals)
        d[f"c{c}_dims"] = np.asarray(dims, np.uint32)
        for m in range(len(dims)):
            d[f"c{c}_ind{m}"] = inds[m]
            d[f"c{c}_map{m}"] = maps[m]
        d[f"c{c}_vals"] = vals
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
