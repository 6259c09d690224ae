"""TEST INFRASTRUCTURE ONLY -- the checker for hiparti_b200.

Two CPU implementations of the reference's MTTKRP / COO->HiCOO / CPD-ALS path,
driven from numpy:

* ``Orc``: our plain-C restatement (oracle/orc.c), each function citing the
  reference lines it follows.  FP32 MTTKRP, bit-exact conversion, FP64 CPD.
* ``Ref``: the reference library itself, compiled from its own sources by
  ``make -C oracle ref`` into oracle/_ref/libHiParTI.so (CPU/OpenMP build),
  used to pin ``Orc`` and as the timed CPU baseline.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  The product library never loads anything from here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_SO = HERE / "_build" / "liborc.so"
REF_SO = HERE / "_ref" / "libHiParTI.so"
BFS_SO = HERE / "_ref" / "libbfsref.so"
# the reference checkout: $HIPARTI_REF, else a "reference" directory beside the repository
REF_SRC = Path(os.environ.get("HIPARTI_REF", HERE.parent.parent / "reference")).resolve()


def ensure_built(ref: bool = True) -> None:
    """Builds liborc.so (always possible: plain C) and, where the reference
    sources exist, the reference library.  No-op when up to date."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)
    if ref and (REF_SRC / "src").is_dir():
        subprocess.run(["make", "-s", "-j8", "-C", str(HERE), "ref"], check=True,
                       capture_output=True)


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _ptr_array(arrs, ctype):
    arr = (C.POINTER(ctype) * len(arrs))()
    for i, a in enumerate(arrs):
        arr[i] = a.ctypes.data_as(C.POINTER(ctype))
    return arr


# ----------------------------------------------------------------------------
# Our C restatement
# ----------------------------------------------------------------------------
class Orc:
    def __init__(self):
        if not ORC_SO.exists():
            ensure_built(ref=False)
        L = C.CDLL(str(ORC_SO))
        L.orc_mttkrp_coo_f32.restype = None
        L.orc_mttkrp_coo_f64.restype = None
        L.orc_mttkrp_hicoo_f32.restype = None
        L.orc_hicoo_build.restype = C.c_void_p
        L.orc_hicoo_build.argtypes = [C.c_uint32, C.POINTER(C.c_uint32), C.c_uint64,
                                      C.c_void_p, C.c_void_p, C.c_uint8, C.c_uint8, C.c_uint8]
        L.orc_hicoo_counts.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        L.orc_hicoo_free.argtypes = [C.c_void_p]
        L.orc_hicoo_export.argtypes = [C.c_void_p] + [C.c_void_p] * 11
        L.orc_cpd_als_f64.restype = C.c_double
        L.orc_kruskal_fit_f64.restype = C.c_double
        self.L = L

    # -- MTTKRP --------------------------------------------------------------
    def mttkrp_coo(self, inds, vals, mats, R, mode, mats_order=None):
        """inds: list of uint32 arrays; mats: list of (I_k, stride) float32."""
        N = len(inds)
        stride = mats[0].shape[1]
        if mats_order is None:
            mats_order = [(mode + i) % N for i in range(N)]
        inds = [np.ascontiguousarray(i, np.uint32) for i in inds]
        vals = np.ascontiguousarray(vals, np.float32)
        mats = [np.ascontiguousarray(m, np.float32) for m in mats]
        order = np.asarray(mats_order, np.uint32)
        out = np.zeros((mats[mode].shape[0], stride), np.float32)
        self.L.orc_mttkrp_coo_f32(C.c_uint32(N), C.c_uint64(vals.size),
                                  _ptr_array(inds, C.c_uint32), vals.ctypes.data_as(C.c_void_p),
                                  _ptr_array(mats, C.c_float), C.c_uint32(R), C.c_uint32(stride),
                                  _u32p(order), C.c_uint32(mode), C.c_uint32(out.shape[0]),
                                  out.ctypes.data_as(C.c_void_p))
        return out

    def mttkrp_coo_f64(self, inds, vals, mats, R, mode):
        N = len(inds)
        stride = mats[0].shape[1]
        inds = [np.ascontiguousarray(i, np.uint32) for i in inds]
        vals = np.ascontiguousarray(vals, np.float32)
        mats = [np.ascontiguousarray(m, np.float64) for m in mats]
        out = np.zeros((mats[mode].shape[0], stride), np.float64)
        self.L.orc_mttkrp_coo_f64(C.c_uint32(N), C.c_uint64(vals.size),
                                  _ptr_array(inds, C.c_uint32), vals.ctypes.data_as(C.c_void_p),
                                  _ptr_array(mats, C.c_double), C.c_uint32(R), C.c_uint32(stride),
                                  C.c_uint32(mode), C.c_uint32(out.shape[0]),
                                  out.ctypes.data_as(C.c_void_p))
        return out

    def mttkrp_hicoo(self, h, mats, R, mode, mats_order=None):
        """h: dict from hicoo_build."""
        N = len(h["binds"])
        stride = mats[0].shape[1]
        if mats_order is None:
            mats_order = [(mode + i) % N for i in range(N)]
        order = np.asarray(mats_order, np.uint32)
        mats = [np.ascontiguousarray(m, np.float32) for m in mats]
        out = np.zeros((mats[mode].shape[0], stride), np.float32)
        nb = h["bptr"].size - 1
        self.L.orc_mttkrp_hicoo_f32(
            C.c_uint32(N), C.c_uint64(h["vals"].size), C.c_uint64(nb), C.c_uint8(h["sb"]),
            h["bptr"].ctypes.data_as(C.c_void_p), _ptr_array(h["binds"], C.c_uint32),
            _ptr_array(h["einds"], C.c_uint8), h["vals"].ctypes.data_as(C.c_void_p),
            _ptr_array(mats, C.c_float), C.c_uint32(R), C.c_uint32(stride), _u32p(order),
            C.c_uint32(mode), C.c_uint32(out.shape[0]), out.ctypes.data_as(C.c_void_p))
        return out

    # -- conversion ----------------------------------------------------------
    def hicoo_build(self, dims, inds, vals, sb, sk, sc):
        N = len(inds)
        inds = [np.ascontiguousarray(i, np.uint32) for i in inds]
        vals = np.ascontiguousarray(vals, np.float32)
        d = np.asarray(dims, np.uint32)
        h = self.L.orc_hicoo_build(N, _u32p(d), vals.size, C.cast(_ptr_array(inds, C.c_uint32), C.c_void_p),
                                   vals.ctypes.data, sb, sk, sc)
        if not h:
            raise ValueError("unsupported tensor for HiCOO conversion")
        cnt = (C.c_uint64 * 5)()
        self.L.orc_hicoo_counts(h, cnt)
        nb, nk, nc, max_nnzb, ktot = [int(x) for x in cnt]
        nnz = vals.size
        krows = sum((int(x) + (1 << sk) - 1) >> sk for x in dims)
        out = dict(
            bptr=np.empty(nb + 1, np.uint64), binds=[np.empty(nb, np.uint32) for _ in range(N)],
            einds=[np.empty(nnz, np.uint8) for _ in range(N)], vals=np.empty(nnz, np.float32),
            kptr=np.empty(nk + 1, np.uint64), cptr=np.empty(nc, np.uint64),
            knnzs=np.empty(nk, np.uint64), perm=np.empty(nnz, np.uint64),
            nkiters=np.empty(N, np.uint32), kschr=np.empty(max(ktot, 1), np.uint32)[:ktot],
            kschr_rowptr=np.empty(krows + 1, np.uint64))
        self.L.orc_hicoo_export(
            h, out["bptr"].ctypes.data, C.cast(_ptr_array(out["binds"], C.c_uint32), C.c_void_p),
            C.cast(_ptr_array(out["einds"], C.c_uint8), C.c_void_p), out["vals"].ctypes.data,
            out["kptr"].ctypes.data, out["cptr"].ctypes.data, out["knnzs"].ctypes.data,
            out["perm"].ctypes.data, out["nkiters"].ctypes.data,
            out["kschr"].ctypes.data if ktot else None, out["kschr_rowptr"].ctypes.data)
        self.L.orc_hicoo_free(h)
        out.update(max_nnzb=max_nnzb, sb=sb, sk=sk, sc=sc)
        return out

    # -- CPD -----------------------------------------------------------------
    def cpd_als(self, dims, inds, vals, R, niters, init_mats):
        """FP64 CPD-ALS from the given initial factors (list of (I_k, R))."""
        N = len(inds)
        inds = [np.ascontiguousarray(i, np.uint32) for i in inds]
        vals = np.ascontiguousarray(vals, np.float32)
        mats = [np.array(m[:, :R], np.float64, order="C") for m in init_mats]
        lam = np.zeros(R, np.float64)
        fits = np.zeros(max(niters, 1), np.float64)
        d = np.asarray(dims, np.uint32)
        fit = self.L.orc_cpd_als_f64(C.c_uint32(N), _u32p(d), C.c_uint64(vals.size),
                                     _ptr_array(inds, C.c_uint32), vals.ctypes.data_as(C.c_void_p),
                                     C.c_uint32(R), C.c_uint32(niters), _ptr_array(mats, C.c_double),
                                     lam.ctypes.data_as(C.c_void_p), fits.ctypes.data_as(C.c_void_p))
        return dict(fit=fit, fits=fits[:niters], lambda_=lam, factors=mats)

    def kruskal_fit(self, dims, inds, vals, lam, mats):
        N = len(inds)
        R = lam.size
        inds = [np.ascontiguousarray(i, np.uint32) for i in inds]
        vals = np.ascontiguousarray(vals, np.float32)
        mats = [np.ascontiguousarray(m[:, :R], np.float64) for m in mats]
        lam = np.ascontiguousarray(lam, np.float64)
        d = np.asarray(dims, np.uint32)
        return self.L.orc_kruskal_fit_f64(C.c_uint32(N), _u32p(d), C.c_uint64(vals.size),
                                          _ptr_array(inds, C.c_uint32), vals.ctypes.data_as(C.c_void_p),
                                          C.c_uint32(R), _ptr_array(mats, C.c_double),
                                          lam.ctypes.data_as(C.c_void_p))


def bfs_like(dims, inds):
    """BFS-like renumbering (src/sptensor/renumber.c:534-839; ptiIndexRenumber
    with renumber == 2), restated with every vertex starting unvisited (the
    reference reads the visit marks of other modes' vertices without setting
    them, renumber.c:768).  The tensor is a hypergraph: a vertex per index of
    every mode, a hyperedge per nonzero.  Mode by mode, the mode's vertices are
    taken from a binary max-heap on a key, all keys 0 at first; the heap
    compares the keys, and on equal keys prefers the smaller degree when it
    sifts down (heapify, :666-701) and the larger degree when it sifts up
    (heapIncreaseKey, :644-664).  The vertex taken gets the next new index;
    every vertex of its hyperedges not yet visited in this mode's pass is
    visited, and each hyperedge of that vertex raises by one the key of its
    own vertex in the mode, if still in the heap.  Returns newIndices per
    mode (old index -> new).  Pure Python: small tensors only."""
    N = len(dims)
    dims = [int(d) for d in dims]
    inds = [np.asarray(i, np.int64) for i in inds]
    nnz = inds[0].size if N else 0
    lists = []
    for m in range(N):
        order = np.argsort(inds[m], kind="stable")
        off = np.searchsorted(inds[m][order], np.arange(dims[m] + 1), side="left")
        lists.append((order, off))
    out = []
    for d in range(N):
        order_d, off_d = lists[d]
        deg = np.diff(off_d)
        n = dims[d]
        heap = [0] + list(range(n))
        pos = list(range(1, n + 1))  # pos[v]: heap slot of v, 0 once taken
        key = [0] * n
        size = n

        def down(j):
            while j <= size // 2:
                l, r = 2 * j, 2 * j + 1
                big = l if (key[heap[l]] > key[heap[j]] or
                            (key[heap[l]] == key[heap[j]] and deg[heap[l]] < deg[heap[j]])) else j
                if r <= size and (key[heap[r]] > key[heap[big]] or
                                  (key[heap[r]] == key[heap[big]] and deg[heap[r]] < deg[heap[big]])):
                    big = r
                if big == j:
                    break
                heap[big], heap[j] = heap[j], heap[big]
                pos[heap[big]], pos[heap[j]] = big, j
                j = big

        def up(v):
            i = pos[v]
            key[v] += 1
            while i > 1 and (key[v] > key[heap[i >> 1]] or
                             (key[v] == key[heap[i >> 1]] and deg[v] > deg[heap[i >> 1]])):
                heap[i] = heap[i >> 1]
                pos[heap[i]] = i
                i >>= 1
            heap[i] = v
            pos[v] = i

        for j in range(size // 2, 0, -1):
            down(j)
        visited = [np.zeros(dims[m], bool) for m in range(N)]
        new = np.zeros(n, np.uint32)
        for t in range(n):
            v = heap[1]
            heap[1] = heap[size]
            pos[heap[1]] = 1
            size -= 1
            pos[v] = 0
            down(1)
            new[v] = t
            for h in order_d[off_d[v]:off_d[v + 1]]:
                for k in range(N):
                    if k == d:
                        continue
                    w = inds[k][h]
                    if visited[k][w]:
                        continue
                    visited[k][w] = True
                    ok, oo = lists[k]
                    for h2 in ok[oo[w]:oo[w + 1]]:
                        u = inds[d][h2]
                        if pos[u]:
                            up(u)
        out.append(new)
    return out


# ----------------------------------------------------------------------------
# The reference library (compiled from its own sources)
# ----------------------------------------------------------------------------
def lexi_order(dims, inds, iterations):
    """Lexi-order renumbering restated (src/sptensor/renumber.c:26-92,
    403-520; lexOrderThem :93-225).  For each mode in turn, `iterations` times:
    rows are the other modes' coordinate tuples in lexicographic order (the
    other modes ascending), each index's list is its rows in ascending order,
    and the indices are ordered by their lists, where at the first differing
    row the index present in that row comes first (a list precedes its own
    prefixes; indices without nonzeros come last).  This is the order the
    reference's partition refinement over the rows yields.  Indices with equal
    lists keep their current order.  Pure Python: small tensors only.
    Returns newIndices (per mode, original index -> new index)."""
    N = len(dims)
    cur = [np.asarray(i, np.int64).copy() for i in inds]
    org = [np.arange(d) for d in dims]          # current index -> original
    nnz = cur[0].size
    for _ in range(iterations):
        for m in range(N):
            others = [k for k in range(N) if k != m]
            tuples = sorted({tuple(int(cur[k][z]) for k in others) for z in range(nnz)})
            rid = {t: r for r, t in enumerate(tuples)}
            lists = [[] for _ in range(dims[m])]
            for z in range(nnz):
                lists[int(cur[m][z])].append(rid[tuple(int(cur[k][z]) for k in others)])
            inf = len(tuples)
            order = sorted(range(dims[m]), key=lambda c: (tuple(sorted(lists[c])) + (inf,), c))
            inv = np.empty(dims[m], np.int64)
            inv[np.asarray(order, np.int64)] = np.arange(dims[m])
            cur[m] = inv[cur[m]]
            org[m] = org[m][np.asarray(order, np.int64)]
    out = []
    for m in range(N):
        mp = np.empty(dims[m], np.uint32)
        mp[org[m]] = np.arange(dims[m], dtype=np.uint32)
        out.append(mp)
    return out


class _Vec(C.Structure):
    _fields_ = [("len", C.c_uint64), ("cap", C.c_uint64), ("data", C.c_void_p)]


class _Matrix(C.Structure):
    _fields_ = [("nrows", C.c_uint32), ("ncols", C.c_uint32), ("cap", C.c_uint32),
                ("stride", C.c_uint32), ("values", C.c_void_p)]


class _RankMatrix(C.Structure):
    _fields_ = [("nrows", C.c_uint32), ("ncols", C.c_uint8), ("cap", C.c_uint32),
                ("stride", C.c_uint8), ("values", C.c_void_p)]


class _SpTensor(C.Structure):
    _fields_ = [("nmodes", C.c_uint32), ("sortorder", C.c_void_p), ("ndims", C.c_void_p),
                ("nnz", C.c_uint64), ("inds", C.POINTER(_Vec)), ("values", _Vec)]


class _HiCOO(C.Structure):
    _fields_ = [("nmodes", C.c_uint32), ("sortorder", C.c_void_p), ("ndims", C.c_void_p),
                ("nnz", C.c_uint64), ("sb_bits", C.c_uint8), ("sk_bits", C.c_uint8),
                ("sc_bits", C.c_uint8), ("kptr", _Vec), ("kschr", C.POINTER(C.POINTER(_Vec))),
                ("nkiters", C.POINTER(C.c_uint32)), ("cptr", _Vec),
                ("kschr_balanced", C.c_void_p), ("kschr_balanced_pos", C.c_void_p),
                ("nkpars", C.c_void_p), ("kschr_rest", C.c_void_p), ("knnzs", _Vec),
                ("bptr", _Vec), ("binds", C.POINTER(_Vec)), ("einds", C.POINTER(_Vec)),
                ("values", _Vec)]


assert C.sizeof(_HiCOO) == 224 and C.sizeof(_SpTensor) == 64 and C.sizeof(_Matrix) == 24


class _SemiSparse(C.Structure):
    _fields_ = [("nmodes", C.c_uint32), ("ndims", C.c_void_p), ("mode", C.c_uint32), ("nnz", C.c_uint64),
                ("inds", C.POINTER(_Vec)), ("stride", C.c_uint32), ("values", _Matrix)]


def _np_from(ptr, n, dtype):
    if n == 0:
        return np.empty(0, dtype)
    buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=n).copy()


class Ref:
    """The reference's own CPU implementation (oracle/_ref/libHiParTI.so)."""

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self):
        if not REF_SO.exists():
            ensure_built(ref=True)
        if not REF_SO.exists():
            raise RuntimeError("reference library not built (needs the reference sources)")
        self.L = C.CDLL(str(REF_SO), mode=C.RTLD_LOCAL)
        self.L.CpdAlsStep.restype = C.c_double
        self.L.OmpCpdAlsStep.restype = C.c_double

    def load(self, fname, start_index=1):
        """ptiLoadSparseTensor of the reference.  Returns (rc, dims, inds, vals)."""
        t = _SpTensor()
        rc = self.L.ptiLoadSparseTensor(C.byref(t), C.c_uint32(start_index), str(fname).encode())
        if rc != 0:
            return rc, None, None, None
        N, nnz = int(t.nmodes), int(t.nnz)
        dims = list(_np_from(t.ndims, N, np.uint32))
        inds = [_np_from(t.inds[m].data, nnz, np.uint32) for m in range(N)]
        vals = _np_from(t.values.data, nnz, np.float32)
        self.L.ptiFreeSparseTensor(C.byref(t))
        return 0, dims, inds, vals

    def renumber(self, dims, inds, vals, iterations, impl_num=1):
        """ptiIndexRenumber(renumber=1) of the reference: newIndices per mode."""
        t, keep = self._coo(dims, inds, vals)
        maps = [np.zeros(d, np.uint32) for d in dims]
        arr = (C.c_void_p * len(dims))(*[m.ctypes.data for m in maps])
        self.L.ptiIndexRenumber(C.byref(t), arr, C.c_int(1), C.c_uint32(iterations), C.c_uint8(7), C.c_int(1),
                                C.c_int(impl_num))
        return maps

    def ttm(self, dims, inds, vals, U, mode, sortorder=None, vector=False):
        """ptiSparseTensorMulMatrix (or, with vector=True and U a vector,
        ptiSparseTensorMulVector) of the reference.  Returns (fiber inds per
        mode, Y values nfibers x stride, X's arrays after the call, X's
        sortorder after the call)."""
        t, keep = self._coo(dims, inds, vals)
        if sortorder is not None:
            keep["sortorder"][:] = sortorder
        Y = _SemiSparse()
        if vector:
            v = np.ascontiguousarray(U, np.float32)
            vec = _Vec(v.size, v.size, v.ctypes.data)
            rc = self.L.ptiSparseTensorMulVector(C.byref(Y), C.byref(t), C.byref(vec), C.c_uint32(mode))
        else:
            R = U.shape[1]
            st = ((R - 1) // 8 + 1) * 8
            buf = np.zeros((U.shape[0], st), np.float32)
            buf[:, :R] = U
            m = _Matrix(U.shape[0], R, U.shape[0], st, buf.ctypes.data)
            rc = self.L.ptiSparseTensorMulMatrix(C.byref(Y), C.byref(t), C.byref(m), C.c_uint32(mode))
        assert rc == 0
        nf, st = int(Y.nnz), int(Y.stride)
        finds = [_np_from(Y.inds[m].data, int(Y.inds[m].len), np.uint32) if Y.inds[m].len else np.empty(0, np.uint32)
                 for m in range(len(dims))]
        yv = _np_from(Y.values.values, nf * st, np.float32).reshape(nf, st) if nf else np.empty((0, st), np.float32)
        after = ([k.copy() for k in keep["inds"]], keep["vals"].copy(), keep["sortorder"].copy())
        return finds, yv, after

    def ssp_to_sparse(self, Y, epsilon):
        """ptiSemiSparseTensorToSparseTensor of the reference on a ttm() result
        dict (mode, dims, inds, vals).  Returns (inds, vals)."""
        N, mode = len(Y["dims"]), Y["mode"]
        nf, st = Y["vals"].shape
        keep = {"dims": np.asarray(Y["dims"], np.uint32).copy(),
                "vals": np.ascontiguousarray(Y["vals"], np.float32).copy(),
                "inds": [np.ascontiguousarray(i, np.uint32).copy() for i in Y["inds"]]}
        vecs = (_Vec * N)(*[_Vec(keep["inds"][m].size, keep["inds"][m].size, keep["inds"][m].ctypes.data)
                            for m in range(N)])
        y = _SemiSparse(N, keep["dims"].ctypes.data, mode, nf, vecs, st,
                        _Matrix(nf, st, nf, st, keep["vals"].ctypes.data))
        t = _SpTensor()
        rc = self.L.ptiSemiSparseTensorToSparseTensor(C.byref(t), C.byref(y), C.c_float(epsilon))
        assert rc == 0
        nnz = int(t.nnz)
        inds = [_np_from(t.inds[m].data, nnz, np.uint32) for m in range(N)]
        return inds, _np_from(t.values.data, nnz, np.float32)

    def ssp_ttm(self, Y, U):
        """ptiSemiSparseTensorMulMatrix of the reference on a ttm() result dict.
        Returns (fiber inds per mode, values nfibers x stride)."""
        N, mode = len(Y["dims"]), Y["mode"]
        nf, st = Y["vals"].shape
        keep = {"dims": np.asarray(Y["dims"], np.uint32).copy(),
                "vals": np.ascontiguousarray(Y["vals"], np.float32).copy(),
                "inds": [np.ascontiguousarray(i, np.uint32).copy() for i in Y["inds"]]}
        vecs = (_Vec * N)(*[_Vec(keep["inds"][m].size, keep["inds"][m].size, keep["inds"][m].ctypes.data)
                            for m in range(N)])
        y = _SemiSparse(N, keep["dims"].ctypes.data, mode, nf, vecs, st,
                        _Matrix(nf, st, nf, st, keep["vals"].ctypes.data))
        R = U.shape[1]
        ust = ((R - 1) // 8 + 1) * 8
        buf = np.zeros((U.shape[0], ust), np.float32)
        buf[:, :R] = U
        m = _Matrix(U.shape[0], R, U.shape[0], ust, buf.ctypes.data)
        out = _SemiSparse()
        rc = self.L.ptiSemiSparseTensorMulMatrix(C.byref(out), C.byref(y), C.byref(m), C.c_uint32(mode))
        assert rc == 0
        n2, st2 = int(out.nnz), int(out.stride)
        finds = [_np_from(out.inds[k].data, int(out.inds[k].len), np.uint32) if out.inds[k].len
                 else np.empty(0, np.uint32) for k in range(N)]
        vals = _np_from(out.values.values, n2 * st2, np.float32).reshape(n2, st2) if n2 else \
            np.empty((0, st2), np.float32)
        return finds, vals

    @staticmethod
    def bfs_available() -> bool:
        return BFS_SO.exists()

    def bfs_like(self, dims, inds, vals):
        """The reference's ptiBFSLike (src/sptensor/renumber.c:794-839) from
        oracle/_ref/libbfsref.so: its own source compiled with an allocator that
        fills fresh blocks with 0xFF (oracle/ff_malloc.c), so the visit marks it
        reads before writing are -1 ("not visited") and the result is
        deterministic.  newIndices per mode."""
        if not hasattr(self, "_bfs"):
            self._bfs = C.CDLL(str(BFS_SO), mode=C.RTLD_LOCAL)
        t, keep = self._coo(dims, inds, vals)
        maps = [np.zeros(d, np.uint32) for d in dims]
        arr = (C.c_void_p * len(dims))(*[m.ctypes.data for m in maps])
        self._bfs.ptiBFSLike(C.byref(t), arr)
        return maps

    def orderit(self, dims, inds, vals, iterations):
        """orderit(renumber=1) of the reference (src/sptensor/orderit.c:121-208),
        its Lexi-order driver with a correct coordinate sort."""
        t, keep = self._coo(dims, inds, vals)
        maps = [np.zeros(d, np.uint32) for d in dims]
        arr = (C.c_void_p * len(dims))(*[m.ctypes.data for m in maps])
        self.L.orderit(C.byref(t), arr, C.c_int(1), C.c_uint32(iterations))
        return maps

    # A COO tensor whose arrays point into numpy buffers owned by `keep`.
    def _coo(self, dims, inds, vals):
        N = len(inds)
        keep = {}
        keep["inds"] = [np.ascontiguousarray(i, np.uint32).copy() for i in inds]
        keep["vals"] = np.ascontiguousarray(vals, np.float32).copy()
        keep["dims"] = np.asarray(dims, np.uint32).copy()
        keep["sortorder"] = np.arange(N, dtype=np.uint32)
        vecs = (_Vec * N)()
        for m in range(N):
            vecs[m] = _Vec(keep["vals"].size, keep["vals"].size, keep["inds"][m].ctypes.data)
        keep["vecs"] = vecs
        t = _SpTensor(N, keep["sortorder"].ctypes.data, keep["dims"].ctypes.data, keep["vals"].size,
                      vecs, _Vec(keep["vals"].size, keep["vals"].size, keep["vals"].ctypes.data))
        return t, keep

    @staticmethod
    def _mats(mats_np, R):
        ms = []
        for a in mats_np:
            ms.append(_Matrix(a.shape[0], R, a.shape[0], a.shape[1], a.ctypes.data))
        arr = (C.POINTER(_Matrix) * len(ms))(*[C.pointer(m) for m in ms])
        return arr, ms

    def mttkrp_coo(self, dims, inds, vals, mats, R, mode, variant="seq", tk=8):
        N = len(inds)
        t, keep = self._coo(dims, inds, vals)
        stride = mats[0].shape[1]
        fac = [np.ascontiguousarray(m, np.float32) for m in mats]
        out = np.zeros((max(dims), stride), np.float32)
        arr, ms = self._mats(fac + [out], R)
        order = np.asarray([(mode + i) % N for i in range(N)], np.uint32)
        if variant == "seq":
            rc = self.L.ptiMTTKRP(C.byref(t), arr, _u32p(order), C.c_uint32(mode))
        elif variant == "omp":
            rc = self.L.ptiOmpMTTKRP(C.byref(t), arr, _u32p(order), C.c_uint32(mode), C.c_int(tk))
        else:
            cm = [np.zeros((dims[mode], stride), np.float32) for _ in range(tk)]
            carr, cms = self._mats(cm, R)
            rc = self.L.ptiOmpMTTKRP_Reduce(C.byref(t), arr, carr, _u32p(order), C.c_uint32(mode),
                                            C.c_int(tk))
        assert rc == 0
        return out[: dims[mode]].copy()

    def to_hicoo(self, dims, inds, vals, sb, sk, sc):
        """Runs ptiSparseTensorToHiCOO(tk=1); returns the arrays and the COO
        order it leaves behind (the reference sorts its input in place)."""
        N = len(inds)
        t, keep = self._coo(dims, inds, vals)
        h = _HiCOO()
        maxnb = C.c_uint64(0)
        rc = self.L.ptiSparseTensorToHiCOO(C.byref(h), C.byref(maxnb), C.byref(t), C.c_uint8(sb),
                                           C.c_uint8(sk), C.c_uint8(sc), C.c_int(1))
        assert rc == 0
        nb = int(h.bptr.len) - 1
        nnz = int(h.nnz)
        res = dict(
            bptr=_np_from(h.bptr.data, nb + 1, np.uint64),
            binds=[_np_from(h.binds[m].data, nb, np.uint32) for m in range(N)],
            einds=[_np_from(h.einds[m].data, nnz, np.uint8) for m in range(N)],
            vals=_np_from(h.values.data, nnz, np.float32),
            kptr=_np_from(h.kptr.data, int(h.kptr.len), np.uint64),
            cptr=_np_from(h.cptr.data, int(h.cptr.len), np.uint64),
            knnzs=_np_from(h.knnzs.data, int(h.knnzs.len), np.uint64),
            nkiters=_np_from(C.cast(h.nkiters, C.c_void_p).value, N, np.uint32),
            max_nnzb=int(maxnb.value), sb=sb, sk=sk, sc=sc,
            sorted_inds=[keep["inds"][m].copy() for m in range(N)],
            sorted_vals=keep["vals"].copy())
        rows = []
        for m in range(N):
            for i in range((int(dims[m]) + (1 << sk) - 1) >> sk):
                v = h.kschr[m][i]
                rows.append(_np_from(v.data, int(v.len), np.uint32))
        res["kschr_rows"] = rows
        # balanced scheduler (convert.c:475-571)
        kb = C.cast(h.kschr_balanced, C.POINTER(C.POINTER(_Vec)))
        kp = C.cast(h.kschr_balanced_pos, C.POINTER(C.POINTER(_Vec)))
        kr = C.cast(h.kschr_rest, C.POINTER(_Vec))
        bal, pos, rest = [], [], []
        for m in range(N):
            for i in range((int(dims[m]) + (1 << sk) - 1) >> sk):
                bal.append(_np_from(kb[m][i].data, int(kb[m][i].len), np.uint32))
                pos.append(_np_from(kp[m][i].data, int(kp[m][i].len), np.uint32))
            rest.append(_np_from(kr[m].data, int(kr[m].len), np.uint32))
        res["kschr_balanced_rows"] = bal
        res["kschr_balanced_pos_rows"] = pos
        res["kschr_rest"] = rest
        res["nkpars"] = _np_from(h.nkpars, N, np.uint32)
        self.L.ptiFreeSparseTensorHiCOO(C.byref(h))
        return res

    def _hicoo_struct(self, h, dims):
        N = len(h["binds"])
        keep = {"h": h}
        keep["dims"] = np.asarray(dims, np.uint32).copy()
        keep["so"] = np.arange(N, dtype=np.uint32)
        nb = h["bptr"].size - 1
        nnz = h["vals"].size
        bv = (_Vec * N)(*[_Vec(nb, nb, h["binds"][m].ctypes.data) for m in range(N)])
        ev = (_Vec * N)(*[_Vec(nnz, nnz, h["einds"][m].ctypes.data) for m in range(N)])
        keep["bv"], keep["ev"] = bv, ev
        hs = _HiCOO()
        hs.nmodes = N
        hs.sortorder = keep["so"].ctypes.data
        hs.ndims = keep["dims"].ctypes.data
        hs.nnz = nnz
        hs.sb_bits, hs.sk_bits, hs.sc_bits = h["sb"], h["sk"], h["sc"]
        hs.kptr = _Vec(h["kptr"].size, h["kptr"].size, h["kptr"].ctypes.data)
        hs.bptr = _Vec(nb + 1, nb + 1, h["bptr"].ctypes.data)
        hs.binds = bv
        hs.einds = ev
        hs.values = _Vec(nnz, nnz, h["vals"].ctypes.data)
        return hs, keep

    def mttkrp_hicoo(self, dims, h, mats, R, mode, variant="seq", tk=8):
        N = len(h["binds"])
        hs, keep = self._hicoo_struct(h, dims)
        stride = mats[0].shape[1]
        fac = [np.ascontiguousarray(m, np.float32) for m in mats]
        out = np.zeros((max(dims), stride), np.float32)
        arr, ms = self._mats(fac + [out], R)
        order = np.asarray([(mode + i) % N for i in range(N)], np.uint32)
        if variant == "seq":
            rc = self.L.ptiMTTKRPHiCOO(C.byref(hs), arr, _u32p(order), C.c_uint32(mode))
        else:
            rc = self.L.ptiOmpMTTKRPHiCOO(C.byref(hs), arr, _u32p(order), C.c_uint32(mode),
                                          C.c_int(tk), C.c_int(1))
        assert rc == 0
        return out[: dims[mode]].copy()

    def omp_hicoo_mttkrp_runner(self, dims, h, mats, R, tk):
        """A callable mode -> output for repeated ptiOmpMTTKRPHiCOO(tk, tb=1)
        calls on the same HiCOO tensor and factors, with the C structs built
        once (so a timed loop measures the reference call alone).  Every call
        overwrites the returned output array's first dims[mode] rows."""
        N = len(h["binds"])
        hs, keep = self._hicoo_struct(h, dims)
        stride = mats[0].shape[1]
        fac = [np.ascontiguousarray(m, np.float32) for m in mats]
        out = np.zeros((max(dims), stride), np.float32)
        arr, ms = self._mats(fac + [out], R)
        orders = [np.asarray([(m + i) % N for i in range(N)], np.uint32) for m in range(N)]
        keep.update(fac=fac, arr=arr, ms=ms, orders=orders)

        def run(mode):
            _ = keep
            rc = self.L.ptiOmpMTTKRPHiCOO(C.byref(hs), arr, _u32p(orders[mode]), C.c_uint32(mode),
                                          C.c_int(tk), C.c_int(1))
            assert rc == 0
            return out
        return run

    def mttkrp_hicoo_rank(self, dims, h, mats, R, mode):
        """ptiMTTKRPHiCOO_MatrixTiling (ptiRankMatrix factors) of the reference."""
        N = len(h["binds"])
        hs, keep = self._hicoo_struct(h, dims)
        stride = mats[0].shape[1]
        fac = [np.ascontiguousarray(m, np.float32) for m in mats]
        out = np.zeros((max(dims), stride), np.float32)
        ms = [_RankMatrix(a.shape[0], R, a.shape[0], stride, a.ctypes.data) for a in fac + [out]]
        ms[-1].nrows = dims[mode]
        arr = (C.POINTER(_RankMatrix) * len(ms))(*[C.pointer(m) for m in ms])
        order = np.asarray([(mode + i) % N for i in range(N)], np.uint32)
        rc = self.L.ptiMTTKRPHiCOO_MatrixTiling(C.byref(hs), arr, _u32p(order), C.c_uint32(mode))
        assert rc == 0
        return out[: dims[mode]].copy()

    def cpd_als_step(self, dims, inds, vals, R, niters, init_mats, tk=0):
        """CpdAlsStep (tk=0) or OmpCpdAlsStep(tk, use_reduce=0) from the given
        FP32 factors with tol=0.  Returns (fit, lambda, factors)."""
        N = len(inds)
        t, keep = self._coo(dims, inds, vals)
        stride = ((R - 1) // 8 + 1) * 8
        fac = []
        for m in init_mats:
            a = np.zeros((m.shape[0], stride), np.float32)
            a[:, :R] = m[:, :R]
            fac.append(a)
        tmp = np.zeros((max(dims), stride), np.float32)
        arr, ms = self._mats(fac + [tmp], R)
        lam = np.zeros(R, np.float32)
        if tk:
            fit = self.L.OmpCpdAlsStep(C.byref(t), C.c_uint32(R), C.c_uint32(niters), C.c_double(0.0),
                                       C.c_int(tk), C.c_int(0), arr, None, lam.ctypes.data_as(C.c_void_p))
        else:
            fit = self.L.CpdAlsStep(C.byref(t), C.c_uint32(R), C.c_uint32(niters), C.c_double(0.0), arr,
                                    lam.ctypes.data_as(C.c_void_p))
        return fit, lam, [f[:, :R].copy() for f in fac]
