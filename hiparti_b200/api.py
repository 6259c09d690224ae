"""Python mirror of the reference's Python layer (HiParTIPy/Tensor.py,
HiParTIPy/Matrix.py) for the MTTKRP / CPD path, over the C ABI.

Host-side objects (``COOTensor``, ``HiCOOTensor``) hold numpy arrays and hand
the library struct views of them, so every call goes through the same C entry
points a C program uses.  ``DeviceTensor`` keeps a tensor resident on the GPU
(``ptiB200*`` extensions) and takes torch CUDA tensors as factors.
"""
from __future__ import annotations

import numpy as np

from ._ffi import PtiError, check, ffi, lib

_F32 = 0
_BF16 = 1


def _stride(R: int) -> int:
    return ((R - 1) // 8 + 1) * 8


def _ptr(arr, ctype):
    return ffi.cast(ctype, arr.ctypes.data)


class _MatrixSet:
    """N+1 ptiMatrix structs over numpy arrays (factors + output)."""

    def __init__(self, arrays, R):
        self.arrays = arrays
        self.structs = ffi.new("ptiMatrix[]", len(arrays))
        self.ptrs = ffi.new("ptiMatrix *[]", len(arrays))
        for i, a in enumerate(arrays):
            s = self.structs[i]
            s.nrows = a.shape[0]
            s.ncols = R
            s.cap = a.shape[0]
            s.stride = a.shape[1]
            s.values = _ptr(a, "float *")
            self.ptrs[i] = ffi.addressof(self.structs, i)


class COOTensor:
    """A COO sparse tensor whose index/value arrays live in numpy."""

    def __init__(self, dims, inds, vals):
        self.dims = [int(d) for d in dims]
        self.inds = [np.ascontiguousarray(i, dtype=np.uint32) for i in inds]
        self.vals = np.ascontiguousarray(vals, dtype=np.float32)
        if len(self.inds) != len(self.dims):
            raise ValueError("one index array per mode")
        if any(i.size != self.vals.size for i in self.inds):
            raise ValueError("index and value arrays differ in length")
        self._build()

    @classmethod
    def load(cls, fname: str, start_index: int = 1) -> "COOTensor":
        """ptiLoadSparseTensor (text .tns or SPLATT .bin)."""
        t = ffi.new("ptiSparseTensor *")
        check(lib().ptiLoadSparseTensor(t, start_index, fname.encode()), "ptiLoadSparseTensor")
        N, nnz = t.nmodes, t.nnz
        dims = [t.ndims[m] for m in range(N)]
        inds = [np.frombuffer(ffi.buffer(t.inds[m].data, 4 * nnz), np.uint32).copy() for m in range(N)]
        vals = np.frombuffer(ffi.buffer(t.values.data, 4 * nnz), np.float32).copy()
        lib().ptiFreeSparseTensor(t)
        return cls(dims, inds, vals)

    def _build(self):
        N = len(self.dims)
        self._dims = np.asarray(self.dims, np.uint32)
        self._so = np.arange(N, dtype=np.uint32)
        self._vecs = ffi.new("ptiIndexVector[]", N)
        for m in range(N):
            self._vecs[m].len = self._vecs[m].cap = self.vals.size
            self._vecs[m].data = _ptr(self.inds[m], "ptiIndex *")
        self.c = ffi.new("ptiSparseTensor *")
        self.c.nmodes = N
        self.c.sortorder = _ptr(self._so, "ptiIndex *")
        self.c.ndims = _ptr(self._dims, "ptiIndex *")
        self.c.nnz = self.vals.size
        self.c.inds = self._vecs
        self.c.values.len = self.c.values.cap = self.vals.size
        self.c.values.data = _ptr(self.vals, "ptiValue *")

    @property
    def nmodes(self):
        return len(self.dims)

    @property
    def nnz(self):
        return int(self.vals.size)

    def mttkrp(self, mats, R, mode, variant="seq"):
        """Runs the reference entry point `variant` ("seq" -> ptiMTTKRP, "omp"
        -> ptiOmpMTTKRP, "cuda" -> ptiCudaMTTKRP, "onekernel" ->
        ptiCudaMTTKRPOneKernel) on the GPU; returns (dims[mode], stride)."""
        return _host_mttkrp(self, mats, R, mode, variant)

    def to_hicoo(self, sb=7, sk=10, sc=14) -> "HiCOOTensor":
        """ptiSparseTensorToHiCOO (GPU).  As in the reference, this tensor's
        arrays are left sorted in HiCOO order."""
        h = ffi.new("ptiSparseTensorHiCOO *")
        maxnb = ffi.new("ptiNnzIndex *")
        check(lib().ptiSparseTensorToHiCOO(h, maxnb, self.c, sb, sk, sc, 1), "ptiSparseTensorToHiCOO")
        out = HiCOOTensor._from_struct(h, int(maxnb[0]))
        lib().ptiFreeSparseTensorHiCOO(h)
        return out

    def cpd_als(self, R, niters, tol=0.0, variant="seq"):
        return _host_cpd(self, R, niters, tol, variant)

    def _semi_sparse(self, Y):
        N, nf, st = Y.nmodes, Y.nnz, Y.stride
        inds = [np.frombuffer(ffi.buffer(Y.inds[m].data, 4 * Y.inds[m].len), np.uint32).copy()
                if Y.inds[m].len else np.empty(0, np.uint32) for m in range(N)]
        vals = (np.frombuffer(ffi.buffer(Y.values.values, 4 * nf * st), np.float32).reshape(nf, st).copy()
                if nf else np.empty((0, st), np.float32))
        dims = [int(Y.ndims[m]) for m in range(N)]
        mode = int(Y.mode)
        lib().ptiFreeSemiSparseTensor(Y)
        return {"mode": mode, "dims": dims, "inds": inds, "vals": vals}

    @staticmethod
    def _semi_struct(Y, keep):
        N, mode = len(Y["dims"]), Y["mode"]
        nf, st = Y["vals"].shape
        keep["dims"] = np.asarray(Y["dims"], np.uint32)
        keep["vals"] = np.ascontiguousarray(Y["vals"], np.float32)
        keep["inds"] = [np.ascontiguousarray(i, np.uint32) for i in Y["inds"]]
        y = ffi.new("ptiSemiSparseTensor *")
        y.nmodes, y.mode, y.nnz, y.stride = N, mode, nf, st
        y.ndims = _ptr(keep["dims"], "ptiIndex *")
        vecs = ffi.new("ptiIndexVector[]", N)
        keep["vecs"] = vecs
        for m in range(N):
            vecs[m].len = vecs[m].cap = keep["inds"][m].size
            vecs[m].data = _ptr(keep["inds"][m], "ptiIndex *") if keep["inds"][m].size else ffi.NULL
        y.inds = vecs
        y.values.nrows, y.values.ncols, y.values.cap, y.values.stride = nf, st, nf, st
        y.values.values = _ptr(keep["vals"], "ptiValue *") if nf else ffi.NULL
        return y

    @classmethod
    def semi_sparse_ttm(cls, Y, U):
        """ptiSemiSparseTensorMulMatrix on a ttm()/ttv() result: its dense
        fibers (ndims[mode] columns used) times U, in the same layout."""
        keep = {}
        y = cls._semi_struct(Y, keep)
        U = np.ascontiguousarray(U, np.float32)
        I, R = U.shape
        st = ((R - 1) // 8 + 1) * 8
        buf = np.zeros((I, st), np.float32)
        buf[:, :R] = U
        m = ffi.new("ptiMatrix *")
        m.nrows, m.ncols, m.cap, m.stride = I, R, I, st
        m.values = _ptr(buf, "ptiValue *")
        out = ffi.new("ptiSemiSparseTensor *")
        check(lib().ptiSemiSparseTensorMulMatrix(out, y, m, Y["mode"]), "ptiSemiSparseTensorMulMatrix")
        return cls._semi_sparse(None, out)

    @classmethod
    def from_semi_sparse(cls, Y, epsilon=1e-6) -> "COOTensor":
        """ptiSemiSparseTensorToSparseTensor of a ttm()/ttv() result: the
        entries that are NaN, infinite or normal with |v| >= epsilon, sorted."""
        N = len(Y["dims"])
        keep = {}
        y = cls._semi_struct(Y, keep)
        t = ffi.new("ptiSparseTensor *")
        check(lib().ptiSemiSparseTensorToSparseTensor(t, y, float(epsilon)), "ptiSemiSparseTensorToSparseTensor")
        nnz = t.nnz
        dims = [t.ndims[m] for m in range(N)]
        inds = [np.frombuffer(ffi.buffer(t.inds[m].data, 4 * nnz), np.uint32).copy() if nnz
                else np.empty(0, np.uint32) for m in range(N)]
        vals = np.frombuffer(ffi.buffer(t.values.data, 4 * nnz), np.float32).copy() if nnz else np.empty(0, np.float32)
        lib().ptiFreeSparseTensor(t)
        return cls(dims, inds, vals)

    def ttm(self, U, mode):
        """ptiSparseTensorMulMatrix: returns {"mode", "inds" (fiber coordinates
        per mode, the mode's own empty), "vals" (nfibers x stride)}.  As in the
        reference, this tensor's arrays are left sorted with `mode` last."""
        U = np.ascontiguousarray(U, np.float32)
        I, R = U.shape
        st = ((R - 1) // 8 + 1) * 8
        buf = np.zeros((I, st), np.float32)
        buf[:, :R] = U
        m = ffi.new("ptiMatrix *")
        m.nrows, m.ncols, m.cap, m.stride = I, R, I, st
        m.values = _ptr(buf, "ptiValue *")
        Y = ffi.new("ptiSemiSparseTensor *")
        check(lib().ptiSparseTensorMulMatrix(Y, self.c, m, mode), "ptiSparseTensorMulMatrix")
        return self._semi_sparse(Y)

    def ttv(self, v, mode):
        """ptiSparseTensorMulVector (same result layout as ttm, width 1)."""
        v = np.ascontiguousarray(v, np.float32)
        vec = ffi.new("ptiValueVector *")
        vec.len = vec.cap = v.size
        vec.data = _ptr(v, "ptiValue *")
        Y = ffi.new("ptiSemiSparseTensor *")
        check(lib().ptiSparseTensorMulVector(Y, self.c, vec, mode), "ptiSparseTensorMulVector")
        return self._semi_sparse(Y)

    def renumber(self, iterations=1, method="lexi", impl_num=1):
        """Index renumbering (ptiIndexRenumber): method "lexi" (Lexi-order,
        renumber = 1, on the GPU, `iterations` passes) or "bfs" (BFS-like,
        renumber = 2).  Per mode, original index -> new index.  The tensor is
        not changed."""
        maps = [np.empty(d, np.uint32) for d in self.dims]
        mp = ffi.new("ptiIndex *[]", [ffi.cast("ptiIndex *", m.ctypes.data) for m in maps])
        renumber = {"lexi": 1, "bfs": 2}[method]
        lib().ptiClearLastError()
        lib().ptiIndexRenumber(self.c, mp, renumber, int(iterations), 7, 1, int(impl_num))
        code = lib().ptiGetLastError(ffi.NULL, ffi.NULL, ffi.NULL, ffi.NULL)
        if code:
            raise PtiError(code, "ptiIndexRenumber")
        return maps

    def shuffled(self, maps):
        """A copy with every coordinate replaced by maps[m][old] (ptiSparseTensorShuffleIndices)."""
        t = COOTensor(self.dims, [i.copy() for i in self.inds], self.vals.copy())
        keep = [np.ascontiguousarray(m, np.uint32) for m in maps]
        mp = ffi.new("ptiIndex *[]", [ffi.cast("ptiIndex *", m.ctypes.data) for m in keep])
        lib().ptiSparseTensorShuffleIndices(t.c, mp)
        return t


class HiCOOTensor:
    """A HiCOO tensor held as numpy arrays (the fields of ptiSparseTensorHiCOO)."""

    def __init__(self, dims, sb, sk, sc, bptr, binds, einds, vals, kptr=None, cptr=None,
                 knnzs=None, nkiters=None, kschr_rows=None, max_nnzb=0, balanced=None):
        self.dims = [int(d) for d in dims]
        self.sb, self.sk, self.sc = int(sb), int(sk), int(sc)
        self.bptr = np.ascontiguousarray(bptr, np.uint64)
        self.binds = [np.ascontiguousarray(b, np.uint32) for b in binds]
        self.einds = [np.ascontiguousarray(e, np.uint8) for e in einds]
        self.vals = np.ascontiguousarray(vals, np.float32)
        self.kptr = None if kptr is None else np.ascontiguousarray(kptr, np.uint64)
        self.cptr = None if cptr is None else np.ascontiguousarray(cptr, np.uint64)
        self.knnzs = None if knnzs is None else np.ascontiguousarray(knnzs, np.uint64)
        self.nkiters = None if nkiters is None else np.ascontiguousarray(nkiters, np.uint32)
        self.kschr_rows = kschr_rows
        self.max_nnzb = max_nnzb
        self.balanced = balanced  # dict: rows, pos_rows, rest, nkpars (from the converter)
        self._build()

    @classmethod
    def _from_struct(cls, h, max_nnzb):
        N, nnz = h.nmodes, h.nnz
        nb = h.bptr.len - 1

        def arr(vec, n, dt):
            return np.frombuffer(ffi.buffer(vec.data, n * np.dtype(dt).itemsize), dt).copy() if n else np.empty(0, dt)
        dims = [h.ndims[m] for m in range(N)]
        rows, brows, prows, rest = [], [], [], []
        for m in range(N):
            for i in range((dims[m] + (1 << h.sk_bits) - 1) >> h.sk_bits):
                rows.append(arr(h.kschr[m][i], h.kschr[m][i].len, np.uint32))
                brows.append(arr(h.kschr_balanced[m][i], h.kschr_balanced[m][i].len, np.uint32))
                prows.append(arr(h.kschr_balanced_pos[m][i], h.kschr_balanced_pos[m][i].len, np.uint32))
            rest.append(arr(h.kschr_rest[m], h.kschr_rest[m].len, np.uint32))
        balanced = {"rows": brows, "pos_rows": prows, "rest": rest,
                    "nkpars": np.array([h.nkpars[m] for m in range(N)], np.uint32)}
        return cls(dims, h.sb_bits, h.sk_bits, h.sc_bits,
                   arr(h.bptr, nb + 1, np.uint64),
                   [arr(h.binds[m], nb, np.uint32) for m in range(N)],
                   [arr(h.einds[m], nnz, np.uint8) for m in range(N)],
                   arr(h.values, nnz, np.float32),
                   kptr=arr(h.kptr, h.kptr.len, np.uint64), cptr=arr(h.cptr, h.cptr.len, np.uint64),
                   knnzs=arr(h.knnzs, h.knnzs.len, np.uint64),
                   nkiters=np.array([h.nkiters[m] for m in range(N)], np.uint32),
                   kschr_rows=rows, max_nnzb=max_nnzb, balanced=balanced)

    def _build(self):
        N = len(self.dims)
        nb = self.bptr.size - 1
        nnz = self.vals.size
        self._dims = np.asarray(self.dims, np.uint32)
        self._so = np.arange(N, dtype=np.uint32)
        self._bv = ffi.new("ptiBlockIndexVector[]", N)
        self._ev = ffi.new("ptiElementIndexVector[]", N)
        for m in range(N):
            self._bv[m].len = self._bv[m].cap = nb
            self._bv[m].data = _ptr(self.binds[m], "ptiBlockIndex *")
            self._ev[m].len = self._ev[m].cap = nnz
            self._ev[m].data = _ptr(self.einds[m], "ptiElementIndex *")
        c = ffi.new("ptiSparseTensorHiCOO *")
        c.nmodes = N
        c.sortorder = _ptr(self._so, "ptiIndex *")
        c.ndims = _ptr(self._dims, "ptiIndex *")
        c.nnz = nnz
        c.sb_bits, c.sk_bits, c.sc_bits = self.sb, self.sk, self.sc
        c.bptr.len = c.bptr.cap = nb + 1
        c.bptr.data = _ptr(self.bptr, "ptiNnzIndex *")
        c.binds = self._bv
        c.einds = self._ev
        c.values.len = c.values.cap = nnz
        c.values.data = _ptr(self.vals, "ptiValue *")
        if self.kptr is not None:
            c.kptr.len = c.kptr.cap = self.kptr.size
            c.kptr.data = _ptr(self.kptr, "ptiNnzIndex *")
        self.c = c

    @property
    def nmodes(self):
        return len(self.dims)

    @property
    def nnz(self):
        return int(self.vals.size)

    @property
    def nb(self):
        return int(self.bptr.size - 1)

    def mttkrp(self, mats, R, mode, variant="seq"):
        """"seq" -> ptiMTTKRPHiCOO, "omp" -> ptiOmpMTTKRPHiCOO, "cuda" ->
        ptiCudaMTTKRPHiCOO; all on the GPU."""
        return _host_mttkrp(self, mats, R, mode, variant)


def _host_mttkrp(t, mats, R, mode, variant):
    N = t.nmodes
    mats = [np.ascontiguousarray(m, np.float32) for m in mats]
    stride = mats[0].shape[1]
    out = np.zeros((max(t.dims), stride), np.float32)
    ms = _MatrixSet(mats + [out], R)
    order = ffi.new("ptiIndex[]", [(mode + i) % N for i in range(N)])
    L = lib()
    if isinstance(t, COOTensor):
        fn = {"seq": lambda: L.ptiMTTKRP(t.c, ms.ptrs, order, mode),
              "omp": lambda: L.ptiOmpMTTKRP(t.c, ms.ptrs, order, mode, 8),
              "cuda": lambda: L.ptiCudaMTTKRP(t.c, ms.ptrs, order, mode, 5),
              "onekernel": lambda: L.ptiCudaMTTKRPOneKernel(t.c, ms.ptrs, order, mode, 15)}[variant]
    else:
        fn = {"seq": lambda: L.ptiMTTKRPHiCOO(t.c, ms.ptrs, order, mode),
              "omp": lambda: L.ptiOmpMTTKRPHiCOO(t.c, ms.ptrs, order, mode, 8, 1),
              "cuda": lambda: L.ptiCudaMTTKRPHiCOO(t.c, ms.ptrs, order, mode, 0, 1)}[variant]
    check(fn(), f"MTTKRP[{variant}]")
    return out[: t.dims[mode]].copy()


def _host_cpd(t, R, niters, tol, variant):
    L = lib()
    k = ffi.new("ptiKruskalTensor *")
    dims = ffi.new("ptiIndex[]", t.dims)
    check(L.ptiNewKruskalTensor(k, t.nmodes, dims, R), "ptiNewKruskalTensor")
    fn = {"seq": lambda: L.ptiCpdAls(t.c, R, niters, tol, k),
          "omp": lambda: L.ptiOmpCpdAls(t.c, R, niters, tol, 8, 0, k),
          "cuda": lambda: L.ptiCudaCpdAls(t.c, R, niters, tol, k)}[variant]
    try:
        check(fn(), f"CpdAls[{variant}]")
        lam = np.frombuffer(ffi.buffer(getattr(k, "lambda"), 4 * R), np.float32).copy()
        facs = []
        for m in range(t.nmodes):
            f = k.factors[m]
            a = np.frombuffer(ffi.buffer(f.values, 4 * f.nrows * f.stride), np.float32)
            facs.append(a.reshape(f.nrows, f.stride)[:, :R].copy())
        return dict(fit=k.fit, lambda_=lam, factors=facs)
    finally:
        L.ptiFreeKruskalTensor(k)


# ----------------------------------------------------------------------------
# Device-resident tensors (torch)
# ----------------------------------------------------------------------------
class DeviceTensor:
    """A tensor kept in GPU memory through the ptiB200 extension entry points."""

    def __init__(self, handle, dims):
        self._h = handle
        self.dims = list(dims)

    @classmethod
    def from_coo(cls, t: COOTensor) -> "DeviceTensor":
        hp = ffi.new("ptiB200Tensor **")
        check(lib().ptiB200UploadSparseTensor(hp, t.c), "ptiB200UploadSparseTensor")
        return cls(hp[0], t.dims)

    @classmethod
    def from_hicoo(cls, t: HiCOOTensor) -> "DeviceTensor":
        hp = ffi.new("ptiB200Tensor **")
        check(lib().ptiB200UploadSparseTensorHiCOO(hp, t.c), "ptiB200UploadSparseTensorHiCOO")
        return cls(hp[0], t.dims)

    @classmethod
    def load(cls, fname, start_index: int = 1, dedupe: bool = False) -> "DeviceTensor":
        """ptiB200LoadSparseTensor: a .tns/.bin file parsed on the GPU into a
        device COO tensor.  dedupe=True sorts by coordinate and sums the values
        of repeated coordinates (the reference keeps duplicates)."""
        hp = ffi.new("ptiB200Tensor **")
        check(lib().ptiB200LoadSparseTensor(hp, start_index, str(fname).encode(), int(bool(dedupe)), ffi.NULL),
              "ptiB200LoadSparseTensor")
        info = ffi.new("ptiNnzIndex[7]")
        dims = ffi.new("ptiIndex[8]")
        check(lib().ptiB200TensorInfo(hp[0], info, dims), "ptiB200TensorInfo")
        return cls(hp[0], [dims[m] for m in range(info[0])])

    def coo_arrays(self):
        """(inds, vals) of a device COO tensor as numpy arrays (ptiB200DownloadCOO)."""
        info = ffi.new("ptiNnzIndex[7]")
        dims = ffi.new("ptiIndex[8]")
        check(lib().ptiB200TensorInfo(self._h, info, dims), "ptiB200TensorInfo")
        N, nnz = int(info[0]), int(info[1])
        inds = [np.empty(nnz, np.uint32) for _ in range(N)]
        vals = np.empty(nnz, np.float32)
        ip = ffi.new("ptiIndex *[]", [ffi.cast("ptiIndex *", a.ctypes.data) for a in inds])
        check(lib().ptiB200DownloadCOO(self._h, ip, ffi.cast("ptiValue *", vals.ctypes.data)), "ptiB200DownloadCOO")
        return inds, vals

    @classmethod
    def from_torch_coo(cls, dims, inds, vals) -> "DeviceTensor":
        """inds: list of int32/uint32-valued CUDA tensors (nnz,), vals: float32 (nnz,)."""
        import torch
        N = len(dims)
        inds = [i.contiguous() for i in inds]
        vals = vals.contiguous().to(torch.float32)
        ip = ffi.new("ptiIndex *[]", [ffi.cast("ptiIndex *", i.data_ptr()) for i in inds])
        d = ffi.new("ptiIndex[]", [int(x) for x in dims])
        hp = ffi.new("ptiB200Tensor **")
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200TensorFromDeviceCOO(hp, N, d, vals.numel(), ip,
                                               ffi.cast("ptiValue *", vals.data_ptr()), stream),
              "ptiB200TensorFromDeviceCOO")
        return cls(hp[0], dims)

    def to_hicoo(self, sb=7, sk=10, sc=14) -> "DeviceTensor":
        import torch
        hp = ffi.new("ptiB200Tensor **")
        nb = ffi.new("ptiNnzIndex *")
        mx = ffi.new("ptiNnzIndex *")
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200ConvertToHiCOO(hp, self._h, sb, sk, sc, nb, mx, stream), "ptiB200ConvertToHiCOO")
        out = DeviceTensor(hp[0], self.dims)
        out.nb, out.max_nnzb = int(nb[0]), int(mx[0])
        return out

    def info(self):
        info = ffi.new("ptiNnzIndex[7]")
        check(lib().ptiB200TensorInfo(self._h, info, ffi.NULL), "ptiB200TensorInfo")
        keys = ["nmodes", "nnz", "nb", "sb", "sk", "sc", "hicoo"]
        return {k: int(info[i]) for i, k in enumerate(keys)}

    def prepare(self, mode=None):
        import torch
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        modes = range(len(self.dims)) if mode is None else [mode]
        for m in modes:
            check(lib().ptiB200Prepare(self._h, m, stream), "ptiB200Prepare")

    def check(self):
        """Waits for the current stream and raises if this tensor's kernels
        recorded a device error (ptiB200CheckTensor)."""
        import torch
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200CheckTensor(self._h, stream), "ptiB200CheckTensor")

    def mttkrp(self, factors, mode, rank=None, out=None, mats_order=None):
        """factors: list of CUDA tensors (I_k, stride), float32 or bfloat16, all
        of one dtype; returns / fills a float32 (I_mode, stride) tensor."""
        import torch
        N = len(self.dims)
        ft = factors[0].dtype
        if ft not in (torch.float32, torch.bfloat16) or any(f.dtype != ft for f in factors):
            raise TypeError("factors must all be float32 or all bfloat16")
        stride = factors[0].shape[1]
        R = stride if rank is None else int(rank)
        if out is None:
            out = torch.empty((self.dims[mode], stride), dtype=torch.float32, device=factors[0].device)
        if mats_order is None:
            mats_order = [(mode + i) % N for i in range(N)]
        mp = ffi.new("void *[]", [ffi.cast("void *", f.data_ptr()) for f in factors])
        order = ffi.new("ptiIndex[]", list(mats_order))
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200MTTKRP(self._h, mp, _F32 if ft == torch.float32 else _BF16, R, stride, order,
                                  mode, ffi.cast("float *", out.data_ptr()), stream), "ptiB200MTTKRP")
        return out

    def kruskal_values(self, factors, rank=None, out=None):
        """The CP model sum_r prod_k A_k[i_k, r] at every nonzero (input order)."""
        import torch
        stride = factors[0].shape[1]
        R = stride if rank is None else int(rank)
        if out is None:
            out = torch.empty(self.info()["nnz"], dtype=torch.float32, device=factors[0].device)
        fp = ffi.new("float *[]", [ffi.cast("float *", f.data_ptr()) for f in factors])
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200KruskalValues(self._h, fp, R, stride, ffi.cast("float *", out.data_ptr()), stream),
              "ptiB200KruskalValues")
        return out

    def mttkrp_values(self, vals, factors, mode, rank=None, out=None):
        """MTTKRP with the nonzero values replaced by `vals` (float32, input order)."""
        import torch
        N = len(self.dims)
        stride = factors[0].shape[1]
        R = stride if rank is None else int(rank)
        if out is None:
            out = torch.empty((self.dims[mode], stride), dtype=torch.float32, device=factors[0].device)
        vals = vals.contiguous().to(torch.float32)
        mp = ffi.new("void *[]", [ffi.cast("void *", f.data_ptr()) for f in factors])
        order = ffi.new("ptiIndex[]", [(mode + i) % N for i in range(N)])
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        check(lib().ptiB200MTTKRPValues(self._h, ffi.cast("float *", vals.data_ptr()), mp, _F32, R, stride, order,
                                        mode, ffi.cast("float *", out.data_ptr()), stream), "ptiB200MTTKRPValues")
        return out

    def cpd_als(self, factors, niters, tol=0.0, precision="fp32", fp32_sweeps=1, rank=None,
                checkpoint=None, checkpoint_every=0, resume=False):
        """CPD-ALS on the device (ptiB200CpdAls).  factors: list of float32 CUDA
        tensors (I_k, stride) holding the initial factors; updated in place.
        precision "bf16" makes the MTTKRP gathers read BF16 copies for all but
        the last fp32_sweeps iterations.  checkpoint: a file that receives the
        loop state after every checkpoint_every iterations (0: only the last);
        resume=True continues from it when it exists
        (ptiB200CpdAlsCheckpoint).  Returns (lambda, fits), fits counting the
        restored iterations too."""
        import torch
        stride = factors[0].shape[1]
        R = stride if rank is None else int(rank)
        lam = torch.empty(R, dtype=torch.float32, device=factors[0].device)
        fits = ffi.new("double[]", max(int(niters), 1))
        done = ffi.new("ptiIndex *")
        fp = ffi.new("float *[]", [ffi.cast("float *", f.data_ptr()) for f in factors])
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        prec = {"fp32": _F32, "bf16": _BF16}[precision]
        path = ffi.NULL if checkpoint is None else str(checkpoint).encode()
        check(lib().ptiB200CpdAlsCheckpoint(self._h, R, niters, tol, prec, fp32_sweeps, fp, stride,
                                            ffi.cast("float *", lam.data_ptr()), fits, done, path,
                                            int(checkpoint_every), int(bool(resume)), stream),
              "ptiB200CpdAlsCheckpoint")
        return lam, [fits[i] for i in range(done[0])]

    def ttm(self, U, mode, rank=None):
        """TTM along `mode` on the device (ptiB200TTM).  U: CUDA float32
        (ndims[mode], ldu); rank columns used (default all; 0 = TTV with U's
        first column read as a vector, ldu 1).  Returns
        (fiber coordinates per mode as CUDA int32 tensors, the mode's own
        None; Y as a (nfibers, ldy) CUDA float32 tensor, ldy = rank rounded up
        to 8)."""
        import torch
        stream = ffi.cast("void *", torch.cuda.current_stream().cuda_stream)
        R = U.shape[1] if rank is None else int(rank)
        ldy = ((max(R, 1) - 1) // 8 + 1) * 8  # rank 0 (TTV): one column
        nf = ffi.new("ptiNnzIndex *")
        N = len(self.dims)
        check(lib().ptiB200TTMFibers(self._h, mode, nf, ffi.NULL, stream), "ptiB200TTMFibers")
        finds = [None if m == mode else torch.empty(int(nf[0]), dtype=torch.int32, device=U.device)
                 for m in range(N)]
        fp = ffi.new("ptiIndex *[]", [ffi.NULL if f is None else ffi.cast("ptiIndex *", f.data_ptr())
                                      for f in finds])
        check(lib().ptiB200TTMFibers(self._h, mode, nf, fp, stream), "ptiB200TTMFibers")
        Y = torch.empty((int(nf[0]), ldy), dtype=torch.float32, device=U.device)
        check(lib().ptiB200TTM(self._h, mode, ffi.cast("float *", U.data_ptr()), R, U.shape[1],
                               ffi.cast("float *", Y.data_ptr()), ldy, stream), "ptiB200TTM")
        return finds, Y

    def renumber(self, iterations=1, apply=True):
        """Lexi-order renumbering on the GPU (ptiB200Renumber): per mode,
        original index -> new index; apply=True renumbers this tensor's
        coordinates in place."""
        maps = [np.empty(d, np.uint32) for d in self.dims]
        mp = ffi.new("ptiIndex *[]", [ffi.cast("ptiIndex *", m.ctypes.data) for m in maps])
        check(lib().ptiB200Renumber(self._h, int(iterations), mp, int(bool(apply)), ffi.NULL), "ptiB200Renumber")
        return maps

    def free(self):
        if self._h is not None:
            lib().ptiB200FreeTensor(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ----------------------------------------------------------------------------
# CPD results on the host: checkpoints and the reference's text dump
# ----------------------------------------------------------------------------
def load_cpd_checkpoint(path):
    """Reads a CPD checkpoint (ptiB200LoadCpdCheckpoint): the result the ALS
    loop returns after the stored iterations.  Returns a dict with iters, fit,
    lambda_ (R,) and factors (list of (I_k, R) float32 arrays)."""
    k = ffi.new("ptiKruskalTensor *")
    it = ffi.new("ptiIndex *")
    check(lib().ptiB200LoadCpdCheckpoint(k, it, str(path).encode()), "ptiB200LoadCpdCheckpoint")
    try:
        R = k.rank
        lam = np.frombuffer(ffi.buffer(getattr(k, "lambda"), 4 * R), np.float32).copy()
        facs = []
        for m in range(k.nmodes):
            f = k.factors[m]
            a = np.frombuffer(ffi.buffer(f.values, 4 * f.nrows * f.stride), np.float32)
            facs.append(a.reshape(f.nrows, f.stride)[:, :R].copy())
        return dict(iters=int(it[0]), fit=float(k.fit), lambda_=lam, factors=facs)
    finally:
        lib().ptiFreeKruskalTensor(k)


def dump_kruskal(path, lambda_, factors, fit=0.0):
    """Writes a Kruskal tensor as text in the reference's format
    (ptiDumpKruskalTensor, src/ktensor/dump.c:23-55)."""
    lam = np.ascontiguousarray(lambda_, np.float32)
    facs = [np.ascontiguousarray(f, np.float32) for f in factors]
    R, N = lam.size, len(facs)
    dims = ffi.new("ptiIndex[]", [f.shape[0] for f in facs])
    k = ffi.new("ptiKruskalTensor *")
    L = lib()
    check(L.ptiNewKruskalTensor(k, N, dims, R), "ptiNewKruskalTensor")
    mats = ffi.new("ptiMatrix *[]", N + 1)
    structs = [ffi.new("ptiMatrix *") for _ in range(N)]
    try:
        for m, f in enumerate(facs):
            check(L.ptiNewMatrix(structs[m], f.shape[0], R), "ptiNewMatrix")
            st = structs[m].stride
            buf = np.frombuffer(ffi.buffer(structs[m].values, 4 * f.shape[0] * st), np.float32)
            buf.reshape(f.shape[0], st)[:, :R] = f[:, :R]
            mats[m] = structs[m]
        ffi.memmove(getattr(k, "lambda"), lam.tobytes(), 4 * R)
        k.fit = float(fit)
        k.factors = mats
        with open(path, "wb") as fh:
            check(L.ptiDumpKruskalTensor(k, fh), "ptiDumpKruskalTensor")
    finally:
        k.factors = ffi.NULL
        for sm in structs:
            if sm.values != ffi.NULL:
                L.ptiFreeMatrix(sm)
        L.ptiFreeKruskalTensor(k)
