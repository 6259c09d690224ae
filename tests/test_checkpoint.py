"""CPU tests of the CPD result files: the text dump against the reference
library's own ptiDumpKruskalTensor / ptiDumpRankKruskalTensor (byte for byte),
and the checkpoint reader against files written here by a restatement of the
checkpoint layout (header, sizes, fits, weights, factors, FNV-1a word sum)."""
import ctypes as C
import struct

import numpy as np
import pytest

from hiparti_b200 import PtiError, dump_kruskal, ffi, lib, load_cpd_checkpoint


# ---------------------------------------------------------------------------
# Text dumps
# ---------------------------------------------------------------------------
class _RefMatrix(C.Structure):
    _fields_ = [("nrows", C.c_uint32), ("ncols", C.c_uint32), ("cap", C.c_uint32), ("stride", C.c_uint32),
                ("values", C.c_void_p)]


class _RefRankMatrix(C.Structure):
    _fields_ = [("nrows", C.c_uint32), ("ncols", C.c_uint8), ("cap", C.c_uint32), ("stride", C.c_uint8),
                ("values", C.c_void_p)]


def _kruskal_struct(mat_t, rank_t):
    class K(C.Structure):
        _fields_ = [("nmodes", C.c_uint32), ("rank", rank_t), ("ndims", C.c_void_p), ("lambda_", C.c_void_p),
                    ("fit", C.c_double), ("factors", C.POINTER(C.POINTER(mat_t)))]
    return K


def _ref_dump(ref, tmp_path, lam, facs, fit, rank_kind):
    """Dumps through the reference library with the same contents."""
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    R = lam.size
    stride = ((R - 1) // 8 + 1) * 8
    mat_t = _RefRankMatrix if rank_kind else _RefMatrix
    K = _kruskal_struct(mat_t, C.c_uint8 if rank_kind else C.c_uint32)
    keep = []
    mats = []
    for f in facs:
        buf = np.zeros((f.shape[0], stride), np.float32)
        buf[:, :R] = f
        keep.append(buf)
        mats.append(mat_t(f.shape[0], R, f.shape[0], stride, buf.ctypes.data))
    arr = (C.POINTER(mat_t) * (len(facs) + 1))(*[C.pointer(m) for m in mats], None)
    dims = np.array([f.shape[0] for f in facs], np.uint32)
    lam32 = np.ascontiguousarray(lam, np.float32)
    k = K(len(facs), R, dims.ctypes.data, lam32.ctypes.data, fit, arr)
    path = tmp_path / ("ref_rank.txt" if rank_kind else "ref.txt")
    fp = libc.fopen(str(path).encode(), b"w")
    fn = ref.L.ptiDumpRankKruskalTensor if rank_kind else ref.L.ptiDumpKruskalTensor
    assert fn(C.byref(k), C.c_void_p(fp)) == 0
    libc.fclose(fp)
    return path.read_bytes()


def _sample(seed, dims, R):
    rng = np.random.default_rng(seed)
    lam = (rng.standard_normal(R) * 100).astype(np.float32)
    facs = [(rng.standard_normal((d, R)) * 10.0 ** rng.integers(-3, 4)).astype(np.float32) for d in dims]
    return lam, facs


@pytest.mark.parametrize("dims,R", [((4, 3, 5), 3), ((2, 6, 3, 4), 9), ((7, 1, 2), 16)])
def test_kruskal_dump_matches_reference(ref, tmp_path, dims, R):
    lam, facs = _sample(R, dims, R)
    fit = 0.123456789
    ours = tmp_path / "ours.txt"
    dump_kruskal(ours, lam, facs, fit)
    assert ours.read_bytes() == _ref_dump(ref, tmp_path, lam, facs, fit, rank_kind=False)


def test_rank_kruskal_dump_matches_reference(ref, tmp_path):
    """ptiDumpRankKruskalTensor (8-bit rank and stride) through both libraries."""
    dims, R = (5, 4, 3), 10
    lam, facs = _sample(7, dims, R)
    L = lib()
    k = ffi.new("ptiRankKruskalTensor *")
    cd = ffi.new("ptiIndex[]", list(dims))
    assert L.ptiNewRankKruskalTensor(k, 3, cd, R) == 0
    mats = ffi.new("ptiRankMatrix *[]", 4)
    structs = [ffi.new("ptiRankMatrix *") for _ in dims]
    for m, f in enumerate(facs):
        assert L.ptiNewRankMatrix(structs[m], f.shape[0], R) == 0
        st = structs[m].stride
        np.frombuffer(ffi.buffer(structs[m].values, 4 * f.shape[0] * st), np.float32).reshape(-1, st)[:, :R] = f
        mats[m] = structs[m]
    ffi.memmove(getattr(k, "lambda"), lam.tobytes(), 4 * R)
    k.fit = 0.75
    k.factors = mats
    ours = tmp_path / "ours_rank.txt"
    with open(ours, "wb") as fh:
        assert L.ptiDumpRankKruskalTensor(k, fh) == 0
    k.factors = ffi.NULL
    for s in structs:
        L.ptiFreeRankMatrix(s)
    L.ptiFreeRankKruskalTensor(k)
    assert ours.read_bytes() == _ref_dump(ref, tmp_path, lam, facs, 0.75, rank_kind=True)


# ---------------------------------------------------------------------------
# Checkpoint files
# ---------------------------------------------------------------------------
def _fnv_words(data: bytes) -> int:
    h = 0xcbf29ce484222325
    for (w,) in struct.iter_unpack("<Q", data):
        h = ((h ^ w) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    return h


def write_checkpoint(path, dims, nnz, normX2, fits, lam, facs, converged=False):
    """The checkpoint layout, restated: 48-byte header, sizes padded to 8
    bytes, fits, weights and factors (padded to 8 bytes), FNV-1a word sum."""
    R = lam.size
    head = b"PTICPDCK" + struct.pack("<6I", 1, len(dims), R, len(fits), 1 if converged else 0, 0)
    head += struct.pack("<Qd", nnz, normX2)
    nd = list(dims) + [0] * (len(dims) % 2)
    body = struct.pack(f"<{len(nd)}I", *nd) + np.asarray(fits, np.float64).tobytes()
    vals = np.asarray(lam, np.float32).tobytes() + b"".join(np.ascontiguousarray(f, np.float32).tobytes()
                                                            for f in facs)
    vals += b"\0" * (-len(vals) % 8)
    data = head + body + vals
    path.write_bytes(data + struct.pack("<Q", _fnv_words(data)))


def _finished(lam, facs):
    """The loop's closing step: unit 2-norm columns, weights times the norms."""
    lam = lam.astype(np.float32).copy()
    out = []
    for f in facs:
        norm = np.sqrt((f.astype(np.float64) ** 2).sum(0))
        out.append((f / norm.astype(np.float32)).astype(np.float32))
        lam *= norm.astype(np.float32)
    return lam, out


@pytest.mark.parametrize("dims,R,iters", [((5, 4, 3), 3, 7), ((6, 2, 3, 5), 5, 0), ((9, 8, 7), 8, 1)])
def test_checkpoint_reader(tmp_path, dims, R, iters):
    rng = np.random.default_rng(R)
    lam = rng.uniform(1, 3, R).astype(np.float32)
    facs = [rng.standard_normal((d, R)).astype(np.float32) for d in dims]
    fits = np.linspace(0.1, 0.9, iters)
    p = tmp_path / "c.ckpt"
    write_checkpoint(p, dims, 1234, 56.5, fits, lam, facs)
    got = load_cpd_checkpoint(p)
    want_lam, want_facs = _finished(lam, facs)
    assert got["iters"] == iters
    assert got["fit"] == (fits[-1] if iters else 0.0)
    np.testing.assert_allclose(got["lambda_"], want_lam, rtol=1e-6)
    for a, b in zip(got["factors"], want_facs):
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-7)


def test_checkpoint_reader_rejects_damage(tmp_path):
    rng = np.random.default_rng(0)
    dims, R = (5, 4, 3), 3
    facs = [rng.standard_normal((d, R)).astype(np.float32) for d in dims]
    p = tmp_path / "c.ckpt"
    write_checkpoint(p, dims, 10, 1.0, [0.5, 0.6], np.ones(R, np.float32), facs)
    good = p.read_bytes()
    load_cpd_checkpoint(p)
    bad = bytearray(good)
    bad[100] ^= 1  # a factor value
    p.write_bytes(bytes(bad))
    with pytest.raises(PtiError, match="checksum"):
        load_cpd_checkpoint(p)
    p.write_bytes(good[:-16])
    with pytest.raises(PtiError):
        load_cpd_checkpoint(p)
    p.write_bytes(b"NOTACKPT" + good[8:])
    with pytest.raises(PtiError, match="not a CPD checkpoint"):
        load_cpd_checkpoint(p)
    with pytest.raises(PtiError):
        load_cpd_checkpoint(tmp_path / "missing.ckpt")
