"""GPU parity of the tensor loader (ptiLoadSparseTensor, ptiB200LoadSparseTensor)
against the reference's own loader, src/sptensor/load.c, compiled from its
sources (fscanf "%u" / "%lf" on the host).  Bit-exact: indices, values (as
FP32 bit patterns, NaNs included), the nonzero count where reading stops, and
whether the load fails."""
import struct
from decimal import Decimal, getcontext

import numpy as np
import pytest

from hiparti_b200 import COOTensor, DeviceTensor, PtiError

pytestmark = pytest.mark.gpu


def _ours(path, start_index=1):
    try:
        t = COOTensor.load(str(path), start_index)
    except PtiError:
        return None
    return t.dims, t.inds, t.vals


def _theirs(ref, path, start_index=1):
    rc, dims, inds, vals = ref.load(path, start_index)
    if rc != 0:
        return None
    return [int(d) for d in dims], inds, vals


def _same(a, b):
    if a is None or b is None:
        return a is None and b is None
    (da, ia, va), (db, ib, vb) = a, b
    return (da == db and len(ia) == len(ib) and all(np.array_equal(x, y) for x, y in zip(ia, ib))
            and np.array_equal(va.view(np.uint32), vb.view(np.uint32)))


EDGE = {
    "plain": "3\n4 5 6\n1 1 1 1.5\n2 2 2 2.0\n",
    "bad_index": "3\n4 5 6\n1 1 1 1.5\n2 2 x 2.0\n3 3 3 3.0\n",
    "value_prefix": "3\n4 5 6\n1 1 1 1.5x\n2 2 2 2.0\n",
    "bare_exponent": "3\n4 5 6\n1 1 1 1e\n2 2 2 2.5e+\n3 3 3 7E-\n",
    "index_prefix": "3\n4 5 6\n1 1 12abc 2.0\n",
    "incomplete": "3\n4 5 6\n1 1 1 1.5\n2 2 2\n",
    "comment": "3\n4 5 6\n# a comment\n1 1 1 1.5\n",
    "negative_index": "3\n4 5 6\n-1 1 1 1.5\n-7 2 2 2\n",
    "wide_index": "3\n4 5 6\n99999999999 1 1 1.5\n99999999999999999999999 2 2 2.5\n",
    "below_start": "3\n4 5 6\n1 1 1 1.0\n0 1 1 1.5\n",
    "below_start_after_stop": "3\n4 5 6\n1 1 1 x\n0 1 1 1.0\n",
    "specials": "3\n4 5 6\n1 1 1 inf\n1 1 2 -Infinity\n1 1 3 nan\n1 1 4 -NaN\n1 1 5 +INF\n",
    "partial_infinity": "3\n4 5 6\n1 1 1 2\n1 1 2 infinit\n",
    "inf_suffix": "3\n4 5 6\n1 1 1 infx\n1 1 2 3\n",
    "lone_dot": "3\n4 5 6\n1 1 1 .\n",
    "dots": "3\n4 5 6\n1 1 1 .5\n1 1 2 5.\n1 1 3 +.5e1\n1 1 4 -0\n1 1 5 -0.0e-7\n",
    "two_dots": "3\n4 5 6\n1 1 1 1.2.3\n",
    "glued_header": "3\n4 5 6x\n1 1 1 1\n",
    "bad_header": "3\n4 x 6\n1 1 1 1\n",
    "empty": "3\n4 5 6\n",
    "no_newline": "3\n4 5 6\n1 1 1 1.5\n2 2 2 2.25",
    "crlf_tabs": "3\r\n4\t5\t6\r\n\r\n  1 1\t1   1.5\r\n2 2 2\v2.0\f\n",
    "one_line": "2 3 4 1 1 0.5 2 3 0.25 3 4 -1",
    "four_modes": "4\n2 3 4 5\n1 2 3 4 0.1\n2 3 4 5 0.2\n",
    "leading_zeros": "3\n4 5 6\n001 0002 1 000.0000125\n",
}


@pytest.mark.parametrize("name", sorted(EDGE))
@pytest.mark.parametrize("start_index", [0, 1])
def test_edge_cases_match_reference(lib, cuda, ref, tmp_path, name, start_index):
    p = tmp_path / f"{name}.tns"
    p.write_bytes(EDGE[name].encode())
    assert _same(_ours(p, start_index), _theirs(ref, p, start_index)), name


@pytest.mark.parametrize("text,why", [("3\n4 5 6\n1 1 1 0x1p3\n", "hexadecimal"),
                                      ("3\n4 5 6\n1 1 1 nan(12)\n", "nan")])
def test_refused_values(lib, cuda, tmp_path, text, why):
    p = tmp_path / "r.tns"
    p.write_text(text)
    with pytest.raises(PtiError, match=why):
        COOTensor.load(str(p))


def _near_midpoints(rng, n):
    """Decimals just above or below FP32 rounding midpoints, close enough that
    FP64 rounds them onto the midpoint: FP32 must then see the tie (round half
    to even), not the decimal.  Also exact midpoints."""
    getcontext().prec = 60
    out = []
    for _ in range(n):
        f = np.float32(rng.uniform(-1e6, 1e6) * 10.0 ** rng.integers(-30, 30))
        g = np.nextafter(f, np.float32(np.inf))
        mid = (Decimal(float(f)) + Decimal(float(g))) / 2
        ulp = Decimal(float(np.spacing(float(mid))))
        for d in (mid, mid + ulp / 4, mid - ulp / 4, mid + ulp * Decimal("0.6")):
            out.append(format(d, ".40e"))
    return out


def _value_strings(rng, n):
    kinds = [
        lambda: f"{rng.uniform(-1, 1):.6f}",
        lambda: f"{rng.lognormal(0, 3):.9g}",
        lambda: f"{rng.standard_normal():.17g}",
        lambda: f"{rng.standard_normal() * 1e5:.25g}",
        lambda: f"{rng.uniform(1, 10) * 10.0 ** rng.integers(-60, 45):e}",
        lambda: f"{rng.uniform(1, 10) * 10.0 ** rng.integers(-320, 308):.3e}",
        lambda: str(int(rng.integers(-10**6, 10**6))),
        lambda: f"{rng.uniform(0, 1):.30f}",
        lambda: f"{rng.standard_normal():.8E}",
    ]
    return [kinds[int(rng.integers(len(kinds)))]() for _ in range(n)]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_value_formats_match_reference(lib, cuda, ref, tmp_path, seed):
    rng = np.random.default_rng(seed)
    dims = (50, 40, 30)
    vals = _value_strings(rng, 20000) + _near_midpoints(rng, 500)
    n = len(vals)
    idx = [rng.integers(1, d + 1, n) for d in dims]
    seps = [" ", "\t", "  "]
    lines = [f"{i}{seps[k % 3]}{j} {l} {v}" for k, (i, j, l, v) in enumerate(zip(*idx, vals))]
    p = tmp_path / "rand.tns"
    p.write_text("3\n" + " ".join(map(str, dims)) + "\n" + "\n".join(lines) + "\n")
    ours, theirs = _ours(p), _theirs(ref, p)
    assert theirs is not None and theirs[1][0].size == n
    assert _same(ours, theirs)


def test_large_file_matches_reference(lib, cuda, ref, tmp_path):
    """Two million nonzeros (about 60 MB of text, many 16 KB parse chunks)."""
    rng = np.random.default_rng(7)
    dims = (100000, 80000, 3000)
    n = 2_000_000
    cols = [rng.integers(1, d + 1, n) for d in dims]
    v = rng.standard_normal(n)
    body = np.char.add(np.char.add(np.char.add(np.char.add(cols[0].astype(str), " "),
                                               np.char.add(cols[1].astype(str), " ")),
                                   np.char.add(cols[2].astype(str), " ")),
                       np.char.mod("%.7g", v))
    p = tmp_path / "big.tns"
    with open(p, "w") as f:
        f.write("3\n100000 80000 3000\n")
        f.write("\n".join(body.tolist()))
        f.write("\n")
    ours, theirs = _ours(p), _theirs(ref, p)
    assert theirs[1][0].size == n
    assert _same(ours, theirs)


def _write_bin(path, dims, inds, vals, vw):
    with open(path, "wb") as f:
        f.write(struct.pack("<iQQ", 0, 4, vw))
        f.write(struct.pack("<I", len(dims)) + struct.pack(f"<{len(dims)}I", *dims) +
                struct.pack("<I", vals.size))
        for i in inds:
            f.write(np.asarray(i, np.uint32).tobytes())
        with np.errstate(over="ignore"):  # values beyond FP32 become infinities on purpose
            f.write(np.asarray(vals, np.float32 if vw == 4 else np.float64).tobytes())


@pytest.mark.parametrize("vw", [4, 8])
def test_binary_matches_reference(lib, cuda, ref, tmp_path, vw):
    rng = np.random.default_rng(vw)
    dims = (70, 60, 50, 40)
    n = 33333
    inds = [rng.integers(0, d, n) for d in dims]
    vals = rng.standard_normal(n) * 10.0 ** rng.integers(-40, 40, n)
    p = tmp_path / "t.bin"
    _write_bin(p, dims, inds, vals, vw)
    assert _same(_ours(p), _theirs(ref, p))


def test_device_load_and_dedupe(lib, cuda, ref, tmp_path):
    rng = np.random.default_rng(3)
    dims = (20, 15, 10)
    n = 5000  # many repeated coordinates
    idx = [rng.integers(1, d + 1, n) for d in dims]
    vals = rng.standard_normal(n).astype(np.float32)
    p = tmp_path / "dup.tns"
    p.write_text("3\n20 15 10\n" + "\n".join(f"{a} {b} {c} {v!r}" for a, b, c, v in zip(*idx, vals.tolist())))
    # without dedupe: the file's nonzeros in file order, as the reference loads them
    t = DeviceTensor.load(p)
    inds, v = t.coo_arrays()
    t.free()
    _, rinds, rvals = _theirs(ref, p)
    assert all(np.array_equal(a, b) for a, b in zip(inds, rinds))
    assert np.array_equal(v.view(np.uint32), rvals.view(np.uint32))
    # with dedupe: sorted by coordinate (mode 0 first), FP32 sums in file order
    t = DeviceTensor.load(p, dedupe=True)
    dinds, dv = t.coo_arrays()
    t.free()
    keys = {}
    for k in range(n):
        c = (int(rinds[0][k]), int(rinds[1][k]), int(rinds[2][k]))
        keys[c] = np.float32(keys[c] + rvals[k]) if c in keys else rvals[k]
    order = sorted(keys)
    assert [tuple(int(a[k]) for a in dinds) for k in range(len(order))] == order
    assert dinds[0].size == len(order)
    want = np.array([keys[c] for c in order], np.float32)
    assert np.array_equal(dv.view(np.uint32), want.view(np.uint32))


def test_device_load_rejects_out_of_range_indices(lib, cuda, tmp_path):
    p = tmp_path / "oor.tns"
    p.write_text("3\n4 5 6\n1 1 1 1.0\n5 1 1 2.0\n")
    assert COOTensor.load(str(p)).nnz == 2  # the reference loader does not check
    with pytest.raises(PtiError):
        DeviceTensor.load(p)


def test_load_tns_and_bin(lib, tmp_path):
    p = tmp_path / "t.tns"
    p.write_text("3\n4 5 6\n1 1 1 1.5\n4 5 6 -2.0\n2 3 1 0.25\n")
    t = COOTensor.load(str(p))
    assert t.dims == [4, 5, 6] and t.nnz == 3
    np.testing.assert_array_equal(t.inds[0], [0, 3, 1])
    np.testing.assert_array_equal(t.inds[2], [0, 5, 0])
    np.testing.assert_array_equal(t.vals, np.float32([1.5, -2.0, 0.25]))
    # SPLATT binary: header, nmodes, dims, nnz, indices per mode, values
    b = tmp_path / "t.bin"
    with open(b, "wb") as f:
        f.write(struct.pack("<iQQ", 0, 4, 4))
        f.write(struct.pack("<I", 3) + struct.pack("<3I", 4, 5, 6) + struct.pack("<I", 2))
        f.write(struct.pack("<2I", 0, 3) + struct.pack("<2I", 1, 4) + struct.pack("<2I", 5, 0))
        f.write(struct.pack("<2f", 1.0, 2.0))
    tb = COOTensor.load(str(b))
    assert tb.dims == [4, 5, 6]
    np.testing.assert_array_equal(tb.inds[1], [1, 4])
    np.testing.assert_array_equal(tb.vals, np.float32([1, 2]))
