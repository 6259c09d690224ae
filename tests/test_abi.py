"""CPU: the C-ABI library loads, exports every entry point the header declares,
lays out the reference's structs byte for byte, and runs its host-side logic
(containers, argument checks) without a GPU."""
import re
import struct

import numpy as np
import pytest

from conftest import ROOT
from hiparti_b200 import COOTensor, HiCOOTensor, PtiError, ffi, synth

HEADER = ROOT / "include" / "hiparti_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"^\s*(?:int|void|double)\s+\**\s*(\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib):
    import subprocess
    so = ROOT / "hiparti_b200" / "libhiparti_b200.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)  # cffi resolves each declared symbol


def test_dropin_caller_links_against_this_library_alone(lib):
    """The C caller built against the reference's own header
    (tests/dropin/dropin_main.c) needs no symbol this library does not
    export: every reference entry point it calls resolves here."""
    import subprocess
    binary = ROOT / "tests" / "dropin" / "_build" / "dropin"
    if not binary.exists():
        pytest.skip("drop-in caller not built (needs the reference's header)")
    so = ROOT / "hiparti_b200" / "libhiparti_b200.so"
    exported = {ln.split()[-1] for ln in subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True,
                                                         text=True).stdout.splitlines() if " T " in ln}
    undefined = {ln.split()[-1] for ln in subprocess.run(["nm", "-D", "--undefined-only", str(binary)],
                                                          capture_output=True, text=True).stdout.splitlines()}
    ours = {n for n in undefined if re.match(r"(pti|Kruskal|Sparse|Cpd|GetFinal|GetRank)", n)}
    assert len(ours) >= 15, sorted(ours)
    assert ours <= exported, sorted(ours - exported)
    ldd = subprocess.run(["ldd", str(binary)], capture_output=True, text=True).stdout
    assert "libhiparti_b200.so" in ldd and "not found" not in ldd and "libHiParTI" not in ldd


def test_struct_layout_matches_reference():
    # sizes/offsets of include/includes/structs.h compiled with the reference
    # headers on x86-64 (gcc): see the reference struct definitions.
    assert ffi.sizeof("ptiSparseTensorHiCOO") == 224
    assert ffi.sizeof("ptiSparseTensor") == 64
    assert ffi.sizeof("ptiMatrix") == 24
    assert ffi.sizeof("ptiRankMatrix") == 24
    assert ffi.sizeof("ptiKruskalTensor") == 40
    assert ffi.sizeof("ptiRankKruskalTensor") == 40
    off = {"sb_bits": 32, "kptr": 40, "kschr": 64, "cptr": 80, "knnzs": 136, "bptr": 160,
           "binds": 184, "einds": 192, "values": 200}
    for f, o in off.items():
        assert ffi.offsetof("ptiSparseTensorHiCOO", f) == o, f
    assert ffi.offsetof("ptiRankMatrix", "stride") == 12
    assert ffi.offsetof("ptiKruskalTensor", "fit") == 24
    assert ffi.offsetof("ptiSparseTensor", "values") == 40


def test_matrix_life_cycle(lib):
    m = ffi.new("ptiMatrix *")
    assert lib.ptiNewMatrix(m, 5, 11) == 0
    assert (m.nrows, m.ncols, m.cap, m.stride) == (5, 11, 5, 16)
    assert int(ffi.cast("uintptr_t", m.values)) % 32 == 0
    assert lib.ptiRandomizeMatrix(m) == 0
    assert m.values[2 * 16 + 3] == 6.0  # i + j + 1
    assert lib.ptiConstantMatrix(m, 2.5) == 0
    assert m.values[4 * 16 + 10] == 2.5
    lib.ptiFreeMatrix(m)


def test_shape_mismatch_is_reported_before_any_gpu_work(lib):
    dims = (5, 6, 7)
    coo = COOTensor(dims, [np.array([1], np.uint32)] * 3, np.array([1.0], np.float32))
    mats = synth.factor_matrices((5, 6, 8), 8, seed=1)
    with pytest.raises(PtiError) as e:
        coo.mttkrp(mats, 8, 0)
    assert e.value.code == 2
    code = lib.ptiGetLastError(ffi.NULL, ffi.NULL, ffi.NULL, ffi.NULL)
    assert code == 2
    lib.ptiClearLastError()
    assert lib.ptiGetLastError(ffi.NULL, ffi.NULL, ffi.NULL, ffi.NULL) == 0


def test_conversion_argument_checks(lib):
    dims = (5, 6)
    coo = COOTensor(dims, [np.array([1], np.uint32)] * 2, np.array([1.0], np.float32))
    with pytest.raises(PtiError) as e:
        coo.to_hicoo(2, 3, 3)  # 2-D: the reference has no Morton order for it
    assert e.value.code == 3
    with pytest.raises(PtiError) as e:
        COOTensor((5, 6, 7), [np.array([1], np.uint32)] * 3, np.array([1.0], np.float32)).to_hicoo(4, 3, 5)
    assert e.value.code == 3


def test_hicoo_struct_round_trip(lib):
    h = HiCOOTensor((4, 4, 4), 1, 2, 2, np.array([0, 2], np.uint64), [np.array([1], np.uint32)] * 3,
                    [np.array([0, 1], np.uint8)] * 3, np.array([1, 2], np.float32))
    assert h.nb == 1 and h.nnz == 2
    assert h.c.bptr.len == 2 and h.c.binds[0].data[0] == 1


def test_l2_probe_rejects_bad_arguments_before_any_gpu_work(lib):
    gb = ffi.new("double *", -1.0)
    assert lib.ptiB200ProbeL2ReadBandwidth(1 << 19, 10, gb) == 3      # under 1 MiB: PTIERR_VALUE_ERROR
    assert lib.ptiB200ProbeL2ReadBandwidth(64 << 20, 0, gb) == 3      # no repetition
    assert lib.ptiB200ProbeL2ReadBandwidth(2 << 30, 10, gb) == 3      # over 1 GiB
    assert lib.ptiB200ProbeL2ReadBandwidth(64 << 20, 10, ffi.NULL) == 3
    assert gb[0] == -1.0
