"""cffi (ABI mode) binding of libhiparti_b200.so.

The declarations are read from include/hiparti_b200.h, the same header C
callers use, so the Python and C views of the structs cannot drift apart.  This
replaces the reference's HiParTIPy/PtiCffi.py, whose cdef lacks the MTTKRP,
HiCOO and CPD entry points (PtiCffi.py:188-272).
"""
from __future__ import annotations

import re
from pathlib import Path

import cffi

_PKG = Path(__file__).resolve().parent
HEADER = _PKG.parent / "include" / "hiparti_b200.h"
LIBPATH = _PKG / "libhiparti_b200.so"

ffi = cffi.FFI()


def _cdef_source() -> str:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = []
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#") or s in ('extern "C" {', "}") and "extern" in s:
            continue
        if s == 'extern "C" {':
            continue
        out.append(line)
    src = "\n".join(out)
    # drop the closing brace of the extern "C" block (guarded by #ifdef above)
    return src


_src = _cdef_source()
# The extern "C" braces sit inside #ifdef __cplusplus blocks, which were removed
# with the other preprocessor lines except the lone closing brace; remove it.
_src = re.sub(r"\n\s*}\s*\n(?=\s*$)", "\n", _src)
ffi.cdef(_src)

_lib = None


def lib():
    """The loaded library.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not LIBPATH.exists():
            raise RuntimeError(
                f"{LIBPATH} is missing; build it with `python -m hiparti_b200.build`")
        _lib = ffi.dlopen(str(LIBPATH))
    return _lib


def last_error() -> str:
    L = lib()
    module = ffi.new("char **")
    fname = ffi.new("char **")
    line = ffi.new("unsigned *")
    reason = ffi.new("char **")
    code = L.ptiGetLastError(module, fname, line, reason)
    def s(p):
        return ffi.string(p[0]).decode() if p[0] != ffi.NULL else ""
    return f"code 0x{code:x} [{s(module)}] {s(reason)} ({s(fname)}:{line[0]})"


class PtiError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where} failed: {last_error()}")


def check(code: int, where: str) -> None:
    if code != 0:
        raise PtiError(code, where)
