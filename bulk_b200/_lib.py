"""ctypes binding of libbulkb200.so, generated from include/bulk_b200.h.

Every ``BK_API`` declaration in the header becomes a ctypes function with the
matching argument and return types, so the binding cannot drift from the
C-ABI.  Loading fails loudly when the library has not been built: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "bulk_b200.h"
LIB_PATH = PKG / "lib" / "libbulkb200.so"

_CTYPES = {
    "void": None,
    "int": ctypes.c_int,
    "size_t": ctypes.c_size_t,
    "int32_t": ctypes.c_int32,
    "uint32_t": ctypes.c_uint32,
    "int64_t": ctypes.c_int64,
    "uint64_t": ctypes.c_uint64,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "bk_stream_t": ctypes.c_void_p,
    "const char *": ctypes.c_char_p,
}

_DECL = re.compile(r"^BK_API\s+(.+?)\s*\b(bk_\w+)\((.*?)\);", re.M)


def _ctype(decl: str):
    decl = " ".join(decl.split())
    if decl in _CTYPES:
        return _CTYPES[decl]
    if "*" in decl:
        return ctypes.c_void_p
    raise ValueError(f"unmapped C type: {decl!r}")


def parse_header(text: str | None = None) -> dict[str, tuple]:
    """Map each declared entry point to (restype, [argtypes])."""
    text = HEADER.read_text() if text is None else text
    out = {}
    for ret, name, args in _DECL.findall(text):
        argtypes = []
        args = args.strip()
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                m = re.match(r"(.*?)(\w+)$", a)
                argtypes.append(_ctype(m.group(1).strip()))
        out[name] = (_ctype(ret.strip()), argtypes)
    return out


DECLS = parse_header()


class BulkError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = _lib.bk_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{where}: status {status} ({msg})")


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python bulk_b200/build.py` "
            "(the CUDA library is the only implementation; there is no fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in DECLS.items():
        fn = getattr(lib, name)  # AttributeError = header/library mismatch
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None
_lib = _load()
lib = _lib

BK_OK = 0
BK_ERR_INVALID_ARGUMENT = -1
BK_ERR_WORKSPACE_TOO_SMALL = -2
BK_ERR_SPIN_TIMEOUT = -3
BK_ERR_MISALIGNED = -4
BK_ERR_TOO_LARGE = -5
BK_ERR_UNSUPPORTED = -6

ALGO = {"reduce": 1, "inclusive_scan": 2, "merge": 3, "sort_by_key": 4, "reduce_by_key": 5}
DTYPE = {None: 0, "i32": 1, "u32": 2, "i64": 3, "u64": 4, "f32": 5, "f64": 6}


def check(status: int, where: str) -> None:
    if status != BK_OK:
        raise BulkError(status, where)
