"""TEST INFRASTRUCTURE ONLY: ctypes front of oracle/_ref/libbulkref.so, the
reference's own algorithms compiled for the host (oracle/ref/build_ref.py).

``available()`` is False when the library was not built (the reference
sources are needed to build it; the built library travels with the repo
working tree).  Only tests/ and bench.py's CPU-baseline legs use this.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libbulkref.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(LIB_PATH))
        P, I64, I32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
        sig = {
            "bkref_cpu_reduce_i32": (I32, [P, I64, I32, ctypes.c_int]),
            "bkref_cpu_reduce_f32": (ctypes.c_float, [P, I64, ctypes.c_float, ctypes.c_int]),
            "bkref_cpu_reduce_f64": (ctypes.c_double, [P, I64, ctypes.c_double, ctypes.c_int]),
            "bkref_cpu_inclusive_scan_i32": (None, [P, I64, I32, P, ctypes.c_int]),
            "bkref_cpu_inclusive_scan_f32": (None, [P, I64, ctypes.c_float, P, ctypes.c_int]),
            "bkref_cpu_inclusive_scan_f64": (None, [P, I64, ctypes.c_double, P, ctypes.c_int]),
            "bkref_merge_i32": (None, [P, I64, P, I64, P]),
            "bkref_merge_f32": (None, [P, I64, P, I64, P]),
            "bkref_merge_path_i32": (I64, [P, I64, P, I64, I64]),
            "bkref_group_reduce_i32": (I32, [P, I64, I32]),
            "bkref_group_inclusive_scan_i32": (None, [P, I64, I32, P]),
            "bkref_group_reduce_by_key_i32_i32": (I64, [P, P, I64, P, P]),
            "bkref_group_stable_sort_by_key_i32_i32": (None, [P, P, I64]),
            "bkref_group_merge_by_key_i32_i32": (None, [P, P, I64, P, P, I64, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype, f.argtypes = res, args
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


_TAG = {np.dtype(np.int32): "i32", np.dtype(np.float32): "f32", np.dtype(np.float64): "f64"}


def cpu_reduce(x: np.ndarray, init, threads: int | None = None):
    x = np.ascontiguousarray(x)
    return getattr(lib(), f"bkref_cpu_reduce_{_TAG[x.dtype]}")(_p(x), x.size, init, threads or os.cpu_count() or 1)


def cpu_inclusive_scan(x: np.ndarray, init, threads: int | None = None, out: np.ndarray | None = None):
    x = np.ascontiguousarray(x)
    out = np.empty_like(x) if out is None else out
    getattr(lib(), f"bkref_cpu_inclusive_scan_{_TAG[x.dtype]}")(_p(x), x.size, init, _p(out),
                                                               threads or os.cpu_count() or 1)
    return out


def merge(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    out = np.empty(a.size + b.size, dtype=a.dtype)
    getattr(lib(), f"bkref_merge_{_TAG[a.dtype]}")(_p(a), a.size, _p(b), b.size, _p(out))
    return out


def merge_path(a, b, diag):
    return lib().bkref_merge_path_i32(_p(a), a.size, _p(b), b.size, diag)


def group_reduce(x, init):
    x = np.ascontiguousarray(x, dtype=np.int32)
    return lib().bkref_group_reduce_i32(_p(x), x.size, init)


def group_inclusive_scan(x, init):
    x = np.ascontiguousarray(x, dtype=np.int32)
    out = np.empty_like(x)
    lib().bkref_group_inclusive_scan_i32(_p(x), x.size, init, _p(out))
    return out


def group_reduce_by_key(keys, vals):
    keys = np.ascontiguousarray(keys, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.int32)
    ok, ov = np.empty_like(keys), np.empty_like(vals)
    c = lib().bkref_group_reduce_by_key_i32_i32(_p(keys), _p(vals), keys.size, _p(ok), _p(ov))
    return ok[:c], ov[:c]


def group_stable_sort_by_key(keys, vals):
    k = np.array(keys, dtype=np.int32, copy=True)
    v = np.array(vals, dtype=np.int32, copy=True)
    assert k.size <= 12
    lib().bkref_group_stable_sort_by_key_i32_i32(_p(k), _p(v), k.size)
    return k, v


def group_merge_by_key(ak, av, bk, bv):
    ak, av, bk, bv = (np.ascontiguousarray(t, dtype=np.int32) for t in (ak, av, bk, bv))
    assert ak.size + bk.size <= 12
    ok = np.empty(ak.size + bk.size, np.int32)
    ov = np.empty_like(ok)
    lib().bkref_group_merge_by_key_i32_i32(_p(ak), _p(av), ak.size, _p(bk), _p(bv), bk.size, _p(ok), _p(ov))
    return ok, ov
