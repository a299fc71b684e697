"""TEST INFRASTRUCTURE ONLY: numpy front of the C oracle (oracle.c).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, as the checker of the CUDA library; the product never imports
it.  Each function restates one of the reference's device-wide algorithms
(see the citations in oracle.c).
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "lib" / "liboracle.so"

if not LIB_PATH.exists():
    from .build import build as _build  # gcc is on every machine that runs the tests
    _build()

_lib = ctypes.CDLL(str(LIB_PATH))

_C = {
    np.dtype(np.int32): ("i32", ctypes.c_int32),
    np.dtype(np.uint32): ("u32", ctypes.c_uint32),
    np.dtype(np.int64): ("i64", ctypes.c_int64),
    np.dtype(np.uint64): ("u64", ctypes.c_uint64),
    np.dtype(np.float32): ("f32", ctypes.c_float),
    np.dtype(np.float64): ("f64", ctypes.c_double),
}
EPS = {np.dtype(np.float32): 2.0 ** -23, np.dtype(np.float64): 2.0 ** -52}

P = ctypes.c_void_p
U64 = ctypes.c_uint64


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _fn(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


# ---------------------------------------------------------------- generators
def gen(dtype, n: int, seed: int, lo=None, hi=None) -> np.ndarray:
    """Counter-based synthetic input; ``bko_mix64(seed, i)`` drives element i."""
    dt = np.dtype(dtype)
    out = np.empty(n, dtype=dt)
    if dt == np.int32:
        _fn("bko_gen_i32", None, [P, U64, U64, ctypes.c_int32, ctypes.c_int32])(_p(out), n, seed, lo, hi)
    elif dt == np.uint32:
        _fn("bko_gen_u32", None, [P, U64, U64])(_p(out), n, seed)
    elif dt == np.uint64:
        _fn("bko_gen_u64", None, [P, U64, U64])(_p(out), n, seed)
    elif dt == np.float32:
        _fn("bko_gen_f32", None, [P, U64, U64, ctypes.c_float, ctypes.c_float])(_p(out), n, seed, lo, hi)
    elif dt == np.float64:
        _fn("bko_gen_f64", None, [P, U64, U64, ctypes.c_double, ctypes.c_double])(_p(out), n, seed, lo, hi)
    else:
        raise TypeError(dt)
    return out


def ref_hash(i: int) -> int:
    return _fn("bko_ref_hash", ctypes.c_int64, [ctypes.c_int64])(i)


def ref_hash_fill_i32(n: int, modulus: int = 0) -> np.ndarray:
    """The reference drivers' random_fill (hash of the index, optionally % modulus)."""
    out = np.empty(n, dtype=np.int32)
    _fn("bko_ref_hash_fill_i32", None, [P, U64, ctypes.c_int32])(_p(out), n, modulus)
    return out


def gen_runs_geometric(n: int, seed: int, mean: float) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    _fn("bko_gen_runs_geometric", U64, [P, U64, U64, ctypes.c_double])(_p(out), n, seed, mean)
    return out


def gen_runs_zipf(n: int, seed: int, s: float, cap: int) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    _fn("bko_gen_runs_zipf", U64, [P, U64, U64, ctypes.c_double, U64])(_p(out), n, seed, s, cap)
    return out


# -------------------------------------------------------------------- bounds
def fp_bound(n: int, dtype, abs_sum):
    """2 * ceil(log2 n) * eps * sum|x|: the stated float tolerance."""
    dt = np.dtype(dtype)
    lg = max(1, math.ceil(math.log2(max(n, 2))))
    return 2.0 * lg * EPS[dt] * np.asarray(abs_sum, dtype=np.float64)


# -------------------------------------------------------------------- reduce
def reduce(x: np.ndarray, init, op: str = "sum"):
    """Integer: exact (wrapping) result.  Float sum: (fp64 result, sum|x|)."""
    x = np.ascontiguousarray(x)
    tag, ct = _C[x.dtype]
    if op == "sum" and tag in ("f32", "f64"):
        mag = ctypes.c_double()
        f = _fn(f"bko_reduce_sum_{tag}", ctypes.c_double, [P, U64, ct, ctypes.POINTER(ctypes.c_double)])
        return f(_p(x), x.size, init, ctypes.byref(mag)), mag.value
    f = _fn(f"bko_reduce_{op}_{tag}", ct, [P, U64, ct])
    return f(_p(x), x.size, init)


def inclusive_scan(x: np.ndarray, init, op: str = "sum"):
    """Integer: exact array.  Float sum: (fp64 prefix array, sum|x| prefix array)."""
    x = np.ascontiguousarray(x)
    tag, ct = _C[x.dtype]
    if op == "sum" and tag in ("f32", "f64"):
        out = np.empty(x.size, dtype=np.float64)
        mag = np.empty(x.size, dtype=np.float64)
        _fn(f"bko_inclusive_scan_sum_{tag}", None, [P, U64, ct, P, P])(_p(x), x.size, init, _p(out), _p(mag))
        return out, mag
    out = np.empty_like(x)
    _fn(f"bko_inclusive_scan_{op}_{tag}", None, [P, U64, ct, P])(_p(x), x.size, init, _p(out))
    return out


# --------------------------------------------------------------- merge / sort
def merge_path(a: np.ndarray, b: np.ndarray, diag: int) -> int:
    tag, _ = _C[a.dtype]
    return _fn(f"bko_merge_path_{tag}", U64, [P, U64, P, U64, U64])(_p(a), a.size, _p(b), b.size, diag)


def merge(a: np.ndarray, b: np.ndarray, av: np.ndarray | None = None, bv: np.ndarray | None = None):
    """Stable merge (ties take A first); returns keys or (keys, values)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b.astype(a.dtype, copy=False))
    tag, _ = _C[a.dtype]
    out = np.empty(a.size + b.size, dtype=a.dtype)
    vb = 0
    outv = None
    if av is not None:
        av = np.ascontiguousarray(av)
        bv = np.ascontiguousarray(bv.astype(av.dtype, copy=False))
        vb = av.dtype.itemsize
        outv = np.empty(a.size + b.size, dtype=av.dtype)
    _fn(f"bko_merge_{tag}", None, [P, P, U64, P, P, U64, P, P, ctypes.c_int])(
        _p(a), _p(av), a.size, _p(b), _p(bv), b.size, _p(out), _p(outv), vb)
    return out if av is None else (out, outv)


def stable_sort_by_key(keys: np.ndarray, vals: np.ndarray | None = None):
    """Returns sorted copies: keys, or (keys, values) in stable order."""
    k = np.array(keys, copy=True, order="C")
    v = None if vals is None else np.array(vals, copy=True, order="C")
    tag, _ = _C[k.dtype]
    _fn(f"bko_stable_sort_by_key_{tag}", None, [P, P, U64, ctypes.c_int])(
        _p(k), _p(v), k.size, 0 if v is None else v.dtype.itemsize)
    return k if v is None else (k, v)


# ------------------------------------------------------------ reduce_by_key
def reduce_by_key(keys: np.ndarray, vals: np.ndarray):
    """Integer values: (keys, sums) exact.  Float values: (keys, fp64 sums, sum|v| per run)."""
    keys = np.ascontiguousarray(keys)
    vals = np.ascontiguousarray(vals)
    kt, _ = _C[keys.dtype]
    vt, _ = _C[vals.dtype]
    n = keys.size
    ok = np.empty(n, dtype=keys.dtype)
    if vt in ("f32", "f64"):
        ov = np.empty(n, dtype=np.float64)
        om = np.empty(n, dtype=np.float64)
        r = _fn(f"bko_reduce_by_key_{kt}_{vt}", U64, [P, P, U64, P, P, P])(_p(keys), _p(vals), n, _p(ok), _p(ov), _p(om))
        return ok[:r], ov[:r], om[:r]
    ov = np.empty(n, dtype=vals.dtype)
    r = _fn(f"bko_reduce_by_key_{kt}_{vt}", U64, [P, P, U64, P, P])(_p(keys), _p(vals), n, _p(ok), _p(ov))
    return ok[:r], ov[:r]
