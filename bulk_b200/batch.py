"""Batched entry points: many independent arrays per launch.

No counterpart in the reference, whose drivers launch once per array.  Each
call hands up to ``BATCH_MAX`` arrays to one persistent launch (longer lists
are split into several); every array's result is what the single-array entry
point gives for it.  Small arrays are where this pays: one launch keeps all
SMs busy with many of them instead of a mostly idle grid per array.

torch provides device memory and streams only; the work runs in
libbulkb200.so.  Errors raise :class:`bulk_b200.BulkError`.
"""
from __future__ import annotations

import ctypes
from functools import lru_cache

import torch

from . import _lib
from ._lib import check, lib
from .algorithms import _require_cuda, _stream_obj, dtype_tag, workspaces

BATCH_MAX = 256

_CT = {"i32": ctypes.c_int32, "u32": ctypes.c_uint32, "i64": ctypes.c_int64, "u64": ctypes.c_uint64,
       "f32": ctypes.c_float, "f64": ctypes.c_double}


@lru_cache(maxsize=None)
def scan_item_type(tag: str):
    """ctypes mirror of bk_scan_item_<tag>."""
    return type(f"bk_scan_item_{tag}", (ctypes.Structure,),
                {"_fields_": [("d_in", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("n", ctypes.c_uint64),
                              ("init", _CT[tag])]})


@lru_cache(maxsize=None)
def rbk_item_type(key: str, value: str):
    """ctypes mirror of bk_rbk_item_<key>_<value>."""
    return type(f"bk_rbk_item_{key}_{value}", (ctypes.Structure,),
                {"_fields_": [("keys", ctypes.c_void_p), ("vals", ctypes.c_void_p), ("n", ctypes.c_uint64),
                              ("out_keys", ctypes.c_void_p), ("out_vals", ctypes.c_void_p),
                              ("d_num_out", ctypes.c_void_p)]})


@lru_cache(maxsize=None)
def sort_item_type(key: str, value: str):
    """ctypes mirror of bk_sort_item_<key>_<value>."""
    return type(f"bk_sort_item_{key}_{value}", (ctypes.Structure,),
                {"_fields_": [("keys", ctypes.c_void_p), ("vals", ctypes.c_void_p), ("n", ctypes.c_uint64)]})


@lru_cache(maxsize=None)
def sort_copy_item_type(key: str, value: str):
    """ctypes mirror of bk_sort_copy_item_<key>_<value>."""
    return type(f"bk_sort_copy_item_{key}_{value}", (ctypes.Structure,),
                {"_fields_": [("in_keys", ctypes.c_void_p), ("in_vals", ctypes.c_void_p), ("keys", ctypes.c_void_p),
                              ("vals", ctypes.c_void_p), ("n", ctypes.c_uint64)]})


def batch_workspace_bytes(algo: str, key: str, value: str | None, sizes) -> int:
    arr = (ctypes.c_uint64 * max(len(sizes), 1))(*sizes)
    return lib.bk_batch_workspace_bytes(_lib.ALGO[algo], _lib.DTYPE[key], _lib.DTYPE[value], arr, len(sizes))


def _chunks(n: int):
    for lo in range(0, n, BATCH_MAX):
        yield lo, min(n, lo + BATCH_MAX)


def inclusive_scan_batch(xs, inits=None, outs=None, stream: torch.cuda.Stream | None = None):
    """Inclusive sum scan of every tensor in ``xs`` (all of one dtype):
    outs[k][i] = inits[k] + xs[k][0] + ... + xs[k][i].  Returns the outputs."""
    xs = list(xs)
    if not xs:
        return []
    dev = _require_cuda(*xs, *(outs or []))
    tag = dtype_tag(xs[0].dtype)
    if any(dtype_tag(x.dtype) != tag for x in xs):
        raise TypeError("one dtype per batch")
    inits = list(inits) if inits is not None else [0] * len(xs)
    outs = list(outs) if outs is not None else [torch.empty_like(x) for x in xs]
    if len(inits) != len(xs) or len(outs) != len(xs):
        raise ValueError("xs, inits and outs must have the same length")
    so = _stream_obj(stream, dev)
    s = so.cuda_stream
    item_t = scan_item_type(tag)
    fn = getattr(lib, f"bk_inclusive_scan_sum_{tag}_batch")
    for lo, hi in _chunks(len(xs)):
        items = (item_t * (hi - lo))()
        for j, k in enumerate(range(lo, hi)):
            items[j].d_in, items[j].d_out, items[j].n, items[j].init = xs[k].data_ptr(), outs[k].data_ptr(), \
                xs[k].numel(), inits[k]
        need = batch_workspace_bytes("inclusive_scan", tag, None, [xs[k].numel() for k in range(lo, hi)])
        with torch.cuda.device(dev):
            ws, wsb = workspaces.get(max(need, 256), dev, so)
            check(fn(ctypes.cast(items, ctypes.c_void_p), hi - lo, ws, wsb, s), fn.__name__)
    return outs


def reduce_by_key_batch(keys_list, vals_list, stream: torch.cuda.Stream | None = None, sync: bool = False,
                        outs=None):
    """reduce_by_key (equal keys, sum) of every (keys, vals) pair.

    Returns a list of (out_keys, out_vals, count): with ``sync=False`` count
    is a 1-element device tensor and the outputs are full-length buffers; with
    ``sync=True`` (one synchronisation for the whole batch) counts are ints and
    the outputs are trimmed.  ``outs`` optionally supplies the buffers: one
    (out_keys, out_vals, count) per pair, count a 1-element int64 tensor."""
    keys_list, vals_list = list(keys_list), list(vals_list)
    if len(keys_list) != len(vals_list):
        raise ValueError("keys_list and vals_list must have the same length")
    if not keys_list:
        return []
    dev = _require_cuda(*keys_list, *vals_list)
    kt, vt = dtype_tag(keys_list[0].dtype), dtype_tag(vals_list[0].dtype)
    for k, v in zip(keys_list, vals_list):
        if dtype_tag(k.dtype) != kt or dtype_tag(v.dtype) != vt:
            raise TypeError("one key dtype and one value dtype per batch")
        if k.numel() != v.numel():
            raise ValueError("keys and vals must have the same length")
    so = _stream_obj(stream, dev)
    s = so.cuda_stream
    item_t = rbk_item_type(kt, vt)
    fn = getattr(lib, f"bk_reduce_by_key_{kt}_{vt}_batch")
    if outs is not None:
        outs = list(outs)
        if len(outs) != len(keys_list):
            raise ValueError("one (out_keys, out_vals, count) per pair")
        _require_cuda(*(t for o in outs for t in o))
        res = [(o[0], o[1]) for o in outs]
        cnt = [o[2] for o in outs]
    else:
        counts = torch.empty(len(keys_list), dtype=torch.int64, device=dev)
        res = []
        for k, v in zip(keys_list, vals_list):
            res.append((torch.empty(max(k.numel(), 1), dtype=k.dtype, device=dev),
                        torch.empty(max(v.numel(), 1), dtype=v.dtype, device=dev)))
        cnt = [counts[i:i + 1] for i in range(len(keys_list))]
    for lo, hi in _chunks(len(keys_list)):
        items = (item_t * (hi - lo))()
        for j, i in enumerate(range(lo, hi)):
            it = items[j]
            it.keys, it.vals, it.n = keys_list[i].data_ptr(), vals_list[i].data_ptr(), keys_list[i].numel()
            it.out_keys, it.out_vals = res[i][0].data_ptr(), res[i][1].data_ptr()
            it.d_num_out = cnt[i].data_ptr()
        need = batch_workspace_bytes("reduce_by_key", kt, vt, [keys_list[i].numel() for i in range(lo, hi)])
        with torch.cuda.device(dev):
            ws, wsb = workspaces.get(max(need, 256), dev, so)
            check(fn(ctypes.cast(items, ctypes.c_void_p), hi - lo, ws, wsb, s), fn.__name__)
    if not sync:
        return [(ok, ov, cnt[i]) for i, (ok, ov) in enumerate(res)]
    cs = [int(c) for c in torch.cat([c.view(1) for c in cnt]).tolist()]
    return [(ok[:c], ov[:c], c) for (ok, ov), c in zip(res, cs)]


def stable_sort_by_key_batch(keys_list, vals_list, stream: torch.cuda.Stream | None = None):
    """Stable sort of every (keys, vals) pair in place (payloads of 4 or 8
    bytes, passed through unchanged).  Returns the lists."""
    keys_list, vals_list = list(keys_list), list(vals_list)
    if len(keys_list) != len(vals_list):
        raise ValueError("keys_list and vals_list must have the same length")
    if not keys_list:
        return keys_list, vals_list
    dev = _require_cuda(*keys_list, *vals_list)
    kt = dtype_tag(keys_list[0].dtype)
    vsize = vals_list[0].element_size()
    if vsize not in (4, 8):
        raise TypeError("payloads must be 4 or 8 bytes")
    vt = "u32" if vsize == 4 else "u64"
    for k, v in zip(keys_list, vals_list):
        if dtype_tag(k.dtype) != kt or v.element_size() != vsize:
            raise TypeError("one key dtype and one payload size per batch")
        if k.numel() != v.numel():
            raise ValueError("keys and vals must have the same length")
    so = _stream_obj(stream, dev)
    s = so.cuda_stream
    item_t = sort_item_type(kt, vt)
    fn = getattr(lib, f"bk_sort_by_key_{kt}_{vt}_batch")
    for lo, hi in _chunks(len(keys_list)):
        items = (item_t * (hi - lo))()
        for j, i in enumerate(range(lo, hi)):
            items[j].keys, items[j].vals, items[j].n = keys_list[i].data_ptr(), vals_list[i].data_ptr(), \
                keys_list[i].numel()
        need = batch_workspace_bytes("sort_by_key", kt, vt, [keys_list[i].numel() for i in range(lo, hi)])
        with torch.cuda.device(dev):
            ws, wsb = workspaces.get(max(need, 256), dev, so)
            check(fn(ctypes.cast(items, ctypes.c_void_p), hi - lo, ws, wsb, s), fn.__name__)
    return keys_list, vals_list


def stable_sort_by_key_copy_batch(in_keys, in_vals, out_keys=None, out_vals=None,
                                  stream: torch.cuda.Stream | None = None):
    """Stable sort of every (in_keys[i], in_vals[i]) pair into (out_keys[i],
    out_vals[i]) (allocated when not given); the inputs are left unchanged.
    Returns (out_keys, out_vals)."""
    in_keys, in_vals = list(in_keys), list(in_vals)
    if len(in_keys) != len(in_vals):
        raise ValueError("in_keys and in_vals must have the same length")
    out_keys = list(out_keys) if out_keys is not None else [torch.empty_like(k) for k in in_keys]
    out_vals = list(out_vals) if out_vals is not None else [torch.empty_like(v) for v in in_vals]
    if not in_keys:
        return out_keys, out_vals
    dev = _require_cuda(*in_keys, *in_vals, *out_keys, *out_vals)
    kt = dtype_tag(in_keys[0].dtype)
    vsize = in_vals[0].element_size()
    if vsize not in (4, 8):
        raise TypeError("payloads must be 4 or 8 bytes")
    vt = "u32" if vsize == 4 else "u64"
    for k, v, ok, ov in zip(in_keys, in_vals, out_keys, out_vals):
        if dtype_tag(k.dtype) != kt or v.element_size() != vsize or ok.dtype != k.dtype or \
                ov.element_size() != vsize:
            raise TypeError("one key dtype and one payload size per batch")
        if not (k.numel() == v.numel() == ok.numel() == ov.numel()):
            raise ValueError("every array of an item must have the same length")
    so = _stream_obj(stream, dev)
    s = so.cuda_stream
    item_t = sort_copy_item_type(kt, vt)
    fn = getattr(lib, f"bk_sort_by_key_{kt}_{vt}_copy_batch")
    for lo, hi in _chunks(len(in_keys)):
        items = (item_t * (hi - lo))()
        for j, i in enumerate(range(lo, hi)):
            it = items[j]
            it.in_keys, it.in_vals = in_keys[i].data_ptr(), in_vals[i].data_ptr()
            it.keys, it.vals, it.n = out_keys[i].data_ptr(), out_vals[i].data_ptr(), in_keys[i].numel()
        need = batch_workspace_bytes("sort_by_key", kt, vt, [in_keys[i].numel() for i in range(lo, hi)])
        with torch.cuda.device(dev):
            ws, wsb = workspaces.get(max(need, 256), dev, so)
            check(fn(ctypes.cast(items, ctypes.c_void_p), hi - lo, ws, wsb, s), fn.__name__)
    return out_keys, out_vals
