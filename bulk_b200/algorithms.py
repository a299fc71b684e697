"""Device-wide algorithms over torch CUDA tensors, calling the C-ABI.

These mirror the reference's device-wide drivers (their names, argument
meaning and in-place behaviour) so tests and benchmarks read like the
reference's own drivers:

=====================  ======================================================
this module            reference (jaredhoberock/bulk)
=====================  ======================================================
``reduce``             ``my_reduce(first, last, init, op)``  reduce.cu:58-97
``inclusive_scan``     ``::inclusive_scan(first, last, result, init, op)``
                       scan.cu:87-148
``merge``              ``my_merge(first1, last1, first2, last2, result, comp)``
                       merge.cu:127-162 (+ by-key block merge merge.hpp:507-607)
``stable_sort_by_key`` ``stable_merge_sort_by_key(keys_first, keys_last,
                       values_first, comp)`` merge_sort_by_key.cu:150-209
``reduce_by_key``      ``my_reduce_by_key(keys_first, keys_last, values_first,
                       keys_result, values_result, pred, op)``
                       reduce_by_key.cu:176-272
=====================  ======================================================

torch provides device memory and streams only; every computation runs in
libbulkb200.so.  Errors raise :class:`bulk_b200.BulkError`.
"""
from __future__ import annotations

import ctypes
import threading

import torch

from . import _lib
from ._lib import check, lib

_TORCH_TO_TAG = {
    torch.int32: "i32",
    torch.int64: "i64",
    torch.float32: "f32",
    torch.float64: "f64",
}
for _name, _tag in (("uint32", "u32"), ("uint64", "u64")):
    if hasattr(torch, _name):
        _TORCH_TO_TAG[getattr(torch, _name)] = _tag


def dtype_tag(t: torch.dtype) -> str:
    try:
        return _TORCH_TO_TAG[t]
    except KeyError:
        raise TypeError(f"unsupported dtype {t}") from None


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_obj(stream: torch.cuda.Stream | None, device: torch.device) -> torch.cuda.Stream:
    return stream if stream is not None else torch.cuda.current_stream(device)


def _stream_handle(stream: torch.cuda.Stream | None, device: torch.device) -> int:
    return _stream_obj(stream, device).cuda_stream


def _require_cuda(*ts: torch.Tensor) -> torch.device:
    dev = None
    for t in ts:
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError("bulk_b200 operates on CUDA tensors (device memory)")
        if not t.is_contiguous():
            raise ValueError("bulk_b200 needs contiguous tensors")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise ValueError("all tensors must be on the same device")
    return dev


class _WorkspacePool:
    """One zero-initialised device workspace per (device, stream), grown on demand.

    The library leaves every workspace's counters zeroed after each call, so a
    workspace is reused across calls on the same stream without re-clearing.
    A workspace is allocated and zero-filled on the stream that uses it, so the
    fill is ordered before the library's kernels there; when it grows, the old
    buffer goes back to torch's caching allocator as a block of that stream,
    which hands it out again only in that stream's order, after the kernels
    already queued on it.
    """

    def __init__(self):
        self._lock = threading.Lock()
        self._ws: dict[tuple[int, int], torch.Tensor] = {}

    def get(self, nbytes: int, device: torch.device, stream: torch.cuda.Stream) -> tuple[int, int]:
        key = (device.index if device.index is not None else torch.cuda.current_device(), stream.cuda_stream)
        with self._lock:
            t = self._ws.get(key)
            if t is None or t.numel() < nbytes:
                size = max(nbytes, 1 << 16, 0 if t is None else 2 * t.numel())
                with torch.cuda.stream(stream):
                    t = torch.zeros(size, dtype=torch.uint8, device=device)
                self._ws[key] = t
            return t.data_ptr(), t.numel()

    def status(self, device: torch.device | None = None, stream: torch.cuda.Stream | None = None) -> int:
        device = device or torch.device("cuda", torch.cuda.current_device())
        s = _stream_handle(stream, device)
        key = (device.index if device.index is not None else torch.cuda.current_device(), s)
        t = self._ws.get(key)
        if t is None:
            return _lib.BK_OK
        return lib.bk_workspace_status(t.data_ptr(), t.numel(), s)

    def clear(self):
        with self._lock:
            self._ws.clear()


workspaces = _WorkspacePool()


def workspace_bytes(algo: str, key: str, value: str | None, n: int) -> int:
    return lib.bk_workspace_bytes(_lib.ALGO[algo], _lib.DTYPE[key], _lib.DTYPE[value], n)


def workspace_status(device=None, stream=None) -> int:
    """Synchronize and return (and clear) the device-side status of this stream's workspace."""
    return workspaces.status(device, stream)


def debug_set_fault(skip_publish_tile: int = -1, spin_limit_ns: int = 0) -> None:
    check(lib.bk_debug_set_fault(skip_publish_tile, spin_limit_ns), "bk_debug_set_fault")


def _ws(algo, key, value, n, device, stream: torch.cuda.Stream):
    need = workspace_bytes(algo, key, value, n)
    if need == 0 and algo not in ("reduce",):
        return None, 0
    return workspaces.get(max(need, 256), device, stream)


# ---------------------------------------------------------------------------
def reduce(x: torch.Tensor, init=0, op: str = "sum", out: torch.Tensor | None = None,
           stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """Return a 1-element device tensor holding init (+) x[0] (+) ... (+) x[n-1]."""
    dev = _require_cuda(x, out)
    tag = dtype_tag(x.dtype)
    if out is None:
        out = torch.empty(1, dtype=x.dtype, device=dev)
    with torch.cuda.device(dev):
        so = _stream_obj(stream, dev)
        s = so.cuda_stream
        ws, wsb = _ws("reduce", tag, None, x.numel(), dev, so)
        fn = getattr(lib, f"bk_reduce_{op}_{tag}")
        check(fn(_ptr(x), x.numel(), init, _ptr(out), ws, wsb, s), fn.__name__)
    return out


def inclusive_scan(x: torch.Tensor, init=0, op: str = "sum", out: torch.Tensor | None = None,
                   stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """out[i] = init (+) x[0] (+) ... (+) x[i]; ``out`` may be ``x`` (in place).

    ``init`` may be a device tensor of x's dtype (one element, or a view of
    one, e.g. the last output of a previous scan): it is then read on the
    device when the scan runs, with no copy to the host."""
    dev = _require_cuda(x, out)
    tag = dtype_tag(x.dtype)
    if out is None:
        out = torch.empty_like(x)
    dinit = isinstance(init, torch.Tensor)
    if dinit:
        if not init.is_cuda or init.device != dev or init.dtype != x.dtype or init.numel() != 1:
            raise ValueError("a tensor init must be one element of x's dtype on x's device")
    with torch.cuda.device(dev):
        so = _stream_obj(stream, dev)
        s = so.cuda_stream
        ws, wsb = _ws("inclusive_scan", tag, None, x.numel(), dev, so)
        if dinit:
            fn = getattr(lib, f"bk_inclusive_scan_{op}_{tag}_dinit")
            check(fn(_ptr(x), x.numel(), _ptr(init), _ptr(out), ws, wsb, s), fn.__name__)
        else:
            fn = getattr(lib, f"bk_inclusive_scan_{op}_{tag}")
            check(fn(_ptr(x), x.numel(), init, _ptr(out), ws, wsb, s), fn.__name__)
    return out


def _payload_tag(t: torch.Tensor | None) -> str | None:
    if t is None:
        return None
    if t.element_size() == 4:
        return "u32"
    if t.element_size() == 8:
        return "u64"
    raise TypeError("payloads must be 4- or 8-byte elements")


def merge(a: torch.Tensor, b: torch.Tensor, a_vals: torch.Tensor | None = None, b_vals: torch.Tensor | None = None,
          out: torch.Tensor | None = None, out_vals: torch.Tensor | None = None,
          stream: torch.cuda.Stream | None = None):
    """Stable merge of sorted a and b (ties: a first).  Returns keys, or (keys, vals) with payloads."""
    dev = _require_cuda(a, b, a_vals, b_vals, out, out_vals)
    if a.dtype != b.dtype:
        raise TypeError("a and b must have the same dtype")
    tag = dtype_tag(a.dtype)
    n = a.numel() + b.numel()
    if out is None:
        out = torch.empty(n, dtype=a.dtype, device=dev)
    if a_vals is not None and (b_vals is None or a_vals.element_size() != b_vals.element_size()):
        raise TypeError("a_vals and b_vals must both be given, with the same element size")
    if a_vals is not None and out_vals is None:
        out_vals = torch.empty(n, dtype=a_vals.dtype, device=dev)
    with torch.cuda.device(dev):
        so = _stream_obj(stream, dev)
        s = so.cuda_stream
        ws, wsb = _ws("merge", tag, _payload_tag(a_vals), n, dev, so)
        if a_vals is None:
            fn = getattr(lib, f"bk_merge_{tag}")
            check(fn(_ptr(a), a.numel(), _ptr(b), b.numel(), _ptr(out), ws, wsb, s), fn.__name__)
            return out
        fn = getattr(lib, f"bk_merge_by_key_{tag}_{_payload_tag(a_vals)}")
        check(fn(_ptr(a), _ptr(a_vals), a.numel(), _ptr(b), _ptr(b_vals), b.numel(), _ptr(out), _ptr(out_vals),
                 ws, wsb, s), fn.__name__)
    return out, out_vals


def stable_sort_by_key(keys: torch.Tensor, vals: torch.Tensor | None = None,
                       stream: torch.cuda.Stream | None = None):
    """In-place stable sort of keys (and vals with them).  Returns keys, or (keys, vals)."""
    dev = _require_cuda(keys, vals)
    tag = dtype_tag(keys.dtype)
    n = keys.numel()
    if vals is not None and vals.numel() != n:
        raise ValueError("keys and vals must have the same length")
    with torch.cuda.device(dev):
        so = _stream_obj(stream, dev)
        s = so.cuda_stream
        ws, wsb = _ws("sort_by_key", tag, _payload_tag(vals), n, dev, so)
        if vals is None:
            fn = getattr(lib, f"bk_sort_keys_{tag}")
            check(fn(_ptr(keys), n, ws, wsb, s), fn.__name__)
            return keys
        fn = getattr(lib, f"bk_sort_by_key_{tag}_{_payload_tag(vals)}")
        check(fn(_ptr(keys), _ptr(vals), n, ws, wsb, s), fn.__name__)
    return keys, vals


def reduce_by_key(keys: torch.Tensor, vals: torch.Tensor, out_keys: torch.Tensor | None = None,
                  out_vals: torch.Tensor | None = None, num_out: torch.Tensor | None = None,
                  stream: torch.cuda.Stream | None = None, sync: bool = True):
    """One (key, sum) pair per run of equal consecutive keys.

    Returns (out_keys, out_vals, count).  With ``sync=True`` (the reference's
    behaviour, reduce_by_key.cu:269) count is a Python int and the outputs are
    trimmed to it; with ``sync=False`` count stays a 1-element device tensor
    and the outputs are the full-length buffers.
    """
    dev = _require_cuda(keys, vals, out_keys, out_vals, num_out)
    n = keys.numel()
    if vals.numel() != n:
        raise ValueError("keys and vals must have the same length")
    kt, vt = dtype_tag(keys.dtype), dtype_tag(vals.dtype)
    if out_keys is None:
        out_keys = torch.empty(max(n, 1), dtype=keys.dtype, device=dev)
    if out_vals is None:
        out_vals = torch.empty(max(n, 1), dtype=vals.dtype, device=dev)
    if num_out is None:
        num_out = torch.empty(1, dtype=torch.int64, device=dev)
    with torch.cuda.device(dev):
        so = _stream_obj(stream, dev)
        s = so.cuda_stream
        ws, wsb = _ws("reduce_by_key", kt, vt, n, dev, so)
        fn = getattr(lib, f"bk_reduce_by_key_{kt}_{vt}")
        check(fn(_ptr(keys), _ptr(vals), n, _ptr(out_keys), _ptr(out_vals), _ptr(num_out), ws, wsb, s),
              fn.__name__)
    if not sync:
        return out_keys, out_vals, num_out
    c = int(num_out.item())
    return out_keys[:c], out_vals[:c], c
