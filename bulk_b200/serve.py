"""Serving loop: a stream of mixed requests answered one call per request
("plain") or by continuous batching ("batched").

No counterpart in the reference, whose drivers run one array at a time.  A
request is one of

* ``sort``  -- stable sort_by_key of u32 keys (full 32-bit range) with a u32
  payload (the element index), in place on the request's own copy;
* ``rbk``   -- reduce_by_key of i32 keys (run lengths 1 + Geometric, mean
  ``rbk_mean_run``) with f32 values;
* ``scan``  -- inclusive sum scan of f32 values,

of n elements, n log-uniform in [lo, hi].  Arrivals are Poisson.  Inputs are
synthetic and seeded: a request's input is a window (chosen by its id) of a
pre-generated source array of its kind, so it depends only on the id.

The loop itself is native (``bk_serve_run`` in libbulkb200.so): admission in
arrival order against an HBM budget, a pooled first-fit allocator over one
device buffer, issue on the caller's stream, completion by event polling.
``plain`` issues every admitted request as its own call (the single-array
entry points); ``batched`` issues every admitted request that has arrived at
once as one round, one batched call per kind (the kinds side by side on
streams of their own), with at most ``max_inflight`` rounds of more than four
requests queued (smaller rounds go out at once as plain calls).
Latency = completion time - arrival time, on the host's steady clock.  This
module builds the request stream and the sources, and reads the records.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .algorithms import _require_cuda, _stream_handle

KINDS = ("sort", "rbk", "scan")


# --------------------------------------------------------------------------
class DevicePool:
    """The serving loop's pooled allocator (bk_pool_*: first fit over an
    address-ordered free list, 256-byte granules, neighbours coalesced on
    free) over a byte buffer of ``capacity`` bytes on ``device``."""

    ALIGN = 256

    def __init__(self, capacity: int, device="cuda"):
        self.capacity = capacity // self.ALIGN * self.ALIGN
        self.buf = torch.empty(self.capacity, dtype=torch.uint8, device=device)
        self._h = lib.bk_pool_create(self.capacity)
        if not self._h:
            raise MemoryError("bk_pool_create failed")

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and lib is not None:
            try:
                lib.bk_pool_destroy(h)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass

    def alloc(self, nbytes: int) -> int | None:
        off = ctypes.c_uint64()
        st = lib.bk_pool_alloc(self._h, nbytes, ctypes.byref(off))
        if st == _lib.BK_ERR_TOO_LARGE:
            return None
        check(st, "bk_pool_alloc")
        return off.value

    def free(self, off: int) -> None:
        check(lib.bk_pool_free(self._h, off), "bk_pool_free")

    @property
    def in_use(self) -> int:
        return lib.bk_pool_in_use(self._h)

    @property
    def high_water(self) -> int:
        return lib.bk_pool_high_water(self._h)

    def free_blocks(self) -> int:
        return lib.bk_pool_free_blocks(self._h)

    def view(self, off: int, n: int, dtype: torch.dtype) -> torch.Tensor:
        nbytes = n * torch.empty(0, dtype=dtype).element_size()
        return self.buf[off:off + nbytes].view(dtype)


# --------------------------------------------------------------------------
@dataclass
class Request:
    rid: int
    kind: str
    n: int
    arrival: float  # seconds from the start of the run
    start: float = math.nan
    done: float = math.nan

    def nbytes(self) -> int:
        """Bytes the request holds while admitted (its own buffers)."""
        return lib.bk_serve_request_bytes(KINDS.index(self.kind), self.n)


def make_requests(count: int, rate: float, seed: int = 1000, lo: int = 1 << 10, hi: int = 1 << 24,
                  mix=(0.4, 0.3, 0.3)) -> list[Request]:
    """Poisson arrivals at `rate` req/s (rate = inf: all at t = 0); kinds drawn
    with probabilities `mix` (sort, rbk, scan); n log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    gaps = np.zeros(count) if math.isinf(rate) else rng.exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps) - (gaps[0] if count else 0)
    kinds = rng.choice(len(KINDS), size=count, p=np.asarray(mix) / np.sum(mix))
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)
    return [Request(i, KINDS[int(k)], int(n), float(a)) for i, (k, n, a) in enumerate(zip(kinds, sizes, arrivals))]


class Sources:
    """Pre-generated device inputs; a request's input is a window of one."""

    def __init__(self, n_max: int, device="cuda", seed: int = 7, rbk_mean_run: float = 32.0):
        g = torch.Generator(device=device)
        g.manual_seed(seed)
        self.n_max = n_max
        self.sort_keys = torch.randint(0, 1 << 32, (n_max,), generator=g, device=device, dtype=torch.int64).to(
            torch.uint32)
        heads = torch.rand(n_max, generator=g, device=device) < 1.0 / rbk_mean_run
        self.rbk_keys = torch.cumsum(heads.to(torch.int32), 0, dtype=torch.int32)
        self.rbk_vals = torch.rand(n_max, generator=g, device=device)
        self.scan_vals = torch.rand(n_max, generator=g, device=device) * 2 - 1
        self.sort_vals = torch.arange(n_max, device=device, dtype=torch.int64).to(torch.uint32)

    def offset(self, req: Request) -> int:
        """Start of the request's window: a multiple of 64 elements, so views
        keep the sources' 16-byte alignment (the kernels' TMA path)."""
        span = self.n_max - req.n + 1
        return (req.rid * 2654435761) % span // 64 * 64


class _Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("n", ctypes.c_uint64),
                ("src_offset", ctypes.c_uint64), ("arrival_s", ctypes.c_double)]


class _Record(ctypes.Structure):
    _fields_ = [("start_s", ctypes.c_double), ("done_s", ctypes.c_double), ("out", ctypes.c_uint64 * 3)]


class _Config(ctypes.Structure):
    _fields_ = [("sort_keys", ctypes.c_void_p), ("sort_vals", ctypes.c_void_p), ("rbk_keys", ctypes.c_void_p),
                ("rbk_vals", ctypes.c_void_p), ("scan_vals", ctypes.c_void_p), ("source_len", ctypes.c_uint64),
                ("pool", ctypes.c_void_p), ("pool_bytes", ctypes.c_uint64), ("ws", ctypes.c_void_p),
                ("ws_bytes", ctypes.c_uint64), ("budget_bytes", ctypes.c_uint64), ("stream", ctypes.c_void_p),
                ("mode", ctypes.c_int32), ("max_inflight", ctypes.c_int32), ("keep_buffers", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("timeout_s", ctypes.c_double)]


class _Stats(ctypes.Structure):
    _fields_ = [("makespan_s", ctypes.c_double), ("pool_high_water", ctypes.c_uint64), ("calls", ctypes.c_uint64),
                ("batches", ctypes.c_uint64)]


MODES = {"plain": 0, "batched": 1}


class Server:
    """Runs request streams through bk_serve_run over `sources`, with the
    requests' buffers in `pool`'s device buffer and at most `budget_bytes`
    of them admitted at once."""

    def __init__(self, sources: Sources, pool: DevicePool, budget_bytes: int, stream=None, keep_results=False):
        self.src = sources
        self.pool = pool
        self.budget = budget_bytes
        dev = _require_cuda(sources.sort_keys)
        self.stream = stream or torch.cuda.Stream(dev)
        self.keep = keep_results
        self.results: dict[int, tuple] = {}
        self._ws = None

    def _workspace(self, reqs_arr, count: int, mode: int):
        need = max(256, lib.bk_serve_workspace_bytes(ctypes.cast(reqs_arr, ctypes.c_void_p), count, mode))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.zeros(need, dtype=torch.uint8, device=self.pool.buf.device)
        return self._ws

    def run(self, requests: list[Request], mode: str, max_inflight: int = 2, timeout_s: float = 120.0) -> dict:
        """Serve `requests` (sorted by arrival) in `mode` ("plain" or "batched")."""
        pending = sorted(requests, key=lambda r: r.arrival)
        count = len(pending)
        arr = (_Request * max(count, 1))()
        for i, r in enumerate(pending):
            arr[i].kind, arr[i].n = KINDS.index(r.kind), r.n
            arr[i].src_offset, arr[i].arrival_s = self.src.offset(r), r.arrival
        recs = (_Record * max(count, 1))()
        ws = self._workspace(arr, count, MODES[mode])
        s = self.src
        cfg = _Config(s.sort_keys.data_ptr(), s.sort_vals.data_ptr(), s.rbk_keys.data_ptr(), s.rbk_vals.data_ptr(),
                      s.scan_vals.data_ptr(), s.n_max, self.pool.buf.data_ptr(), self.pool.capacity,
                      ws.data_ptr(), ws.numel(), self.budget, _stream_handle(self.stream, self.pool.buf.device),
                      MODES[mode], max_inflight, 1 if self.keep else 0, 0, timeout_s)
        stats = _Stats()
        torch.cuda.current_stream(self.pool.buf.device).synchronize()  # sources and buffers are ready
        check(lib.bk_serve_run(ctypes.byref(cfg), ctypes.cast(arr, ctypes.c_void_p), count,
                               ctypes.cast(recs, ctypes.c_void_p), ctypes.byref(stats)), "bk_serve_run")
        for i, r in enumerate(pending):
            r.start, r.done = recs[i].start_s, recs[i].done_s
            if self.keep:
                self.results[r.rid] = self._result(r, recs[i].out)
        lat = np.array([r.done - r.arrival for r in pending]) if count else np.zeros(1)
        return {"mode": mode, "requests": count, "makespan_s": stats.makespan_s, "latency_s": lat,
                "req_per_s": count / stats.makespan_s if stats.makespan_s > 0 else math.inf,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "pool_high_water_bytes": stats.pool_high_water, "calls": stats.calls, "batches": stats.batches}

    def _result(self, r: Request, out) -> tuple:
        v = self.pool.view
        if r.kind == "sort":
            return v(out[0], r.n, torch.uint32).clone(), v(out[1], r.n, torch.uint32).clone()
        if r.kind == "rbk":
            return (v(out[0], r.n, torch.int32).clone(), v(out[1], r.n, torch.float32).clone(),
                    v(out[2], 1, torch.int64).clone())
        return (v(out[0], r.n, torch.float32).clone(),)


def benchmark(saturation_requests: int = 600, rate: float = 2000.0, open_loop_s: float = 2.0, seed: int = 1000,
              lo: int = 1 << 10, hi: int = 1 << 24, budget_bytes: int = 32 << 30, device="cuda",
              open_loop_repeats: int = 3) -> dict:
    """Plain vs batched serving of the mixed request stream.

    saturation: `saturation_requests` requests all arriving at t = 0 (req/s is
    the throughput); open loop: Poisson arrivals at `rate` for `open_loop_s`
    seconds (latency percentiles at that load), `open_loop_repeats` times with
    the two modes alternating, each repeat on its own arrival sequence; the
    reported percentiles are over the latencies of all repeats together (the
    p99 of one short run is one of its few largest latencies, which moves by
    several percent from run to run).  Both modes serve the same requests,
    after one warm-up run each."""
    src = Sources(hi, device=device)
    pool = DevicePool(min(budget_bytes, 24 << 30) + (1 << 24), device=device)
    out = {"config": {"mix": "40% sort_by_key u32/u32, 30% reduce_by_key i32/f32 (runs mean 32), 30% scan f32",
                      "sizes": f"log-uniform [{lo}, {hi}]", "rate_req_s": rate, "budget_bytes": budget_bytes,
                      "saturation_requests": saturation_requests, "open_loop_s": open_loop_s,
                      "open_loop_repeats": open_loop_repeats}}
    modes = ("plain", "batched")
    servers = {mode: Server(src, pool, budget_bytes) for mode in modes}
    for mode in modes:
        server = servers[mode]
        server.run(make_requests(64, math.inf, seed + 1, lo, hi), mode)  # warm-up (workspaces, kernels)
        torch.cuda.synchronize()
        sat = server.run(make_requests(saturation_requests, math.inf, seed, lo, hi), mode)
        torch.cuda.synchronize()
        out[mode] = {"saturation_req_s": sat["req_per_s"], "saturation_p99_ms": sat["p99_ms"],
                     "saturation_calls": sat["calls"], "saturation_batches": sat["batches"]}
    runs = {mode: [] for mode in modes}
    for r in range(max(1, open_loop_repeats)):
        reqs = max(1, int(rate * open_loop_s))
        for mode in modes:
            runs[mode].append(servers[mode].run(make_requests(reqs, rate, seed + 2 + r, lo, hi), mode))
            torch.cuda.synchronize()
    for mode in modes:
        lat = np.concatenate([o["latency_s"] for o in runs[mode]])
        out[mode].update({
            "open_loop_p50_ms": float(np.percentile(lat, 50) * 1e3),
            "open_loop_p99_ms": float(np.percentile(lat, 99) * 1e3),
            "open_loop_req_s": float(np.median([o["req_per_s"] for o in runs[mode]])),
            "open_loop_requests": int(lat.size),
            "open_loop_p99_runs_ms": [o["p99_ms"] for o in runs[mode]]})
    out["batched_over_plain_req_s"] = out["batched"]["saturation_req_s"] / out["plain"]["saturation_req_s"]
    return out
