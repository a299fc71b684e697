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
pre-generated source array of its kind, so it depends only on the id.  Scan
and reduce_by_key read their window in place; a sort copies its keys and
payload into its own buffers.  Outputs and sort buffers come from a pooled
device allocator; admission keeps the bytes of admitted, unfinished requests
within an HBM budget.

``plain`` issues every admitted request as its own call (bk_* single-array
entry points) on one stream, in arrival order.  ``batched`` gathers all
admitted requests that have arrived, groups them by kind and issues one
batched call per kind (bk_*_batch), keeping at most ``max_inflight`` batches
queued on the stream; a request completes when its call's event does.
Latency = completion time - arrival time, on the host's clock.
"""
from __future__ import annotations

import bisect
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import algorithms, batch
from .algorithms import inclusive_scan, reduce_by_key, stable_sort_by_key

KINDS = ("sort", "rbk", "scan")


# --------------------------------------------------------------------------
class DevicePool:
    """Pooled allocator over one preallocated byte buffer: first-fit over an
    address-ordered free list, 256-byte granules, neighbours coalesced on
    free.  Allocation never calls into the CUDA allocator."""

    ALIGN = 256

    def __init__(self, capacity: int, device="cuda"):
        self.capacity = capacity // self.ALIGN * self.ALIGN
        self.buf = torch.empty(self.capacity, dtype=torch.uint8, device=device)
        self._free = [(0, self.capacity)]  # (offset, size), sorted by offset
        self._used: dict[int, int] = {}
        self.in_use = 0
        self.high_water = 0

    def alloc(self, nbytes: int) -> int | None:
        need = max(self.ALIGN, -(-nbytes // self.ALIGN) * self.ALIGN)
        for i, (off, size) in enumerate(self._free):
            if size >= need:
                if size == need:
                    del self._free[i]
                else:
                    self._free[i] = (off + need, size - need)
                self._used[off] = need
                self.in_use += need
                self.high_water = max(self.high_water, self.in_use)
                return off
        return None

    def free(self, off: int) -> None:
        size = self._used.pop(off)
        self.in_use -= size
        i = bisect.bisect_left(self._free, (off, 0))
        self._free.insert(i, (off, size))
        # coalesce with the right, then the left neighbour
        if i + 1 < len(self._free) and off + size == self._free[i + 1][0]:
            self._free[i] = (off, size + self._free[i + 1][1])
            del self._free[i + 1]
        if i > 0 and self._free[i - 1][0] + self._free[i - 1][1] == off:
            self._free[i - 1] = (self._free[i - 1][0], self._free[i - 1][1] + self._free[i][1])
            del self._free[i]

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
    allocs: list = field(default_factory=list)
    tensors: dict = field(default_factory=dict)
    start: float = math.nan
    done: float = math.nan
    event: torch.cuda.Event | None = None

    def nbytes(self) -> int:
        # the request's own buffers (sort: keys and payload; rbk: outputs and
        # the count word; scan: output); workspaces are shared per stream
        return {"sort": 8, "rbk": 8, "scan": 4}[self.kind] * self.n + 512


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


class Server:
    def __init__(self, sources: Sources, pool: DevicePool, budget_bytes: int, stream=None, keep_results=False):
        self.src = sources
        self.pool = pool
        self.budget = budget_bytes
        self.admitted_bytes = 0
        self.stream = stream or torch.cuda.Stream()
        self.keep = keep_results
        self.results: dict[int, tuple] = {}

    # ---- memory
    def _admit(self, req: Request) -> bool:
        # over budget: wait -- unless nothing is admitted (a request larger
        # than the whole budget still runs, alone)
        if self.admitted_bytes > 0 and self.admitted_bytes + req.nbytes() > self.budget:
            return False
        # the request's own buffers: slot -> (dtype, elements)
        sizes = {"sort": {0: (torch.uint32, req.n), 1: (torch.uint32, req.n)},
                 "rbk": {2: (torch.int32, req.n), 3: (torch.float32, req.n), 4: (torch.int64, 1)},
                 "scan": {1: (torch.float32, req.n)}}[req.kind]
        offs, tensors = [], {}
        for slot, (dt, n) in sizes.items():
            off = self.pool.alloc(n * torch.empty(0, dtype=dt).element_size())
            if off is None:
                for o in offs:
                    self.pool.free(o)
                return False
            offs.append(off)
            tensors[slot] = self.pool.view(off, n, dt)
        # inputs read in place: windows of the sources
        o, n = self.src.offset(req), req.n
        if req.kind == "rbk":
            tensors[0], tensors[1] = self.src.rbk_keys[o:o + n], self.src.rbk_vals[o:o + n]
        elif req.kind == "scan":
            tensors[0] = self.src.scan_vals[o:o + n]
        req.allocs, req.tensors = offs, tensors
        self.admitted_bytes += req.nbytes()
        return True

    def _release(self, req: Request) -> None:
        if self.keep:
            t = req.tensors
            if req.kind == "sort":
                self.results[req.rid] = (t[0].clone(), t[1].clone())
            elif req.kind == "rbk":
                self.results[req.rid] = (t[2].clone(), t[3].clone(), t[4].clone())
            else:
                self.results[req.rid] = (t[1].clone(),)
        for o in req.allocs:
            self.pool.free(o)
        req.allocs, req.tensors = [], {}
        self.admitted_bytes -= req.nbytes()

    def _stage(self, req: Request) -> None:
        """A sort copies its input window into its own buffers (on the stream)."""
        if req.kind == "sort":
            o, n, t = self.src.offset(req), req.n, req.tensors
            t[0].copy_(self.src.sort_keys[o:o + n], non_blocking=True)
            t[1].copy_(self.src.sort_vals[o:o + n], non_blocking=True)

    # ---- issue
    def _issue_one(self, req: Request) -> None:
        t = req.tensors
        if req.kind == "sort":
            stable_sort_by_key(t[0], t[1], stream=self.stream)
        elif req.kind == "rbk":
            reduce_by_key(t[0], t[1], t[2], t[3], t[4], stream=self.stream, sync=False)
        else:
            inclusive_scan(t[0], 0.0, out=t[1], stream=self.stream)

    def _issue_batch(self, kind: str, reqs: list[Request]) -> None:
        ts = [r.tensors for r in reqs]
        if kind == "sort":
            batch.stable_sort_by_key_batch([t[0] for t in ts], [t[1] for t in ts], stream=self.stream)
        elif kind == "rbk":
            batch.reduce_by_key_batch([t[0] for t in ts], [t[1] for t in ts], stream=self.stream,
                                      outs=[(t[2], t[3], t[4]) for t in ts])
        else:
            batch.inclusive_scan_batch([t[0] for t in ts], [0.0] * len(ts), [t[1] for t in ts], stream=self.stream)

    # ---- run
    def run(self, requests: list[Request], mode: str, max_inflight: int = 2, timeout_s: float = 120.0) -> dict:
        """Serve `requests` (sorted by arrival) in `mode` ("plain" or "batched")."""
        pending = sorted(requests, key=lambda r: r.arrival)
        nxt = 0            # next request not yet admitted
        waiting: list[Request] = []   # arrived and admitted, not issued (batched mode)
        inflight: list[tuple[torch.cuda.Event, list[Request]]] = []
        done = 0
        t0 = time.perf_counter()
        with torch.cuda.stream(self.stream):
            while done < len(pending):
                now = time.perf_counter() - t0
                if now > timeout_s:
                    raise TimeoutError(f"serving run exceeded {timeout_s} s")
                # completions (in stream order)
                while inflight and inflight[0][0].query():
                    ev, reqs = inflight.pop(0)
                    tdone = time.perf_counter() - t0
                    for r in reqs:
                        r.done = tdone
                        self._release(r)
                        done += 1
                # arrivals and admission, in arrival order
                now = time.perf_counter() - t0
                while nxt < len(pending) and pending[nxt].arrival <= now and self._admit(pending[nxt]):
                    r = pending[nxt]
                    nxt += 1
                    if mode == "plain":
                        r.start = now
                        self._stage(r)
                        self._issue_one(r)
                        ev = torch.cuda.Event()
                        ev.record(self.stream)
                        inflight.append((ev, [r]))
                    else:
                        waiting.append(r)
                if mode == "batched" and waiting and len(inflight) < max_inflight:
                    by_kind: dict[str, list[Request]] = {}
                    for r in waiting:
                        by_kind.setdefault(r.kind, []).append(r)
                    issued = []
                    for kind, reqs in by_kind.items():
                        for lo in range(0, len(reqs), batch.BATCH_MAX):
                            chunk = reqs[lo:lo + batch.BATCH_MAX]
                            for r in chunk:
                                r.start = now
                                self._stage(r)
                            self._issue_batch(kind, chunk)
                            issued.extend(chunk)
                    ev = torch.cuda.Event()
                    ev.record(self.stream)
                    inflight.append((ev, issued))
                    waiting = []
        makespan = time.perf_counter() - t0
        lat = np.array([r.done - r.arrival for r in pending])
        return {"mode": mode, "requests": len(pending), "makespan_s": makespan,
                "req_per_s": len(pending) / makespan if makespan > 0 else math.inf,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "pool_high_water_bytes": self.pool.high_water}


def benchmark(saturation_requests: int = 600, rate: float = 2000.0, open_loop_s: float = 1.0, seed: int = 1000,
              lo: int = 1 << 10, hi: int = 1 << 24, budget_bytes: int = 32 << 30, device="cuda") -> dict:
    """Plain vs batched serving of the mixed request stream.

    saturation: `saturation_requests` requests all arriving at t = 0 (req/s is
    the throughput); open loop: Poisson arrivals at `rate` for `open_loop_s`
    seconds (latency percentiles at that load).  Both modes serve the same
    requests, after one warm-up run each."""
    src = Sources(hi, device=device)
    pool = DevicePool(min(budget_bytes, 24 << 30) + (1 << 24), device=device)
    out = {"config": {"mix": "40% sort_by_key u32/u32, 30% reduce_by_key i32/f32 (runs mean 32), 30% scan f32",
                      "sizes": f"log-uniform [{lo}, {hi}]", "rate_req_s": rate, "budget_bytes": budget_bytes,
                      "saturation_requests": saturation_requests, "open_loop_s": open_loop_s}}
    for mode in ("plain", "batched"):
        server = Server(src, pool, budget_bytes)
        server.run(make_requests(64, math.inf, seed + 1, lo, hi), mode)  # warm-up (workspaces, kernels)
        torch.cuda.synchronize()
        sat = server.run(make_requests(saturation_requests, math.inf, seed, lo, hi), mode)
        torch.cuda.synchronize()
        ol = server.run(make_requests(max(1, int(rate * open_loop_s)), rate, seed + 2, lo, hi), mode)
        torch.cuda.synchronize()
        out[mode] = {"saturation_req_s": sat["req_per_s"], "saturation_p99_ms": sat["p99_ms"],
                     "open_loop_p50_ms": ol["p50_ms"], "open_loop_p99_ms": ol["p99_ms"],
                     "open_loop_req_s": ol["req_per_s"]}
    out["batched_over_plain_req_s"] = out["batched"]["saturation_req_s"] / out["plain"]["saturation_req_s"]
    return out
