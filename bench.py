#!/usr/bin/env python
"""Benchmark of the device-wide algorithm path on B200.

Headline workload (one "step"): sum-reduce and inclusive sum-scan over
N = 2^28 elements of each of float32 U[-1,1], float64 U[-1,1] and int32
U[-100,100] -- six library calls per step.  The inputs (1 + 2 + 1 GiB) are
larger than L2, so no flush is needed between steps.

value  = algorithmic bytes per step (reduce N*s, scan 2*N*s) / device time,
         whole job over all ranks (each rank runs the same workload on its own
         GPU: replicas, weak scaling).
e2e    = the same through the C-ABI with host buffers: pinned-host -> device
         copies of the step's inputs and device -> host copies of every result
         inside the timed region (in chunks of 2^25 elements on two streams,
         each chunk's scan starting from the previous chunk's last output on
         the device, so copies in the two directions overlap).
ops    = per-op GB/s: the headline's six calls, and the other benchmark
         configurations (merge_by_key 2 x 2^26 f32/u32, stable sort_by_key
         2^26 u32/u64 keys with u32 payload, reduce_by_key 2^27 i32 keys with
         geometric / Zipf runs and f32 / f64 values), timed after the headline.

serving = plain vs batched serving of a mixed request stream (the native loop
         bk_serve_run, driven by bulk_b200/serve.py: 40% sort_by_key u32/u32, 30% reduce_by_key i32/f32, 30% scan f32;
         sizes log-uniform in [2^10, 2^24], and a small-request variant in
         [2^10, 2^16]): saturation req/s and, at 2000 req/s Poisson arrivals
         for 2 s, p50/p99 latency (over the latencies of 3 repeats with the
         modes alternating), for one call per request ("plain") and
         continuous batching ("batched"); rank 0 only.

``--impl reference`` times the reference's CPU implementation of the same
reduce + scan on the host cores instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "effective GB/s & %HBM peak per op at 2^26-2^28; batched req/s + p99 vs plain"
WORKLOAD = "reduce+inclusive_scan sum, N=2^28, f32 U[-1,1] + f64 U[-1,1] + i32 U[-100,100]"
N_HEADLINE = 1 << 28
DTYPES = [("f32", 4), ("f64", 8), ("i32", 4)]


def _traffic_per_unit(kernel_case):
    """DRAM bytes per element of a kernel, from the committed ncu summary
    (profiles/ncu_traffic.json: dram__bytes_read.sum + dram__bytes_write.sum of
    one captured launch on a smaller case, divided by its elements; traffic
    grows in proportion to the elements for these streaming kernels)."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None, None
    d = json.loads(p.read_text())
    e = d.get(kernel_case)
    if not e:
        return None, None
    return e["dram_bytes_per_unit"], e["case"]


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def whole_job(ms_step, bytes_step, world, device=None):
    """(ms per step, whole-job GB/s): the step time is the slowest rank's (a
    MAX all-reduce when world > 1, so every rank must call it), and every rank
    processed bytes_step per step."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms_step], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    return ms_step, bytes_step * world / (ms_step * 1e-3) / 1e9


def _env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return None
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                rows.append((float(c[1]), float(c[2]), c[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
def run_reference(args):
    """CPU reference arm: the reference's reduce + scan on all host cores,
    over the full headline workload (N = 2^28 of each dtype)."""
    rank, world, _ = _env_rank()
    if rank != 0:
        return 0
    line = cpu_reference_line(args.steps, args.warmup, args.n)
    print(json.dumps(line), flush=True)
    return 0


def cpu_model() -> str:
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_time(n_sample: int, steps: int, warmup: int, threads: int):
    """Median seconds per step of reduce + scan over n_sample elements of each
    dtype, and which implementation ran ("reference": the reference's own
    algorithms compiled for the host, oracle/_ref; else "port": the oracle's
    threaded restatement)."""
    import ctypes

    import numpy as np

    import oracle  # CPU baseline leg only
    from oracle import reference as R
    data = [oracle.gen(np.float32, n_sample, 0, -1.0, 1.0), oracle.gen(np.float64, n_sample, 0, -1.0, 1.0),
            oracle.gen(np.int32, n_sample, 0, -100, 100)]
    outs = [np.empty_like(x) for x in data]
    if R.available():
        kind = "reference"

        def step():
            for x, o in zip(data, outs):
                R.cpu_reduce(x, x.dtype.type(0), threads)
                R.cpu_inclusive_scan(x, x.dtype.type(0), threads, out=o)
    else:
        kind = "port"
        olib = oracle._lib
        red = olib.bko_baseline_reduce
        red.restype = ctypes.c_double
        red.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        scn = olib.bko_baseline_inclusive_scan
        scn.restype = None
        scn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]

        def step():
            for t, (x, o) in enumerate(zip(data, outs)):
                red(x.ctypes.data, x.size, t, threads)
                scn(x.ctypes.data, o.ctypes.data, x.size, t, threads)

    for _ in range(warmup):
        step()
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    return statistics.median(times), kind, len(times)


def cpu_reference_line(steps, warmup, n=N_HEADLINE):
    """The reference arm: every step is the whole headline workload (reduce +
    inclusive_scan over n elements of each of f32 / f64 / i32) on all host
    cores; value from the median step time."""
    threads = os.cpu_count() or 1
    steps = max(1, min(steps, 10))
    sec, kind, steps = cpu_reference_time(n, steps, max(1, min(warmup, 3)), threads)
    bytes_per = sum(3 * n * s for _, s in DTYPES)
    gbs = bytes_per / sec / 1e9
    what = ("the reference's agent-level reduce / inclusive_scan compiled for the host, over the drivers' "
            "partitioning (reduce.cu, scan.cu)" if kind == "reference" else "the oracle's threaded restatement")
    sample = (f"the full workload: reduce+inclusive_scan over {n} elements of each of f32/f64/i32, "
              f"{threads} threads ({cpu_model()}), {what}; median of {steps} steps")
    return {"metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": 0, "steps": steps, "warmup": warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64+i32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "n": n, "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind, "cpu_model": cpu_model(),
                             "sample": sample},
            "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline_object():
    """The repo arm's cpu_baseline: the reference compiled for the host on all
    host cores over a 2^26-element sample of each dtype (about 0.1-0.3 s per
    step, median of 5), plus a 1-thread run over a 2^24-element sample."""
    threads = os.cpu_count() or 1
    n_all, n_one = 1 << 26, 1 << 24
    sec, kind, steps = cpu_reference_time(n_all, 5, 1, threads)
    sec1, _, steps1 = cpu_reference_time(n_one, 3, 1, 1)
    per_elem = sum(3 * s for _, s in DTYPES)
    gbs, gbs1 = per_elem * n_all / sec / 1e9, per_elem * n_one / sec1 / 1e9
    return {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind, "cpu_model": cpu_model(),
            "sample": (f"reduce+inclusive_scan over 2^26 elements of each of f32/f64/i32 (1/4 of the 2^28 "
                       f"workload; GB/s is per byte, so it compares), {threads} threads, median of {steps} steps"),
            "one_thread": {"value": gbs1, "unit": "GB/s", "cores": 1,
                           "sample": f"the same over 2^24 elements of each dtype, 1 thread, median of {steps1} steps"}}


# --------------------------------------------------------------------------
def make_inputs(device, n):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(0)
    xs = {
        "f32": torch.rand(n, generator=g, device=device, dtype=torch.float32) * 2 - 1,
        "f64": torch.rand(n, generator=g, device=device, dtype=torch.float64) * 2 - 1,
        "i32": torch.randint(-100, 101, (n,), generator=g, device=device, dtype=torch.int32),
    }
    return xs


def headline(args, device, rank, world):
    import torch
    import torch.distributed as dist

    import bulk_b200

    n = args.n
    xs = make_inputs(device, n)
    outs = {k: torch.empty_like(v) for k, v in xs.items()}
    reds = {k: torch.empty(1, dtype=v.dtype, device=device) for k, v in xs.items()}
    stream = torch.cuda.current_stream(device)
    # per-call events, recorded on the launching stream
    ev = {(k, op): [] for k, _ in DTYPES for op in ("reduce", "scan")}

    def step(record):
        for k, _ in DTYPES:
            if record:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
            bulk_b200.reduce(xs[k], 0, out=reds[k])
            if record:
                b.record(stream)
                ev[(k, "reduce")].append((a, b))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
            bulk_b200.inclusive_scan(xs[k], 0, out=outs[k])
            if record:
                b.record(stream)
                ev[(k, "scan")].append((a, b))

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    if bulk_b200.workspace_status() != 0:
        raise RuntimeError("device-side error during warm-up")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        _queue_ahead(1000)
        start.record(stream)
        for _ in range(args.steps):
            step(True)
        end.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = start.elapsed_time(end)
    if bulk_b200.workspace_status() != 0:
        raise RuntimeError("device-side error during the timed region")
    per = {key: statistics.mean(a.elapsed_time(b) for a, b in lst) for key, lst in ev.items()}
    return ms, per, clk.summary(), xs


E2E_CHUNK = 1 << 25  # elements per copy chunk of the end-to-end leg


def e2e(args, device, xs):
    """Same workload through the public API with host buffers (pinned), copies timed.

    A two-stream pipeline over chunks of E2E_CHUNK elements: one stream copies
    every array to the device chunk by chunk; the other waits for each chunk,
    scans it starting from the previous chunk's last output (read on the
    device: inclusive_scan with a device-tensor init), copies the chunk's
    output back, and reduces each array once its last chunk is in.  So copies
    to the device and copies back (separate copy engines) overlap for the
    whole step, not just between arrays."""
    import torch

    import bulk_b200
    stream = torch.cuda.current_stream(device)
    up, down = torch.cuda.Stream(device), torch.cuda.Stream(device)
    h_in = {k: v.cpu().pin_memory() for k, v in xs.items()}
    h_scan = {k: torch.empty_like(v, device="cpu").pin_memory() for k, v in xs.items()}
    h_red = {k: torch.empty(1, dtype=v.dtype).pin_memory() for k, v in xs.items()}
    d_in = {k: torch.empty_like(v) for k, v in xs.items()}
    d_out = {k: torch.empty_like(v) for k, v in xs.items()}
    d_red = {k: torch.empty(1, dtype=v.dtype, device=device) for k, v in xs.items()}
    h2d = sum(v.numel() * v.element_size() for v in h_in.values())
    d2h = sum(v.numel() * v.element_size() for v in h_scan.values()) + sum(v.element_size() for v in h_red.values())
    chunks = [(k, lo, min(xs[k].numel(), lo + E2E_CHUNK)) for k, _ in DTYPES
              for lo in range(0, xs[k].numel(), E2E_CHUNK)]
    arrived = [torch.cuda.Event() for _ in chunks]

    def step():
        # this step's copies overwrite the inputs the previous step's scans read
        up.wait_stream(down)
        with torch.cuda.stream(up):
            for (k, lo, hi), ev in zip(chunks, arrived):
                d_in[k][lo:hi].copy_(h_in[k][lo:hi], non_blocking=True)
                ev.record(up)
        with torch.cuda.stream(down):
            for (k, lo, hi), ev in zip(chunks, arrived):
                down.wait_event(ev)
                init = 0 if lo == 0 else d_out[k][lo - 1:lo]
                bulk_b200.inclusive_scan(d_in[k][lo:hi], init, out=d_out[k][lo:hi], stream=down)
                h_scan[k][lo:hi].copy_(d_out[k][lo:hi], non_blocking=True)
                if hi == xs[k].numel():
                    bulk_b200.reduce(d_in[k], 0, out=d_red[k], stream=down)
                    h_red[k].copy_(d_red[k], non_blocking=True)

    steps = max(1, min(args.steps, args.e2e_steps))
    for _ in range(min(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    up.wait_event(a)
    down.wait_event(a)
    for _ in range(steps):
        step()
    stream.wait_stream(up)
    stream.wait_stream(down)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, h2d, d2h, steps


def _queue_ahead(us=300):
    """Occupy the GPU for about `us` microseconds (a spin kernel) so that the
    host has queued the timed calls before the start event is reached: the
    timed region then holds device time only, not the host's first launch."""
    import torch
    torch.cuda._sleep(int(us * 2000))


def _time_op(fn, prep=None, reps=5, warm=2):
    """Mean device time (ms) of fn() over reps, CUDA events on the current
    stream; prep() (untimed) runs before each call."""
    import torch
    stream = torch.cuda.current_stream()
    for _ in range(warm):
        if prep:
            prep()
        fn()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(reps):
        if prep:
            prep()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _queue_ahead()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    return tot / reps


def _geometric_runs(n, mean, g, device):
    """i32 run-index keys with run lengths 1 + Geometric(1/mean), truncated to n elements."""
    import torch
    p = 1.0 / mean
    m = int(n / mean * 1.1) + 1024
    while True:
        u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
        lens = 1 + torch.floor(torch.log1p(-u) / math.log1p(-p)).to(torch.int64)
        if int(lens.sum()) >= n:
            break
        m *= 2
    keys = torch.repeat_interleave(torch.arange(m, device=device, dtype=torch.int32), lens)
    return keys[:n].contiguous()


def _zipf_runs(n, s_exp, cap, g, device):
    """i32 run-index keys whose run lengths are Zipf(s_exp)-like (a bounded
    Pareto draw, rounded down) capped at cap, truncated to n elements."""
    import torch
    a = 1.0 - s_exp
    top = (cap + 1.0) ** a - 1.0
    m = max(1024, n // 64)
    while True:
        u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
        lens = torch.floor((1.0 + u * top) ** (1.0 / a)).clamp(1, cap).to(torch.int64)
        csum = torch.cumsum(lens, 0)
        if int(csum[-1]) >= n:
            break
        m *= 2
    r = int(torch.searchsorted(csum, torch.tensor([n], device=device, dtype=torch.int64)).item()) + 1
    lens = lens[:r].clone()
    lens[-1] -= int(csum[r - 1]) - n
    keys = torch.repeat_interleave(torch.arange(r, device=device, dtype=torch.int32), lens)
    return keys


def other_ops(device, peak, quick=False, shift=0):
    """Per-op effective GB/s at the other benchmark configurations (sizes / 2^shift)."""
    import torch

    import bulk_b200
    g = torch.Generator(device=device)
    g.manual_seed(1)
    res = {}
    reps = 3 if quick else 5

    # merge_by_key: A, B = 2^26 float32 U[0,1) each (~1% cross duplicates), u32 payloads
    n = 1 << (26 - shift)
    a = torch.sort(torch.rand(n, generator=g, device=device)).values
    b = torch.rand(n, generator=g, device=device)
    idx = torch.randint(0, n, (n // 100,), generator=g, device=device)
    b[idx] = a[torch.randint(0, n, (n // 100,), generator=g, device=device)]
    b = torch.sort(b).values
    av = torch.arange(n, dtype=torch.int32, device=device)
    bv = av + n
    ok = torch.empty(2 * n, dtype=torch.float32, device=device)
    ov = torch.empty(2 * n, dtype=torch.int32, device=device)
    ms = _time_op(lambda: bulk_b200.merge(a, b, av, bv, out=ok, out_vals=ov), reps=reps)
    byts = 2 * (2 * n) * 8
    res[f"merge_by_key_f32_u32_2x2^{26 - shift}"] = {"ms": ms, "GBps": byts / ms / 1e6, "frac_of_hbm": byts / ms / 1e6 / peak,
                                          "algorithmic_bytes": byts}
    del a, b, av, bv, ok, ov

    # stable sort_by_key: 2^26 u32 keys (full range) / 2^26 u64 keys, payload = index
    for tag in ("u32", "u64"):
        if tag == "u32":
            k0 = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=device,
                               dtype=torch.int32).view(torch.uint32)
        else:
            hi = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=device, dtype=torch.int32)
            lo = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=device, dtype=torch.int32)
            k0 = ((hi.to(torch.int64) << 32) | (lo.to(torch.int64) & 0xFFFFFFFF)).view(torch.uint64)
            del hi, lo
        v0 = torch.arange(n, dtype=torch.int32, device=device)
        k, v = k0.clone(), v0.clone()

        def prep():
            k.copy_(k0)
            v.copy_(v0)
        ms = _time_op(lambda: bulk_b200.stable_sort_by_key(k, v), prep=prep, reps=reps)
        ksz = k0.element_size()
        byts = 2 * n * (ksz + 4)
        # LSD radix: one pass per key byte; a pass reads the keys (digit
        # counts), then reads and writes keys and payloads (scatter), plus the
        # digit counts (n / 4096 tiles x 256 u32) written, scanned and read
        passes = ksz
        counts = (n + 4095) // 4096 * 256 * 4
        moved = passes * (n * ksz + 2 * n * (ksz + 4) + 4 * counts)
        res[f"sort_by_key_{tag}_u32_2^{26 - shift}"] = {
            "ms": ms, "GBps": byts / ms / 1e6, "frac_of_hbm": byts / ms / 1e6 / peak, "algorithmic_bytes": byts,
            "radix_passes": passes,
            "bytes_moved_by_design": moved,
            "GBps_of_bytes_moved": moved / ms / 1e6,
            "frac_of_hbm_by_design": moved / ms / 1e6 / peak}
        del k0, v0, k, v

    # reduce_by_key: 2^27 pairs, i32 keys in runs (geometric mean 16 / Zipf 1.2 cap 2^20), f32/f64 U[0,1)
    n = 1 << (27 - shift)
    for kind in ("geometric", "zipf"):
        keys = _geometric_runs(n, 16.0, g, device) if kind == "geometric" else _zipf_runs(n, 1.2, 1 << 20, g, device)
        for vt, dt in (("f32", torch.float32), ("f64", torch.float64)):
            vals = torch.rand(n, generator=g, device=device, dtype=dt)
            ok = torch.empty(n, dtype=torch.int32, device=device)
            ov = torch.empty(n, dtype=dt, device=device)
            cnt = torch.empty(1, dtype=torch.int64, device=device)
            ms = _time_op(lambda: bulk_b200.reduce_by_key(keys, vals, ok, ov, cnt, sync=False), reps=reps)
            u = int(cnt.item())
            sv = vals.element_size()
            byts = n * (4 + sv) + u * (4 + sv) + 8
            res[f"reduce_by_key_i32_{vt}_{kind}_2^{27 - shift}"] = {"ms": ms, "GBps": byts / ms / 1e6,
                                                          "frac_of_hbm": byts / ms / 1e6 / peak,
                                                          "algorithmic_bytes": byts, "runs": u}
            del vals, ok, ov, cnt
        del keys
    torch.cuda.empty_cache()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_HEADLINE, help=argparse.SUPPRESS)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-ops", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--ops-shift", type=int, default=0, help=argparse.SUPPRESS)
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    import bulk_b200  # noqa: F401  (fails loudly without the CUDA library)

    ms, per, clocks, xs = headline(args, device, rank, world)
    n = args.n
    bytes_step = sum(3 * n * s for _, s in DTYPES)
    ms_step, value = whole_job(ms / args.steps, bytes_step, world, device)
    peak, peak_kind = _peaks()

    # dominant kernel: the call with the largest mean time
    algo_bytes = {(k, "reduce"): n * s for k, s in DTYPES}
    algo_bytes.update({(k, "scan"): 2 * n * s for k, s in DTYPES})
    dom = max(per, key=per.get)
    ops = {f"{op}_{k}": {"GBps": algo_bytes[(k, op)] / (per[(k, op)] * 1e-3) / 1e9,
                         "ms": per[(k, op)],
                         "frac_of_hbm": algo_bytes[(k, op)] / (per[(k, op)] * 1e-3) / 1e9 / peak}
           for (k, op) in per}
    e2e_ms, h2d, d2h, e2e_steps = e2e(args, device, xs)
    del xs
    torch.cuda.empty_cache()
    if not args.no_other_ops:
        ops.update(other_ops(device, peak, shift=args.ops_shift))

    line = None
    if rank == 0:
        achieved = algo_bytes[dom] / (per[dom] * 1e-3) / 1e9
        tcase = {("f32", "scan"): "scan_kernel_0", ("f64", "scan"): "scan_kernel_1", ("i32", "reduce"): "reduce_kernel_2"}
        bpu, tsrc = _traffic_per_unit(tcase.get(dom, ""))
        traffic = bpu * n if bpu is not None else None
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64+i32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "calls_per_step": 6, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (1-2 GiB per array), no flush"},
            "frac_of_hbm_peak": value / world / peak,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": f"{dom[1]}_{dom[0]}", "algorithmic_bytes_per_launch": algo_bytes[dom],
                         "traffic": traffic,
                         "traffic_source": (f"profiles/ncu_traffic.json ({tsrc}), scaled to {n} elements"
                                            if traffic is not None else None)},
            "ops": ops,
            "e2e": {"value": bytes_step / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": e2e_steps},
            "gpu_launches": args.steps * 9,
            "clocks": clocks,
        }
    if rank == 0 and not args.no_serving:
        from bulk_b200 import serve
        sv = serve.benchmark(saturation_requests=600, rate=2000.0, open_loop_s=2.0, open_loop_repeats=3)
        small = serve.benchmark(saturation_requests=2000, rate=2000.0, open_loop_s=2.0, open_loop_repeats=3,
                                hi=1 << 16)
        line["serving"] = {"mix_2^10_2^24": sv, "mix_2^10_2^16": small}
        torch.cuda.empty_cache()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline_object()
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
