"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the step time
is the slowest rank's, the value counts every rank's bytes, and the
reference arm runs on rank 0 only.  The workload itself is replicas only (one
independent copy per GPU, no collective on the data path)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms, value = bench.whole_job(1.0 + rank, 6e9, world, device="cpu")
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_whole_job_takes_the_slowest_rank_and_counts_every_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for _, ms, value in got:
        assert ms == 2.0  # max over ranks of 1.0 and 2.0
        assert abs(value - 6e9 * world / 2e-3 / 1e9) < 1e-6


def test_whole_job_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.whole_job(4.0, 8e9, 1) == (4.0, 8e9 / 4e-3 / 1e9)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line_keeps_the_contract():
    """Rank 0's line, on a small n here (the real arm runs the 2^28 workload)."""
    sys.path.insert(0, str(ROOT))
    import bench
    line = bench.cpu_reference_line(1, 1, n=1 << 20)
    json.dumps(line)
    assert line["impl"] == "reference" and line["unit"] == "GB/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


def test_cpu_baseline_object_reports_all_cores_and_one_thread(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    calls = []

    def fake(n, steps, warmup, threads):
        calls.append((n, threads))
        return 0.5, "reference", steps
    monkeypatch.setattr(bench, "cpu_reference_time", fake)
    cb = bench.cpu_baseline_object()
    assert cb["cores"] == (os.cpu_count() or 1) and cb["one_thread"]["cores"] == 1
    assert calls == [(1 << 26, os.cpu_count() or 1), (1 << 24, 1)]
    # bytes per element: reduce N*s + scan 2*N*s for s = 4, 8, 4
    assert cb["value"] == 48 * (1 << 26) / 0.5 / 1e9 and cb["cpu_model"]
