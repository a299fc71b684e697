"""The serving loop (bk_serve_run in libbulkb200.so, driven by
bulk_b200/serve.py): pooled allocator, request stream, workspace bound,
plain vs batched serving, and the alone-vs-in-mix parity of results.

The allocator (host bookkeeping only), the workspace bound and the request
generator run without a GPU; the serving runs need one.  Parity: a request's sort result (keys and payload), its
reduce_by_key keys and count are bit-identical whether it ran alone or inside
a batch; float sums and scan prefixes agree within the suite's bound
2*ceil(log2 n)*eps*sum|x| (twice, since both sides carry that error).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest
import torch

import bulk_b200
from bulk_b200 import _lib, serve
from bulk_b200.batch import batch_workspace_bytes


def test_pool_first_fit_coalesces_and_tracks_use():
    pool = serve.DevicePool(1 << 20, device="cpu")
    rng = np.random.default_rng(0)
    live = {}
    for step in range(2000):
        if live and (rng.random() < 0.5 or len(live) > 40):
            off = rng.choice(list(live))
            pool.free(off)
            del live[off]
        else:
            n = int(rng.integers(1, 40000))
            off = pool.alloc(n)
            if off is None:
                continue
            assert off % 256 == 0
            # no overlap with any live block
            for o, m in live.items():
                assert off + n <= o or o + m <= off
            live[off] = n
    for off in list(live):
        pool.free(off)
    assert pool.in_use == 0 and pool.free_blocks() == 1
    assert pool.high_water > 0


def test_pool_refuses_when_full_and_views_alias_the_buffer():
    pool = serve.DevicePool(4096, device="cpu")
    a = pool.alloc(3000)
    assert pool.alloc(2000) is None  # only 1024 bytes left
    v = pool.view(a, 10, torch.int32)
    v[:] = 7
    assert pool.buf[a:a + 40].view(torch.int32).tolist() == [7] * 10


def test_pool_rejects_unknown_offsets_and_frees_coalesce_both_ways():
    pool = serve.DevicePool(1 << 16, device="cpu")
    a, b, c = pool.alloc(1000), pool.alloc(1000), pool.alloc(1000)
    assert (a, b, c) == (0, 1024, 2048)
    with pytest.raises(bulk_b200.BulkError):
        pool.free(12345)
    pool.free(a)
    pool.free(c)  # c merges with the tail
    assert pool.free_blocks() == 2
    pool.free(b)  # b merges with both neighbours
    assert pool.free_blocks() == 1 and pool.in_use == 0 and pool.high_water == 3072


def _req_array(reqs):
    arr = (serve._Request * len(reqs))()
    for i, (k, n) in enumerate(reqs):
        arr[i].kind, arr[i].n = k, n
    return arr


def test_workspace_bound_covers_every_call():
    """Plain: the largest single-call workspace.  Batched: at least every
    kind's largest batch of BK_BATCH_MAX requests, and never less than plain
    needs for a one-request batch."""
    ws = bulk_b200.workspace_bytes
    rng = np.random.default_rng(3)
    reqs = [(int(k), int(n)) for k, n in zip(rng.integers(0, 3, 700), rng.integers(1, 1 << 22, 700))]
    arr = _req_array(reqs)
    plain = _lib.lib.bk_serve_workspace_bytes(ctypes.cast(arr, ctypes.c_void_p), len(reqs), 0)
    singles = {0: ("sort_by_key", "u32", "u32"), 1: ("reduce_by_key", "i32", "f32"), 2: ("inclusive_scan", "f32", None)}
    assert plain == max(ws(*singles[k], n) for k, n in reqs)
    batched = _lib.lib.bk_serve_workspace_bytes(ctypes.cast(arr, ctypes.c_void_p), len(reqs), 1)
    for kind in range(3):
        top = sorted((n for k, n in reqs if k == kind), reverse=True)[:256]
        assert batched >= batch_workspace_bytes(*singles[kind], top)
    assert batched >= plain


def test_request_stream_follows_the_config():
    reqs = serve.make_requests(4000, 2000.0, seed=1000)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and arr[0] == 0.0
    assert abs(len(reqs) / arr[-1] - 2000.0) < 200.0  # Poisson rate
    frac = {k: sum(r.kind == k for r in reqs) / len(reqs) for k in serve.KINDS}
    assert abs(frac["sort"] - 0.4) < 0.04 and abs(frac["rbk"] - 0.3) < 0.04 and abs(frac["scan"] - 0.3) < 0.04
    ns = np.array([r.n for r in reqs])
    assert ns.min() >= 1 << 10 and ns.max() <= 1 << 24
    # log-uniform: about half below the geometric middle 2^17
    assert abs(np.mean(ns < (1 << 17)) - 0.5) < 0.05
    assert all(r.arrival == 0.0 for r in serve.make_requests(50, math.inf))
    # same seed, same stream
    again = serve.make_requests(4000, 2000.0, seed=1000)
    assert [(r.kind, r.n) for r in again] == [(r.kind, r.n) for r in reqs]


def _alone(server, req):
    """Run one request by itself (fresh buffers) and return its results."""
    import bulk_b200
    o, n = server.src.offset(req), req.n
    if req.kind == "sort":
        k = server.src.sort_keys[o:o + n].clone()
        v = server.src.sort_vals[o:o + n].clone()
        bulk_b200.stable_sort_by_key(k, v)
        return k, v
    if req.kind == "rbk":
        ok, ov, c = bulk_b200.reduce_by_key(server.src.rbk_keys[o:o + n], server.src.rbk_vals[o:o + n], sync=False)
        return ok, ov, c
    return (bulk_b200.inclusive_scan(server.src.scan_vals[o:o + n], 0.0),)


def _bound(x: torch.Tensor) -> torch.Tensor:
    n = max(x.numel(), 2)
    eps = 2.0 ** -23
    return 2 * 2 * math.ceil(math.log2(n)) * eps * torch.cumsum(x.double().abs(), 0)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "batched"])
def test_serving_results_match_each_request_alone(cuda, mode):
    src = serve.Sources(1 << 19)
    pool = serve.DevicePool(1 << 28)
    server = serve.Server(src, pool, budget_bytes=1 << 27, keep_results=True)
    reqs = serve.make_requests(120, math.inf, seed=77, lo=1 << 10, hi=1 << 18)
    stats = server.run(reqs, mode)
    assert stats["requests"] == 120 and stats["req_per_s"] > 0
    assert all(0 <= r.arrival <= r.start <= r.done for r in reqs)
    if mode == "plain":
        assert stats["calls"] == 120 and stats["batches"] == 0
    else:
        assert 3 <= stats["batches"] < 120  # all 120 arrive at once: few batches
    torch.cuda.synchronize()
    for r in reqs:
        got = server.results[r.rid]
        want = _alone(server, r)
        if r.kind == "sort":
            assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), r
        elif r.kind == "rbk":
            c = int(want[2].item())
            assert int(got[2].item()) == c, r
            assert torch.equal(got[0][:c], want[0][:c]), r
            o = src.offset(r)
            vals = src.rbk_vals[o:o + r.n]
            assert torch.all((got[1][:c].double() - want[1][:c].double()).abs() <= _bound(vals)[-1] + 1e-30), r
        else:
            o = src.offset(r)
            x = src.scan_vals[o:o + r.n]
            assert torch.all((got[0].double() - want[0].double()).abs() <= _bound(x)), r


@pytest.mark.gpu
def test_batched_small_rounds_match_each_request_alone(cuda):
    """Spaced arrivals: batched mode issues rounds of up to four requests as
    plain calls, and a lone sort of 2^20 elements or more as a one-item
    out-of-place batch reading its source window; every result must still be
    the request's own."""
    src = serve.Sources(1 << 21)
    pool = serve.DevicePool(1 << 28)
    server = serve.Server(src, pool, budget_bytes=1 << 27, keep_results=True)
    reqs = serve.make_requests(24, 400.0, seed=31, lo=1 << 20, hi=1 << 21)
    assert any(r.kind == "sort" for r in reqs)
    stats = server.run(reqs, "batched")
    assert stats["requests"] == 24
    torch.cuda.synchronize()
    for r in reqs:
        got = server.results[r.rid]
        want = _alone(server, r)
        if r.kind == "sort":
            assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1]), r
        elif r.kind == "rbk":
            c = int(want[2].item())
            assert int(got[2].item()) == c and torch.equal(got[0][:c], want[0][:c]), r
            o = src.offset(r)
            vals = src.rbk_vals[o:o + r.n]
            assert torch.all((got[1][:c].double() - want[1][:c].double()).abs() <= _bound(vals)[-1] + 1e-30), r
        else:
            o = src.offset(r)
            x = src.scan_vals[o:o + r.n]
            assert torch.all((got[0].double() - want[0].double()).abs() <= _bound(x)), r


@pytest.mark.gpu
def test_admission_respects_the_budget(cuda):
    src = serve.Sources(1 << 18)
    pool = serve.DevicePool(1 << 26)
    budget = 6 << 20  # a few requests at a time
    server = serve.Server(src, pool, budget_bytes=budget)
    reqs = serve.make_requests(60, math.inf, seed=5, lo=1 << 12, hi=1 << 18)
    stats = server.run(reqs, "batched")
    assert stats["requests"] == 60
    assert 0 < stats["pool_high_water_bytes"] <= budget + 60 * 3 * 256  # granule rounding


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["plain", "batched"])
def test_a_request_larger_than_the_budget_runs_alone(cuda, mode):
    src = serve.Sources(1 << 18)
    pool = serve.DevicePool(1 << 26)
    server = serve.Server(src, pool, budget_bytes=1 << 20)
    reqs = serve.make_requests(30, math.inf, seed=9, lo=1 << 16, hi=1 << 18)  # 0.5-2 MB each
    stats = server.run(reqs, mode)
    assert stats["requests"] == 30 and all(r.done >= r.start >= 0 for r in reqs)
    big = max(r.nbytes() for r in reqs)
    assert big > 1 << 20 and stats["pool_high_water_bytes"] <= (1 << 20) + big
