"""The serving loop (bulk_b200/serve.py): pooled allocator, request stream,
plain vs batched serving, and the alone-vs-in-mix parity of results.

The allocator and the request generator run on CPU tensors; the serving runs
need a GPU.  Parity: a request's sort result (keys and payload), its
reduce_by_key keys and count are bit-identical whether it ran alone or inside
a batch; float sums and scan prefixes agree within the suite's bound
2*ceil(log2 n)*eps*sum|x| (twice, since both sides carry that error).
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from bulk_b200 import serve


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
    assert pool.in_use == 0 and pool._free == [(0, pool.capacity)]
    assert pool.high_water > 0


def test_pool_refuses_when_full_and_views_alias_the_buffer():
    pool = serve.DevicePool(4096, device="cpu")
    a = pool.alloc(3000)
    assert pool.alloc(2000) is None  # only 1024 bytes left
    v = pool.view(a, 10, torch.int32)
    v[:] = 7
    assert pool.buf[a:a + 40].view(torch.int32).tolist() == [7] * 10


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
    assert pool.in_use == 0 and server.admitted_bytes == 0
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
def test_admission_respects_the_budget(cuda):
    src = serve.Sources(1 << 18)
    pool = serve.DevicePool(1 << 26)
    budget = 6 << 20  # a few requests at a time
    server = serve.Server(src, pool, budget_bytes=budget)
    reqs = serve.make_requests(60, math.inf, seed=5, lo=1 << 12, hi=1 << 18)
    stats = server.run(reqs, "batched")
    assert stats["requests"] == 60
    assert pool.high_water <= budget + 60 * 3 * 256  # granule rounding
