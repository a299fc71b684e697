"""CUDA-graph capture of library calls.

No entry point allocates device memory, synchronizes with the host or queries
a stream (the workspace is the caller's, and every kernel leaves its
counters zeroed), so a fixed sequence of calls on one stream can be captured
once into a CUDA graph and replayed on new data in the same buffers.  The
test captures a scan, an in-place stable sort_by_key (radix passes), a
reduce_by_key and a reduce, replays the graph three times on fresh seeded
inputs and checks every result against the oracle: integers bit-exact, float
prefixes within 2*ceil(log2 n)*eps*sum|x|.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from tests.gpu_util import assert_within_bound, host

pytestmark = pytest.mark.gpu


def test_calls_capture_in_a_cuda_graph_and_replay(cuda):
    ns, nk, nr = 100_003, 50_001, 70_001
    s = torch.cuda.Stream(device=cuda)
    x = torch.empty(ns, dtype=torch.float32, device=cuda)
    y = torch.empty_like(x)
    k = torch.empty(nk, dtype=torch.int32, device=cuda)
    v = torch.empty(nk, dtype=torch.int32, device=cuda)
    rk = torch.empty(nr, dtype=torch.int32, device=cuda)
    rv = torch.empty(nr, dtype=torch.int32, device=cuda)
    ok = torch.empty(nr, dtype=torch.int32, device=cuda)
    ov = torch.empty(nr, dtype=torch.int32, device=cuda)
    cnt = torch.empty(1, dtype=torch.int64, device=cuda)
    xi = torch.empty(ns, dtype=torch.int32, device=cuda)
    red = torch.empty(1, dtype=torch.int32, device=cuda)

    def fill(seed):
        xs = oracle.gen(np.float32, ns, seed, -1.0, 1.0)
        ks = oracle.gen(np.int32, nk, seed + 1, -3000, 3000)
        rks = oracle.gen_runs_geometric(nr, seed + 2, 16.0).astype(np.int32)
        rvs = oracle.gen(np.int32, nr, seed + 3, -100, 100)
        xis = oracle.gen(np.int32, ns, seed + 4, -1000, 1000)
        for dst, src in ((x, xs), (k, ks), (v, np.arange(nk, dtype=np.int32)), (rk, rks), (rv, rvs), (xi, xis)):
            dst.copy_(torch.from_numpy(src))
        torch.cuda.synchronize()
        return xs, ks, rks, rvs, xis

    def step():
        bulk_b200.inclusive_scan(x, np.float32(0.25), out=y, stream=s)
        bulk_b200.stable_sort_by_key(k, v, stream=s)
        bulk_b200.reduce_by_key(rk, rv, ok, ov, cnt, stream=s, sync=False)
        bulk_b200.reduce(xi, 13, out=red, stream=s)

    # warm-up on the capture stream: kernel attributes set, workspace in place
    fill(1)
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        step()
    for rep in range(3):
        xs, ks, rks, rvs, xis = fill(100 + 10 * rep)
        g.replay()
        torch.cuda.synchronize()
        ref, mag = oracle.inclusive_scan(xs, np.float32(0.25))
        assert_within_bound(host(y), ref, mag, ns, np.float32, f"scan, replay {rep}")
        wk, wv = oracle.stable_sort_by_key(ks, np.arange(nk, dtype=np.uint32))
        assert np.array_equal(host(k), wk) and np.array_equal(host(v).view(np.uint32), wv), rep
        wrk, wrv = oracle.reduce_by_key(rks, rvs)
        c = int(cnt.item())
        assert c == wrk.size and np.array_equal(host(ok)[:c], wrk) and np.array_equal(host(ov)[:c], wrv), rep
        assert int(red.item()) == oracle.reduce(xis, 13), rep
    assert bulk_b200.workspace_status(stream=s) == 0
    del g
