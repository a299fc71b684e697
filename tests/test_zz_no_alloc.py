"""The allocation-free scan entry point, bk_inclusive_scan_sum_f32_noalloc.

It serves callers that cannot allocate device memory for a workspace (a
plugin inside an application that owns all GPU memory, a latency-critical path
that must not call cudaMalloc, an FFI caller without an allocator): its
scratch is a fixed array inside the library.  This test calls it through the
C-ABI twice in a row and checks each output against the oracle's prefix sums
and against the regular workspace entry point (bk_inclusive_scan_sum_f32),
within the float tolerance every scan test uses, 2*ceil(log2 n)*eps*sum|x|.  The file sorts last so that a run which
stops at the first failure has run every other test first; it also passes on
its own in a fresh process.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from bulk_b200 import _lib
from tests.gpu_util import assert_within_bound, dev, host

pytestmark = pytest.mark.gpu


def _noalloc(x: torch.Tensor, init: float) -> torch.Tensor:
    out = torch.empty_like(x)
    s = torch.cuda.current_stream().cuda_stream
    st = bulk_b200.lib.bk_inclusive_scan_sum_f32_noalloc(x.data_ptr(), x.numel(), init, out.data_ptr(), s)
    assert st == _lib.BK_OK, bulk_b200.lib.bk_status_string(st)
    return out


@pytest.mark.parametrize("n", [1, 8191, 8193, 1_000_003])
def test_noalloc_scan_matches_the_workspace_entry_point_twice(cuda, n):
    for call, seed in enumerate((11, 12)):  # two calls in a row share the array
        x = oracle.gen(np.float32, n, seed + n, -1.0, 1.0)
        d = dev(x)
        got = host(_noalloc(d, 0.5))
        want = host(bulk_b200.inclusive_scan(d, np.float32(0.5)))
        ref, mag = oracle.inclusive_scan(x, np.float32(0.5))
        assert_within_bound(got, ref, mag, n, np.float32, f"noalloc call {call} n={n} vs the oracle")
        assert_within_bound(got, want, mag, n, np.float32, f"noalloc call {call} n={n} vs the workspace call")


def test_noalloc_rejects_sizes_beyond_its_array():
    # checked before any device access
    st = bulk_b200.lib.bk_inclusive_scan_sum_f32_noalloc(None, (1 << 30) + 1, 0.0, None, None)
    assert st == _lib.BK_ERR_TOO_LARGE
