"""GPU parity of bk_inclusive_scan_* against the oracle (scan.cu:87-148 semantics:
out[i] = init (+) in[0] (+) ... (+) in[i]).

Integer scans are bit-exact; float prefixes stay within
|err_i| <= 2*ceil(log2 n)*eps*sum_{j<=i}|x_j| of the long-double oracle.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from bulk_b200 import _lib
from tests.gpu_util import NP, assert_within_bound, dev, gen, host
from tests.sizes import EDGE_SIZES, reference_sizes

pytestmark = pytest.mark.gpu
TAGS = ["i32", "u32", "i64", "u64", "f32", "f64"]


def _check(tag, op, x, init, got):
    if tag in ("f32", "f64") and op == "sum":
        ref, mag = oracle.inclusive_scan(x, NP[tag](init))
        assert_within_bound(got, ref, mag, max(x.size, 1), NP[tag], f"scan {tag} n={x.size}")
    else:
        want = oracle.inclusive_scan(x, NP[tag](init), op)
        bad = np.flatnonzero(got != want)
        assert bad.size == 0, f"scan_{op}_{tag} n={x.size}: first mismatch at {bad[0]}"


def test_known_answer_ones_init13(cuda):
    # scan.cu:158-184 with the size schedule of scan.cu:214-229
    for n in reference_sizes():
        x = torch.ones(n, dtype=torch.int32, device=cuda)
        out = bulk_b200.inclusive_scan(x, 13)
        assert torch.equal(out, torch.arange(14, 14 + n, dtype=torch.int32, device=cuda)), n
    assert bulk_b200.workspace_status() == 0


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("op", ["sum", "min", "max"])
def test_edge_sizes(cuda, tag, op):
    for i, n in enumerate(EDGE_SIZES):
        x = gen(tag, n, 200 + i)
        init = NP[tag](3 if tag not in ("f32", "f64") else -0.5)
        got = host(bulk_b200.inclusive_scan(dev(x), init, op))
        _check(tag, op, x, init, got)


def test_in_place(cuda):
    x = gen("i32", 1000003, 5)
    d = dev(x)
    bulk_b200.inclusive_scan(d, 1, out=d)
    _check("i32", "sum", x, 1, host(d))


@pytest.mark.parametrize("tag", ["i32", "f64"])
def test_misaligned_pointers(cuda, tag):
    n = 300001
    x = gen(tag, n + 1, 6)
    d = dev(x)[1:]
    out = torch.empty(n + 3, dtype=d.dtype, device=cuda)[3:]
    bulk_b200.inclusive_scan(d, NP[tag](0), out=out)
    _check(tag, "sum", x[1:], 0, host(out))


@pytest.mark.parametrize("tag", ["i32", "f32", "f64"])
def test_device_init_matches_host_init(cuda, tag):
    # init read on the device (the _dinit entry points) enters the same fold
    # as init passed by value: integers give the same bits; float prefixes
    # stay within the oracle's bound (float scans over several tiles are not
    # bitwise reproducible run to run: the look-back's decomposition varies)
    for i, n in enumerate([1, 777, 8192 * 3 + 5, 1000003]):
        x = gen(tag, n, 300 + i)
        init = NP[tag](7 if tag == "i32" else -1.25)
        d = dev(x)
        got = bulk_b200.inclusive_scan(d, torch.tensor([init], device=cuda))
        if tag == "i32":
            assert torch.equal(got, bulk_b200.inclusive_scan(d, init)), (tag, n)
        _check(tag, "sum", x, init, host(got))


def test_chained_chunks_equal_one_scan(cuda):
    # a stream scanned chunk by chunk, each chunk starting from the previous
    # chunk's last output still on the device, equals one scan of the whole
    x = gen("i32", 3_000_001, 9)
    d = dev(x)
    out = torch.empty_like(d)
    bounds = [0, 1, 4097, 1_000_000, 1_000_003, 2_500_000, 3_000_001]
    for lo, hi in zip(bounds, bounds[1:]):
        init = 13 if lo == 0 else out[lo - 1:lo]
        bulk_b200.inclusive_scan(d[lo:hi], init, out=out[lo:hi])
    _check("i32", "sum", x, 13, host(out))


def test_device_init_rejects_a_null_pointer(cuda):
    d = torch.ones(100, dtype=torch.int32, device=cuda)
    ws = torch.zeros(bulk_b200.workspace_bytes("inclusive_scan", "i32", None, 100), dtype=torch.uint8, device=cuda)
    st = bulk_b200.lib.bk_inclusive_scan_sum_i32_dinit(d.data_ptr(), 100, None, d.data_ptr(), ws.data_ptr(),
                                                       ws.numel(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.BK_ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError):
        bulk_b200.inclusive_scan(d, torch.tensor([1.0], device=cuda))  # wrong dtype


def test_repeated_calls_reuse_the_workspace(cuda):
    x = gen("f32", (1 << 22) + 7, 8)
    d = dev(x)
    for _ in range(3):
        _check("f32", "sum", x, 0, host(bulk_b200.inclusive_scan(d, np.float32(0))))
    assert bulk_b200.workspace_status() == 0


def test_stuck_predecessor_times_out_with_an_error(cuda):
    """Tile 3 never publishes its status: the tiles after it must give up after
    the (short) wait limit and report BK_ERR_SPIN_TIMEOUT, and the context must
    stay usable for the next call."""
    x = torch.ones(16 * 4096, dtype=torch.int32, device=cuda)
    try:
        bulk_b200.debug_set_fault(3, 50_000_000)  # 50 ms
        bulk_b200.inclusive_scan(x, 0)
        assert bulk_b200.workspace_status() == _lib.BK_ERR_SPIN_TIMEOUT
    finally:
        bulk_b200.debug_set_fault(-1, 0)
    out = bulk_b200.inclusive_scan(x, 0)
    assert torch.equal(out, torch.arange(1, x.numel() + 1, dtype=torch.int32, device=cuda))
    assert bulk_b200.workspace_status() == 0


@pytest.mark.slow
@pytest.mark.parametrize("tag", ["i32", "f32", "f64"])
def test_full_size_2_28(cuda, tag):
    n = 1 << 28
    xh = gen(tag, n, 0)
    x = dev(xh)
    out = bulk_b200.inclusive_scan(x, NP[tag](0))
    if tag == "i32":
        # size-independent properties: first element and adjacent differences
        assert out[0].item() == x[0].item()
        assert torch.equal(out[1:] - out[:-1], x[1:])
        # and element by element against the oracle (exact, wrapping)
        assert np.array_equal(host(out), oracle.inclusive_scan(xh, np.int32(0)))
    else:
        ref = torch.cumsum(x.double(), 0)
        mag = torch.cumsum(x.double().abs(), 0)
        err = (out.double() - ref).abs()
        bound = torch.from_numpy(oracle.fp_bound(n, NP[tag], 1.0) * np.ones(1)).cuda() * mag
        assert bool((err <= bound).all())
    assert bulk_b200.workspace_status() == 0
