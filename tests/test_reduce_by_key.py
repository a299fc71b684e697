"""GPU parity of bk_reduce_by_key_* against the oracle (reduce_by_key.cu:176-272
semantics: one (key, sum) per run of equal consecutive keys, in run order).

Keys and run counts are bit-exact; integer sums are exact (wrapping); float
sums stay within 2*ceil(log2 n)*eps*sum|v| over the run of the oracle's
long-double sums.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from bulk_b200 import _lib
from tests.gpu_util import NP, assert_within_bound, dev, host
from tests.sizes import reference_sizes

pytestmark = pytest.mark.gpu
COMBOS = [("i32", "i32"), ("i32", "i64"), ("i32", "f32"), ("i32", "f64"), ("u32", "f32"), ("u32", "f64"),
          ("i64", "i32"), ("i64", "i64"), ("i64", "f32"), ("i64", "f64")]


def _check(keys, vals, gk, gv, count):
    if vals.dtype in (np.float32, np.float64):
        wk, wv, wmag = oracle.reduce_by_key(keys, vals)
        assert count == wk.size
        assert np.array_equal(gk, wk)
        assert_within_bound(gv, wv, wmag, max(keys.size, 1), vals.dtype, f"rbk n={keys.size}")
    else:
        wk, wv = oracle.reduce_by_key(keys, vals)
        assert count == wk.size and np.array_equal(gk, wk) and np.array_equal(gv, wv)


def _run(keys, vals):
    gk, gv, c = bulk_b200.reduce_by_key(dev(keys), dev(vals))
    return host(gk), host(gv), c


def test_known_answer_hash_mod10(cuda):
    # reduce_by_key.cu:364-420: keys = values = hash(i) % 10 over the drivers' size schedule
    for n in reference_sizes():
        keys = oracle.ref_hash_fill_i32(n, 10)
        _check(keys, keys.copy(), *_run(keys, keys.copy()))
    assert bulk_b200.workspace_status() == 0


def _runs(kind, n, seed):
    if kind == "geometric":
        return oracle.gen_runs_geometric(n, seed, 16.0)
    if kind == "zipf":
        return oracle.gen_runs_zipf(n, seed, 1.2, 1 << 20)
    if kind == "distinct":
        return np.arange(n, dtype=np.int32)
    if kind == "one":
        return np.full(n, 7, dtype=np.int32)
    raise ValueError(kind)


def _vals(tag, n, seed):
    if tag in ("f32", "f64"):
        return oracle.gen(NP[tag], n, seed, 0.0, 1.0)
    return oracle.gen(np.int32, n, seed, -1000, 1000).astype(NP[tag])


def _tile(kt, vt):
    """Elements per tile: 256 lanes x 16 elements (8 when key and value are both 8 bytes wide)."""
    return 256 * (16 if NP[kt]().itemsize + NP[vt]().itemsize <= 12 else 8)


@pytest.mark.parametrize("kt,vt", COMBOS)
def test_edge_sizes_and_run_shapes(cuda, kt, vt):
    # around one, two and three tiles T; T + 32 and 3T + 96: a last tile whose
    # rows the tensor copies still cover, next to the sizes whose ragged end is
    # staged by plain loads; 2064, 4128, 12384: ragged ends of other widths
    t = _tile(kt, vt)
    sizes = [0, 1, 2, 3, t // 2 + 16, t - 1, t, t + 1, t + 32, 2 * t, 2 * t + 1, 3 * t + 96,
             2064, 4095, 4096, 4097, 4128, 8192, 12384, 100003]
    for i, n in enumerate(sizes):
        for kind in ("geometric", "distinct", "one"):
            keys = _runs(kind, n, 5 + i).astype(NP[kt])
            vals = _vals(vt, n, 7 + i)
            _check(keys, vals, *_run(keys, vals))


@pytest.mark.parametrize("vt", ["f32", "f64"])
def test_zipf_runs_spanning_many_tiles(cuda, vt):
    n = 3_000_000
    keys = _runs("zipf", n, 6)
    vals = _vals(vt, n, 7)
    _check(keys, vals, *_run(keys, vals))


@pytest.mark.parametrize("kt,vt", [("i32", "i32"), ("i32", "f64"), ("i64", "i64")])
def test_runs_ending_on_tile_boundaries(cuda, kt, vt):
    t = _tile(kt, vt)
    n = t * 8
    keys = (np.arange(n) // t).astype(NP[kt])   # every run is exactly one tile
    vals = _vals(vt, n, 3)
    _check(keys, vals, *_run(keys, vals))
    keys = (np.arange(n) // (t - 1)).astype(NP[kt])   # runs straddle every boundary
    _check(keys, vals, *_run(keys, vals))
    keys = (np.arange(n) // 16).astype(NP[kt])   # a run ends on every lane's last element
    _check(keys, vals, *_run(keys, vals))


def test_misaligned_pointers(cuda):
    n = 50001
    keys = _runs("geometric", n + 1, 9)
    vals = _vals("f32", n + 1, 9)
    gk, gv, c = bulk_b200.reduce_by_key(dev(keys)[1:], dev(vals)[1:])
    _check(keys[1:], vals[1:], host(gk), host(gv), c)


def test_count_stays_on_device_without_sync(cuda):
    keys = _runs("geometric", 10000, 3)
    vals = _vals("i32", 10000, 3)
    ok, ov, cnt = bulk_b200.reduce_by_key(dev(keys), dev(vals), sync=False)
    assert cnt.is_cuda and int(cnt.item()) == oracle.reduce_by_key(keys, vals)[0].size


def test_stuck_predecessor_times_out_with_an_error(cuda):
    keys = torch.zeros(16 * 4096, dtype=torch.int32, device=cuda)
    vals = torch.ones(16 * 4096, dtype=torch.float32, device=cuda)
    try:
        bulk_b200.debug_set_fault(3, 50_000_000)
        bulk_b200.reduce_by_key(keys, vals, sync=False)
        assert bulk_b200.workspace_status() == _lib.BK_ERR_SPIN_TIMEOUT
    finally:
        bulk_b200.debug_set_fault(-1, 0)
    k, v, c = bulk_b200.reduce_by_key(keys, vals)
    assert c == 1 and float(v[0].item()) == 16 * 4096
    assert bulk_b200.workspace_status() == 0


@pytest.mark.slow
@pytest.mark.parametrize("kind", ["geometric", "zipf"])
@pytest.mark.parametrize("vt", ["f32", "f64"])
def test_full_size_2_27(cuda, kind, vt):
    """The benchmark configuration: 2^27 pairs, i32 keys in runs (geometric
    mean 16, or Zipf(1.2) capped at 2^20), values U[0,1).  The count and keys
    are compared bit-exact and every sum within the bound of the oracle's
    long-double run sums (a float64 device reference is not accurate enough
    for float64 sums over runs of up to 2^20 elements)."""
    n = 1 << 27
    keys = _runs(kind, n, 5 if kind == "geometric" else 6)
    vals = _vals(vt, n, 7)
    gk, gv, c = bulk_b200.reduce_by_key(dev(keys), dev(vals))
    _check(keys, vals, host(gk), host(gv), c)
    assert bulk_b200.workspace_status() == 0
