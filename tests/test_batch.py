"""Batched entry points (bk_*_batch): many independent arrays per launch.

Each array's result must be what it gets alone: integer results bit-exact
against the single-array entry point and the oracle, float results within the
suite's bound 2*ceil(log2 n)*eps*sum|x| of the long-double oracle.  Host-side
checks (the C structs' layout, the workspace size, argument errors) need no
GPU.
"""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from bulk_b200 import _lib
from bulk_b200.batch import batch_workspace_bytes, rbk_item_type, scan_item_type, sort_item_type

ROOT_HEADER = _lib.HEADER.read_text()
TAGS = ["i32", "u32", "i64", "u64", "f32", "f64"]
RBK_COMBOS = [("i32", "i32"), ("i32", "i64"), ("i32", "f32"), ("i32", "f64"), ("u32", "f32"), ("u32", "f64"),
              ("i64", "i32"), ("i64", "i64"), ("i64", "f32"), ("i64", "f64")]
SCAN_TILE = {"i32": 8192, "u32": 8192, "f32": 8192, "i64": 4096, "u64": 4096, "f64": 4096}
# a mix of empty, tiny, tile-edge and multi-tile arrays
SIZES = [0, 1, 3, 8191, 8192, 8193, 4095, 4097, 100003, 1, 262144, 0, 777, 1 << 20, 12345]


# ---------------------------------------------------------------- host side
def test_header_declares_batch_entry_points():
    for t in TAGS:
        assert f"bk_inclusive_scan_sum_{t}_batch(" in ROOT_HEADER
        assert re.search(rf"typedef struct bk_scan_item_{t} \{{", ROOT_HEADER)
    for k, v in RBK_COMBOS:
        assert f"bk_reduce_by_key_{k}_{v}_batch(" in ROOT_HEADER
    for t in TAGS:
        for v in ("u32", "u64"):
            assert f"bk_sort_by_key_{t}_{v}_batch(" in ROOT_HEADER
    assert "#define BK_BATCH_MAX 256" in ROOT_HEADER and bulk_b200.BATCH_MAX == 256


@pytest.mark.parametrize("tag", TAGS)
def test_scan_item_layout(tag):
    # pointer, pointer, uint64 n, init (padded to 8)
    assert ctypes.sizeof(scan_item_type(tag)) == 32


@pytest.mark.parametrize("kv", RBK_COMBOS)
def test_rbk_item_layout(kv):
    assert ctypes.sizeof(rbk_item_type(*kv)) == 48


@pytest.mark.parametrize("algo,kv", [("reduce_by_key", ("i32", "f32")), ("reduce_by_key", ("i64", "f64")),
                                     ("inclusive_scan", ("f32", None)), ("inclusive_scan", ("u64", None))])
def test_batch_of_one_needs_what_one_call_needs(algo, kv):
    for n in (1, 4096, 100003, 1 << 22):
        assert batch_workspace_bytes(algo, kv[0], kv[1], [n]) == bulk_b200.workspace_bytes(algo, kv[0], kv[1], n)
    # more arrays never need less
    assert batch_workspace_bytes(algo, kv[0], kv[1], [5000, 7000]) >= batch_workspace_bytes(algo, kv[0], kv[1],
                                                                                            [7000])


def test_sort_item_layout_and_workspace():
    assert ctypes.sizeof(sort_item_type("u32", "u32")) == 24
    # a one-array batch needs what the single-array call needs; more arrays need more
    for n in (2, 5000, 1 << 20):
        for kt, vt in (("u32", "u32"), ("u64", "u32"), ("f64", "u64")):
            assert batch_workspace_bytes("sort_by_key", kt, vt, [n]) == bulk_b200.workspace_bytes(
                "sort_by_key", kt, vt, n)
    one = batch_workspace_bytes("sort_by_key", "u32", "u32", [5000])
    assert batch_workspace_bytes("sort_by_key", "u32", "u32", [5000, 0, 1, 5000]) > one
    # arrays of 0 or 1 element need nothing beyond the header
    assert batch_workspace_bytes("sort_by_key", "u32", "u32", [0, 1]) == batch_workspace_bytes(
        "sort_by_key", "u32", "u32", [])


def test_too_many_items_is_rejected_before_any_device_work():
    items = (scan_item_type("f32") * 257)()
    st = _lib.lib.bk_inclusive_scan_sum_f32_batch(ctypes.cast(items, ctypes.c_void_p), 257, None, 0, None)
    assert st == _lib.BK_ERR_TOO_LARGE


# ---------------------------------------------------------------- GPU side
def _gen(tag, n, seed):
    from tests.gpu_util import gen
    return gen(tag, n, seed)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_scan_batch_matches_each_array_alone(cuda, tag):
    from tests.gpu_util import NP, assert_within_bound, dev, host
    xs_h = [_gen(tag, n, 300 + i) for i, n in enumerate(SIZES)]
    inits = [NP[tag](i % 5) for i in range(len(SIZES))]
    xs = [dev(x) for x in xs_h]
    outs = bulk_b200.inclusive_scan_batch(xs, inits)
    for x, init, out, xd in zip(xs_h, inits, outs, xs):
        got = host(out)
        if tag in ("f32", "f64"):
            ref, mag = oracle.inclusive_scan(x, init)
            assert_within_bound(got, ref, mag, max(x.size, 1), NP[tag], f"batch scan {tag} n={x.size}")
        else:
            alone = host(bulk_b200.inclusive_scan(xd, init))
            assert np.array_equal(got, alone), f"n={x.size}"
            assert np.array_equal(got, oracle.inclusive_scan(x, init, "sum")), f"n={x.size}"
    assert bulk_b200.workspace_status() == 0


@pytest.mark.gpu
def test_scan_batch_unaligned_views_and_in_place(cuda):
    from tests.gpu_util import dev, host
    base = dev(_gen("i32", 300001, 7))
    views = [base[1:100001], base[100003:200000], base[200001:]]  # 4-byte aligned, not 16
    want = [torch.cumsum(v.long(), 0).to(torch.int32) for v in views]
    outs = bulk_b200.inclusive_scan_batch(views, [0, 0, 0], outs=views)  # in place
    for o, w in zip(outs, want):
        assert torch.equal(o, w)
    assert bulk_b200.workspace_status() == 0


@pytest.mark.gpu
def test_scan_batch_of_more_than_256_arrays(cuda):
    xs = [torch.full((17 + (i % 40) * 1000,), i % 7, dtype=torch.int32, device=cuda) for i in range(300)]
    outs = bulk_b200.inclusive_scan_batch(xs, [1] * 300)
    for i, (x, o) in enumerate(zip(xs, outs)):
        assert torch.equal(o, 1 + torch.cumsum(x.long(), 0).to(torch.int32)), i


@pytest.mark.gpu
def test_scan_batch_stuck_predecessor_times_out_with_an_error(cuda):
    """Global tile 3 (inside the second array) never publishes: the tiles
    after it give up after the short limit and the call reports
    BK_ERR_SPIN_TIMEOUT; the next batch is correct."""
    xs = [torch.ones(2 * 8192, dtype=torch.int32, device=cuda), torch.ones(10 * 8192, dtype=torch.int32, device=cuda)]
    try:
        bulk_b200.debug_set_fault(3, 50_000_000)
        bulk_b200.inclusive_scan_batch(xs)
        assert bulk_b200.workspace_status() == _lib.BK_ERR_SPIN_TIMEOUT
    finally:
        bulk_b200.debug_set_fault(-1, 0)
    outs = bulk_b200.inclusive_scan_batch(xs)
    for x, o in zip(xs, outs):
        assert torch.equal(o, torch.arange(1, x.numel() + 1, dtype=torch.int32, device=cuda))
    assert bulk_b200.workspace_status() == 0


def _runs(n, mean, seed):
    rng = np.random.default_rng(seed)
    if n == 0:
        return np.zeros(0, np.int64)
    heads = rng.random(n) < 1.0 / mean
    heads[0] = True
    return np.cumsum(heads).astype(np.int64) * 7 - 3


@pytest.mark.gpu
@pytest.mark.parametrize("kv", RBK_COMBOS)
def test_reduce_by_key_batch_matches_each_array_alone(cuda, kv):
    from tests.gpu_util import NP, assert_within_bound, dev, host
    kt, vt = kv
    keys_h, vals_h = [], []
    for i, n in enumerate(SIZES):
        keys_h.append(_runs(n, (1, 4, 16, 300)[i % 4], 400 + i).astype(NP[kt]))
        vals_h.append(_gen(vt, n, 500 + i))
    res = bulk_b200.reduce_by_key_batch([dev(k) for k in keys_h], [dev(v) for v in vals_h], sync=True)
    for k, v, (gk, gv, c) in zip(keys_h, vals_h, res):
        gk, gv = host(gk), host(gv)
        if vt in ("f32", "f64"):
            wk, wv, wmag = oracle.reduce_by_key(k, v)
            assert c == wk.size and np.array_equal(gk, wk)
            assert_within_bound(gv, wv, wmag, max(k.size, 1), NP[vt], f"batch rbk n={k.size}")
        else:
            wk, wv = oracle.reduce_by_key(k, v)
            assert c == wk.size and np.array_equal(gk, wk) and np.array_equal(gv, wv), f"n={k.size}"
            ak, av, ac = bulk_b200.reduce_by_key(dev(k), dev(v))
            assert ac == c and np.array_equal(host(ak), gk) and np.array_equal(host(av), gv)
    assert bulk_b200.workspace_status() == 0


@pytest.mark.gpu
def test_reduce_by_key_batch_counts_stay_on_device(cuda):
    keys = [torch.tensor([1, 1, 2, 3, 3, 3], dtype=torch.int32, device=cuda),
            torch.zeros(0, dtype=torch.int32, device=cuda),
            torch.tensor([5], dtype=torch.int32, device=cuda)]
    vals = [torch.arange(k.numel(), dtype=torch.float32, device=cuda) for k in keys]
    res = bulk_b200.reduce_by_key_batch(keys, vals)  # sync=False
    counts = [int(c.item()) for _, _, c in res]
    assert counts == [3, 0, 1]
    assert res[0][0][:3].tolist() == [1, 2, 3] and res[0][1][:3].tolist() == [1.0, 2.0, 12.0]


@pytest.mark.gpu
@pytest.mark.parametrize("kv", [("u32", "u32"), ("f32", "u32"), ("i64", "u32"), ("u64", "u64"), ("f64", "u64")])
def test_sort_batch_matches_each_array_alone(cuda, kv):
    """Stable order: payload = original index, ties (few distinct keys) must
    keep it; sizes span 0..2^20 so the arrays need 0..7 merge passes."""
    from tests.gpu_util import NP, dev, host
    kt, vt = kv
    sizes = [0, 1, 2, 100, 4095, 4096, 8193, 20000, 1 << 16, 300001, 1 << 20, 7]
    keys_h, vals_h = [], []
    for i, n in enumerate(sizes):
        rng = np.random.default_rng(600 + i)
        if kt in ("f32", "f64"):
            k = rng.integers(0, 50, n).astype(NP[kt]) / 4
        else:
            k = rng.integers(0, 1000 if i % 2 else 1 << 30, n).astype(NP[kt])
        keys_h.append(k)
        vals_h.append(np.arange(n, dtype=NP[vt]))
    dk = [dev(k) for k in keys_h]
    dv = [dev(v) for v in vals_h]
    bulk_b200.stable_sort_by_key_batch(dk, dv)
    for k, v, gk, gv in zip(keys_h, vals_h, dk, dv):
        order = np.argsort(k, kind="stable")
        assert np.array_equal(host(gk), k[order]), f"n={k.size}"
        assert np.array_equal(host(gv), v[order]), f"n={k.size}"


@pytest.mark.gpu
@pytest.mark.parametrize("kv", [("u32", "u32"), ("f32", "u32"), ("u64", "u64")])
@pytest.mark.parametrize("sizes", [[0, 1, 2, 100, 4095, 8193, 20000, 300001, 7],   # radix passes
                                   [0, 1, 5, 300, 4096, 17]])                     # one block sort
def test_sort_copy_batch_reads_the_sources_and_leaves_them(cuda, kv, sizes):
    """Out of place: each (in_keys, in_vals) sorted stably into its own
    outputs, the sources unchanged (the first radix pass, or the block sort,
    reads them directly)."""
    from tests.gpu_util import NP, dev, host
    kt, vt = kv
    keys_h, vals_h = [], []
    for i, n in enumerate(sizes):
        rng = np.random.default_rng(700 + i)
        k = (rng.integers(0, 50, n) / 4).astype(NP[kt]) if kt == "f32" else \
            rng.integers(0, 1000 if i % 2 else 1 << 30, n).astype(NP[kt])
        keys_h.append(k)
        vals_h.append(np.arange(n, dtype=NP[vt]))
    dk = [dev(k) for k in keys_h]
    dv = [dev(v) for v in vals_h]
    ok, ov = bulk_b200.stable_sort_by_key_copy_batch(dk, dv)
    for k, v, gk, gv, sk, sv in zip(keys_h, vals_h, ok, ov, dk, dv):
        order = np.argsort(k, kind="stable")
        assert np.array_equal(host(gk), k[order]) and np.array_equal(host(gv), v[order]), f"n={k.size}"
        assert np.array_equal(host(sk), k) and np.array_equal(host(sv), v), f"source changed, n={k.size}"
