"""GPU parity of bk_sort_by_key_* / bk_sort_keys_* against the oracle: keys
and payload order bit-exact.  Below 2^30 elements the library sorts by stable
LSD radix, at and above it by merging; a stable sort's output is unique, so
both must equal the oracle's stable merge sort."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from tests.gpu_util import NP, dev, gen, host
from tests.sizes import reference_sizes

pytestmark = pytest.mark.gpu
KEYS = ["i32", "u32", "i64", "u64", "f32", "f64"]


def test_known_answer_hash_fill(cuda):
    # merge_sort_by_key.cu:315-380: keys and values hash-filled, the drivers' size schedule,
    # compared with a stable sort_by_key
    for n in reference_sizes():
        keys = oracle.ref_hash_fill_i32(n)
        vals = keys.copy()
        gk, gv = bulk_b200.stable_sort_by_key(dev(keys), dev(vals))
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(host(gk), keys[order]), n
        assert np.array_equal(host(gv), vals[order]), n


def _keys(tag, n, seed, coarse):
    x = gen(tag, n, seed)
    if coarse:  # many duplicates: stability matters
        if tag in ("f32", "f64"):
            x = np.floor(x * 50).astype(x.dtype)
        else:
            x = (x // np.array(1 << 20 if tag in ("i32", "u32") else 1 << 52).astype(x.dtype)).astype(x.dtype)
    return x


@pytest.mark.parametrize("tag", KEYS)
@pytest.mark.parametrize("payload", [None, np.uint32, np.uint64])
def test_edge_sizes(cuda, tag, payload):
    # 8193-131072 elements: one cluster launch (up to 16 CTAs of 4096-key,
    # then of 8192-key tiles); above: the global-memory radix passes
    sizes = [0, 1, 2, 3, 17, 1023, 4096, 8191, 8192, 8193, 16385, 3 * 8192 + 5, 32769, 65536, 65537, 100003,
             131072, 131075, 300007]
    for i, n in enumerate(sizes):
        for coarse in (False, True):
            keys = _keys(tag, n, 300 + i, coarse)
            if payload is None:
                got = host(bulk_b200.stable_sort_by_key(dev(keys)))
                assert np.array_equal(got, np.sort(keys, kind="stable")), (tag, n)
            else:
                vals = np.arange(n, dtype=payload)
                gk, gv = bulk_b200.stable_sort_by_key(dev(keys), dev(vals))
                wk, wv = oracle.stable_sort_by_key(keys, vals)
                assert np.array_equal(host(gk), wk) and np.array_equal(host(gv), wv), (tag, n, coarse)


def test_presorted_reversed_and_constant(cuda):
    n = 70001
    for keys in (np.arange(n, dtype=np.int32), np.arange(n, 0, -1).astype(np.int32), np.zeros(n, np.int32)):
        vals = np.arange(n, dtype=np.uint32)
        gk, gv = bulk_b200.stable_sort_by_key(dev(keys), dev(vals))
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(host(gv), order.astype(np.uint32))


def test_max_key_values_are_not_confused_with_padding(cuda):
    # partial tiles are padded with the largest key; real largest keys must stay ahead of it
    n = 8192 + 37
    keys = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
    keys[::3] = 5
    vals = np.arange(n, dtype=np.uint32)
    gk, gv = bulk_b200.stable_sort_by_key(dev(keys), dev(vals))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(host(gk), keys[order]) and np.array_equal(host(gv), order.astype(np.uint32))


@pytest.mark.slow
@pytest.mark.parametrize("tag", ["u32", "u64"])
def test_full_size_2_26_payload_is_index(cuda, tag):
    """The benchmark configuration: 2^26 keys over the full range, payload =
    original index.  Properties: keys nondecreasing, equal keys keep increasing
    payloads (stability), payload is a permutation, keys[i] == input[payload[i]]."""
    n = 1 << 26
    keys0 = dev(gen(tag, n, 3 if tag == "u32" else 4))
    keys = keys0.clone()
    vals = torch.arange(n, dtype=torch.int32, device=cuda)
    bulk_b200.stable_sort_by_key(keys, vals)
    # compare as signed views (unsigned order = signed order with the sign bit flipped)
    if tag == "u32":
        k = keys.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
        k0 = keys0.view(torch.int32)
        ks = keys.view(torch.int32)
    else:
        k = keys.view(torch.int64) ^ torch.tensor(-(1 << 63), dtype=torch.int64, device=cuda)
        k0 = keys0.view(torch.int64)
        ks = keys.view(torch.int64)
    ok = (k[1:] > k[:-1]) | ((k[1:] == k[:-1]) & (vals[1:] > vals[:-1]))
    assert bool(ok.all())
    assert torch.equal(torch.sort(vals).values, torch.arange(n, dtype=torch.int32, device=cuda))
    assert torch.equal(ks, k0[vals.long()])
    # and element by element against the oracle's stable sort
    wk, wv = oracle.stable_sort_by_key(host(keys0), np.arange(n, dtype=np.uint32))
    assert np.array_equal(host(keys), wk) and np.array_equal(host(vals).view(np.uint32), wv)


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_signed_zeros_infinities_and_denormals_keep_stable_order(cuda, tag):
    """-0.0 and +0.0 compare equal, so they tie and keep their input order;
    the keys come back with their own bit patterns."""
    dt = NP[tag]
    tiny = np.finfo(dt).smallest_subnormal
    special = np.array([0.0, -0.0, np.inf, -np.inf, tiny, -tiny, 1.0, -1.0, np.finfo(dt).max, -np.finfo(dt).max],
                       dtype=dt)
    rng = np.random.default_rng(11)
    for n in (10, 4097, 70001):
        keys = special[rng.integers(0, special.size, n)]
        vals = np.arange(n, dtype=np.uint32)
        gk, gv = bulk_b200.stable_sort_by_key(dev(keys), dev(vals))
        wk, wv = oracle.stable_sort_by_key(keys, vals)
        ut = np.uint32 if tag == "f32" else np.uint64
        assert np.array_equal(host(gk).view(ut), wk.view(ut)), n
        assert np.array_equal(host(gv), wv), n


@pytest.mark.parametrize("tag", ["u32", "i64"])
def test_views_off_16_byte_boundaries(cuda, tag):
    """Keys and payloads starting 1-3 elements past a 16-byte boundary: the
    scatter reads such tiles directly instead of by bulk copy.  In place and
    out of place (the batch entry point with separate sources), against the
    oracle."""
    from bulk_b200 import batch
    n = 3 * 4096 + 1234
    for off in (1, 2, 3):
        keys = _keys(tag, n, 40 + off, coarse=(off == 2))
        vals = np.arange(n, dtype=np.uint32)
        wk, wv = oracle.stable_sort_by_key(keys, vals)
        kb = torch.zeros(n + off, dtype=dev(keys).dtype, device=cuda)
        vb = torch.zeros(n + off, dtype=torch.int32, device=cuda)
        kb[off:].copy_(dev(keys))
        vb[off:].copy_(dev(vals.view(np.int32)))
        gk, gv = bulk_b200.stable_sort_by_key(kb[off:], vb[off:])
        assert np.array_equal(host(gk), wk) and np.array_equal(host(gv).view(np.uint32), wv), (tag, off)
        kb[off:].copy_(dev(keys))
        vb[off:].copy_(dev(vals.view(np.int32)))
        ok, ov = torch.empty(n + 1, dtype=kb.dtype, device=cuda), torch.empty(n + 1, dtype=torch.int32, device=cuda)
        (gk,), (gv,) = batch.stable_sort_by_key_copy_batch([kb[off:]], [vb[off:]], [ok[1:]], [ov[1:]])
        assert np.array_equal(host(gk), wk) and np.array_equal(host(gv).view(np.uint32), wv), (tag, off, "copy")


@pytest.mark.slow
def test_merge_path_at_2_30(cuda):
    """2^30 elements, the first size sorted by merging: i32 keys with many
    duplicates, payload = index, against torch's stable sort."""
    n = 1 << 30
    g = torch.Generator(device=cuda)
    g.manual_seed(5)
    keys = torch.randint(-(1 << 20), 1 << 20, (n,), generator=g, device=cuda, dtype=torch.int32)
    want = torch.sort(keys, stable=True)
    vals = torch.arange(n, dtype=torch.int32, device=cuda)
    bulk_b200.stable_sort_by_key(keys, vals)
    assert torch.equal(keys, want.values)
    assert torch.equal(vals, want.indices.to(torch.int32))
