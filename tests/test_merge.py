"""GPU parity of bk_merge_* / bk_merge_by_key_* against the oracle: keys and
payload order bit-exact (ties take A first, merge.hpp:35-60, 63-170)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from tests.gpu_util import NP, dev, gen, host

pytestmark = pytest.mark.gpu
KEYS = ["i32", "u32", "i64", "u64", "f32", "f64"]


def _sorted_keys(tag, n, seed, dup_from=None):
    if tag in ("f32", "f64"):
        x = oracle.gen(NP[tag], n, seed, 0.0, 1.0)
    else:
        x = gen(tag, n, seed)
    if dup_from is not None and n and dup_from.size:
        # ~1% of the entries replaced by values drawn from the other array (cross ties)
        idx = oracle.gen(np.uint32, max(1, n // 100), seed + 99) % n
        src = oracle.gen(np.uint32, idx.size, seed + 98) % dup_from.size
        x[idx] = dup_from[src]
    return np.sort(x, kind="stable")


def test_known_answer_hash_fill_large(cuda):
    # merge.cu:258-278 (validate<int>(123456789)): two hash-filled halves, each sorted, merged
    n = 123456789
    a = np.sort(oracle.ref_hash_fill_i32(n // 2), kind="stable")
    b = a.copy()
    got = host(bulk_b200.merge(dev(a), dev(b)))
    assert np.array_equal(got, oracle.merge(a, b))


@pytest.mark.parametrize("tag", KEYS)
@pytest.mark.parametrize("payload", [None, np.uint32, np.uint64])
def test_edge_sizes_by_key(cuda, tag, payload):
    sizes = [(0, 0), (0, 5), (7, 0), (1, 1), (3, 4096), (4095, 1), (4096, 4096), (5000, 3193), (65537, 100003)]
    for i, (na, nb) in enumerate(sizes):
        a = _sorted_keys(tag, na, 10 + i)
        b = _sorted_keys(tag, nb, 50 + i, dup_from=a)
        if payload is None:
            got = host(bulk_b200.merge(dev(a), dev(b)))
            assert np.array_equal(got, oracle.merge(a, b)), (tag, na, nb)
        else:
            av = np.arange(na, dtype=payload)
            bv = (np.arange(nb) + (1 << 26)).astype(payload)
            gk, gv = bulk_b200.merge(dev(a), dev(b), dev(av), dev(bv))
            wk, wv = oracle.merge(a, b, av, bv)
            assert np.array_equal(host(gk), wk) and np.array_equal(host(gv), wv), (tag, na, nb)


@pytest.mark.parametrize("tag", ["i32", "f32"])
def test_all_ties_keep_a_first(cuda, tag):
    a = np.full(10000, 3, dtype=NP[tag])
    b = np.full(7000, 3, dtype=NP[tag])
    av = np.arange(10000, dtype=np.uint32)
    bv = np.arange(10000, 17000, dtype=np.uint32)
    gk, gv = bulk_b200.merge(dev(a), dev(b), dev(av), dev(bv))
    assert np.array_equal(host(gv), np.arange(17000, dtype=np.uint32))


def test_misaligned_and_signed_zero(cuda):
    a = np.array([-1.0, -0.0, 0.0, 2.0] * 1, dtype=np.float32)
    b = np.array([0.0, -0.0, 1.0], dtype=np.float32)
    b = np.sort(b, kind="stable")
    av = np.arange(4, dtype=np.uint32)
    bv = np.arange(100, 103, dtype=np.uint32)
    gk, gv = bulk_b200.merge(dev(a), dev(b), dev(av), dev(bv))
    wk, wv = oracle.merge(a, b, av, bv)
    assert np.array_equal(host(gv), wv)
    assert np.array_equal(host(gk).view(np.uint32), wk.view(np.uint32))
    big = _sorted_keys("i32", 100001, 3)
    d = dev(np.concatenate([np.zeros(1, np.int32), big]))[1:]  # 4-byte offset: unaligned for 16-byte stores
    out = torch.empty(2 * 100001 + 1, dtype=torch.int32, device=cuda)[1:]
    bulk_b200.merge(d, d, out=out)
    assert np.array_equal(host(out), oracle.merge(big, big))


@pytest.mark.slow
def test_full_size_config_2x2_26_f32_u32(cuda):
    """The benchmark configuration: A, B = 2^26 float32 U[0,1) each (~1% cross
    duplicates), payloads A = i, B = 2^26 + i.  Size-independent properties:
    the (key, source, index) sequence is strictly increasing (stable merge
    order, which with unique payloads also makes it a permutation), and every
    key equals its source element."""
    n = 1 << 26
    a = _sorted_keys("f32", n, 1)
    b = _sorted_keys("f32", n, 2, dup_from=a)
    da, db = dev(a), dev(b)
    av = torch.arange(n, dtype=torch.int32, device=cuda)
    bv = av + n
    k, v = bulk_b200.merge(da, db, av, bv)
    from_a = v < n
    src_key = torch.where(from_a, da[v.clamp(max=n - 1)], db[(v - n).clamp(min=0)])
    assert torch.equal(k, src_key)
    kk = k.double()
    nondecreasing = (kk[1:] > kk[:-1]) | ((kk[1:] == kk[:-1]) & (v[1:] > v[:-1]))
    assert bool(nondecreasing.all())
    assert int(from_a.sum()) == n
    # and element by element against the oracle's stable merge
    wk, wv = oracle.merge(a, b, np.arange(n, dtype=np.uint32), np.arange(n, 2 * n, dtype=np.uint32))
    assert np.array_equal(host(k), wk) and np.array_equal(host(v).view(np.uint32), wv)
