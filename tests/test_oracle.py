"""Pin the oracle (CPU, no GPU) against the reference drivers' own known-answer
tests and an independent numpy restatement of each algorithm.

Reference known-answer tests reproduced here:
  reduce.cu:132-148          sequence(0..n-1), init 13, n = 123456789 (int wraps mod 2^32)
  scan.cu:158-184, 214-229   all-ones input, init 13, the drivers' size schedule
  merge.cu:258-278           hash-filled halves, each sorted, merged (== thrust::merge)
  merge_sort_by_key.cu:315-362  hash-filled keys and values, stable sort_by_key
  reduce_by_key.cu:364-402   keys = values = hash(i) % 10, reduce_by_key with ==, +
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from tests.sizes import minstd_rand, reference_sizes


def test_minstd_rand_matches_the_published_sequence():
    # minstd_rand (Park-Miller, multiplier 48271): 10000th value from seed 1 is
    # 399268537 (C++ standard [rand.predef]).
    x = minstd_rand(10000)
    assert x[0] == 48271
    assert x[-1] == 399268537


def test_reduce_known_answer_sequence_init13():
    n = 123456789
    x = np.arange(n, dtype=np.int32)
    got = oracle.reduce(x, 13)
    want = (13 + n * (n - 1) // 2) % (1 << 32)
    want = want - (1 << 32) if want >= (1 << 31) else want
    assert got == want


@pytest.mark.parametrize("n", reference_sizes())
def test_scan_known_answer_ones_init13(n):
    x = np.ones(n, dtype=np.int32)
    out = oracle.inclusive_scan(x, 13)
    assert np.array_equal(out, np.arange(14, 14 + n, dtype=np.int32))


def _np_merge(a, b, av=None, bv=None):
    # stable merge == stable sort of the concatenation (A's elements precede B's on ties)
    keys = np.concatenate([a, b])
    order = np.argsort(keys, kind="stable")
    if av is None:
        return keys[order]
    return keys[order], np.concatenate([av, bv])[order]


@pytest.mark.parametrize("n", [1, 2, 7, 1000, 123457, 1 << 20])
def test_merge_known_answer_hash_fill(n):
    a = np.sort(oracle.ref_hash_fill_i32(n // 2), kind="stable")
    b = np.sort(oracle.ref_hash_fill_i32(n // 2), kind="stable")
    assert np.array_equal(oracle.merge(a, b), _np_merge(a, b))


def test_merge_ties_take_a_first_and_merge_path():
    a = np.array([1, 2, 2, 5], dtype=np.float32)
    b = np.array([2, 2, 3], dtype=np.float32)
    av = np.arange(4, dtype=np.uint32)
    bv = np.arange(100, 103, dtype=np.uint32)
    k, v = oracle.merge(a, b, av, bv)
    assert k.tolist() == [1, 2, 2, 2, 2, 3, 5]
    assert v.tolist() == [0, 1, 2, 100, 101, 102, 3]
    # merge_path(diag) = number of A elements among the first diag outputs
    for diag in range(8):
        assert oracle.merge_path(a, b, diag) == int(np.sum(v[:diag] < 100))


@pytest.mark.parametrize("n", reference_sizes(max_log2=16, include_random=False) + [12345, 99999])
def test_stable_sort_by_key_known_answer_hash_fill(n):
    keys = oracle.ref_hash_fill_i32(n)
    vals = oracle.ref_hash_fill_i32(n)
    k, v = oracle.stable_sort_by_key(keys, vals)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order])
    assert np.array_equal(v, vals[order])


@pytest.mark.parametrize("dtype", [np.uint32, np.uint64, np.float32, np.float64, np.int64])
def test_stable_sort_payload_index_is_stable(dtype):
    n = 50000
    if dtype == np.uint32:
        keys = oracle.gen(np.uint32, n, 3) >> np.uint32(20)   # many duplicates
    elif dtype == np.uint64:
        keys = oracle.gen(np.uint64, n, 4) >> np.uint64(50)
    elif dtype == np.int64:
        keys = (oracle.gen(np.uint64, n, 4) >> np.uint64(50)).astype(np.int64) - 5000
    else:
        keys = np.floor(oracle.gen(dtype, n, 5, 0.0, 100.0))
    idx = np.arange(n, dtype=np.uint32)
    k, v = oracle.stable_sort_by_key(keys, idx)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, order.astype(np.uint32))


def _np_rbk(keys, vals):
    heads = np.ones(keys.size, dtype=bool)
    heads[1:] = keys[1:] != keys[:-1]
    starts = np.flatnonzero(heads)
    sums = np.add.reduceat(vals.astype(np.int64), starts) if keys.size else np.zeros(0, np.int64)
    return keys[starts], sums


@pytest.mark.parametrize("n", reference_sizes(max_log2=18, include_random=False) + [19999, 20000, 20001])
def test_reduce_by_key_known_answer_hash_mod10(n):
    keys = oracle.ref_hash_fill_i32(n, 10)
    vals = keys.copy()
    k, v = oracle.reduce_by_key(keys, vals)
    wk, wv = _np_rbk(keys, vals)
    assert np.array_equal(k, wk)
    assert np.array_equal(v, wv.astype(np.int32))


def test_reference_hash_is_the_64bit_index_form():
    # the hash mixes a 64-bit ptrdiff_t index; the values must stay nonnegative
    h = [oracle.ref_hash(i) for i in range(1000)]
    assert all(x >= 0 for x in h)
    assert len(set(x % 10 for x in h)) == 10


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_float_reduce_and_scan_against_fsum(dtype):
    n = 100003
    x = oracle.gen(dtype, n, 0, -1.0, 1.0)
    got, mag = oracle.reduce(x, dtype(0.5))
    assert abs(got - math.fsum([0.5] + x.astype(np.float64).tolist())) <= 1e-9 * mag
    pref, pmag = oracle.inclusive_scan(x[:2000], dtype(0.5))
    want = np.cumsum(np.concatenate([[0.5], x[:2000].astype(np.float64)]))[1:]
    assert np.allclose(pref, want, rtol=0, atol=1e-12)
    assert np.all(np.diff(pmag) >= 0)


def test_generators_ranges_and_determinism():
    a = oracle.gen(np.int32, 100000, 0, -1000, 1000)
    assert a.min() == -1000 and a.max() == 1000
    assert np.array_equal(a, oracle.gen(np.int32, 100000, 0, -1000, 1000))
    f = oracle.gen(np.float32, 100000, 1, -1.0, 1.0)
    assert f.min() >= -1.0 and f.max() < 1.0
    g = oracle.gen_runs_geometric(1 << 20, 5, 16.0)
    runs = np.count_nonzero(np.diff(g)) + 1
    assert 14.0 < (1 << 20) / runs < 18.0 and np.all(np.diff(g) >= 0)
    z = oracle.gen_runs_zipf(1 << 20, 6, 1.2, 1 << 20)
    assert np.all(np.diff(z) >= 0)


def test_fp_bound():
    assert oracle.fp_bound(1 << 28, np.float32, 1.0) == pytest.approx(2 * 28 * 2.0 ** -23)


# ---------------------------------------------------------------------------
# Golden fixtures recorded from the reference itself (tests/golden/gen_golden.py)
import hashlib  # noqa: E402
import json  # noqa: E402
from pathlib import Path  # noqa: E402

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "reference_outputs.json").read_text())


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_golden_reduce_and_scan():
    for c in GOLDEN["reduce_sequence_init13"]:
        assert oracle.reduce(np.arange(c["n"], dtype=np.int32), 13) == c["out"]
    for c in GOLDEN["scan_ones_init13"]:
        assert _sha(oracle.inclusive_scan(np.ones(c["n"], np.int32), 13)) == c["sha256"], c["n"]
    for c in GOLDEN["group_reduce_scan_i32"]:
        x = oracle.gen(np.int32, c["n"], c["seed"], -1000, 1000)
        assert oracle.reduce(x, c["init"]) == c["reduce"]
        assert _sha(oracle.inclusive_scan(x, c["init"])) == c["scan_sha256"]


def test_golden_merge_and_reduce_by_key():
    for c in GOLDEN["merge_hash_fill"]:
        a = np.sort(oracle.ref_hash_fill_i32(c["n"] // 2), kind="stable")
        assert _sha(oracle.merge(a, a.copy())) == c["sha256"], c["n"]
    for c in GOLDEN["reduce_by_key_hash_mod10"]:
        k = oracle.ref_hash_fill_i32(c["n"], 10)
        wk, wv = oracle.reduce_by_key(k, k)
        assert wk.size == c["count"] and _sha(wk) == c["keys_sha256"] and _sha(wv) == c["values_sha256"]


def test_golden_group_sort_and_merge_tiles():
    for c in GOLDEN["group_sort_tiles"]:
        keys = np.array(c["keys"], np.int32)
        wk, wv = oracle.stable_sort_by_key(keys, np.arange(keys.size, dtype=np.int32))
        assert wk.tolist() == c["sorted_keys"] and wv.tolist() == c["sorted_vals"]
    for c in GOLDEN["group_merge_tiles"]:
        a, b = np.array(c["a"], np.int32), np.array(c["b"], np.int32)
        wk, wv = oracle.merge(a, b, np.arange(a.size, dtype=np.int32), np.arange(100, 100 + b.size, dtype=np.int32))
        assert wk.tolist() == c["keys"] and wv.tolist() == c["vals"]
