"""Pin the oracle against the reference itself (CPU, no GPU).

oracle/_ref/libbulkref.so is the reference's own code compiled for the host
(oracle/ref/build_ref.py): its agent-level algorithms driven over the
device-wide drivers' decompositions, and its cooperative group algorithms run
with one host thread per agent.  Both must agree with the oracle on the
reference drivers' own known-answer inputs.  Skipped when the reference
library was not built.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import reference as R
from tests.sizes import reference_sizes

pytestmark = pytest.mark.skipif(not R.available(), reason="host-compiled reference not built")


def test_reduce_sequence_init13_wraps_like_the_reference():
    n = 123456789  # reduce.cu:132-148
    x = np.arange(n, dtype=np.int32)
    assert R.cpu_reduce(x, 13) == oracle.reduce(x, 13)


@pytest.mark.parametrize("n", [1, 2, 3, 895, 896, 897, 100003, 1 << 22])
def test_reduce_and_scan_device_decomposition(n):
    x = oracle.gen(np.int32, n, n, -1000, 1000)
    assert R.cpu_reduce(x, 7) == oracle.reduce(x, 7)
    assert np.array_equal(R.cpu_inclusive_scan(x, 7), oracle.inclusive_scan(x, 7))


def test_scan_ones_init13_schedule():
    for n in reference_sizes():  # scan.cu:158-184, 214-229
        x = np.ones(n, dtype=np.int32)
        assert np.array_equal(R.cpu_inclusive_scan(x, 13), oracle.inclusive_scan(x, 13)), n


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_float_reduce_and_scan_within_the_bound(dtype):
    n = 1 << 20
    x = oracle.gen(dtype, n, 3, -1.0, 1.0)
    ref, mag = oracle.reduce(x, dtype(0))
    assert abs(float(R.cpu_reduce(x, dtype(0))) - ref) <= oracle.fp_bound(n, dtype, mag)
    pref, pmag = oracle.inclusive_scan(x, dtype(0))
    got = R.cpu_inclusive_scan(x, dtype(0)).astype(np.float64)
    assert np.all(np.abs(got - pref) <= oracle.fp_bound(n, dtype, pmag))


@pytest.mark.parametrize("n", [2, 1000, 123457, 1 << 20])
def test_merge_hash_fill(n):
    a = np.sort(oracle.ref_hash_fill_i32(n // 2), kind="stable")  # merge.cu:258-278
    b = a.copy()
    assert np.array_equal(R.merge(a, b), oracle.merge(a, b))
    for diag in (0, 1, n // 3, n // 2, a.size + b.size):
        assert R.merge_path(a, b, diag) == oracle.merge_path(a, b, diag)


def test_merge_float_ties_take_a_first():
    a = np.floor(oracle.gen(np.float32, 5000, 1, 0.0, 100.0))
    b = np.floor(oracle.gen(np.float32, 7000, 2, 0.0, 100.0))
    a.sort(); b.sort()
    assert np.array_equal(R.merge(a, b), oracle.merge(a, b))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 8, 12, 1000, 19999, 40000])
def test_group_reduce_and_scan(n):
    x = oracle.gen(np.int32, n, 11 * n, -100, 100)
    assert R.group_reduce(x, 13) == oracle.reduce(x, 13)
    if n <= 20000:
        assert np.array_equal(R.group_inclusive_scan(x, 13), oracle.inclusive_scan(x, 13))


@pytest.mark.parametrize("n", [1, 2, 11, 12, 13, 1024, 19999, 40000])
def test_group_reduce_by_key_hash_mod10(n):
    keys = oracle.ref_hash_fill_i32(n, 10)  # reduce_by_key.cu:364-402
    rk, rv = R.group_reduce_by_key(keys, keys)
    wk, wv = oracle.reduce_by_key(keys, keys)
    assert np.array_equal(rk, wk) and np.array_equal(rv, wv)


def test_group_block_sort_is_stable():
    for seed in range(200):
        n = 1 + seed % 12
        keys = (oracle.gen(np.uint32, n, seed) % 4).astype(np.int32)
        vals = np.arange(n, dtype=np.int32)
        gk, gv = R.group_stable_sort_by_key(keys, vals)
        wk, wv = oracle.stable_sort_by_key(keys, vals)
        assert np.array_equal(gk, wk) and np.array_equal(gv, wv), seed


def test_group_merge_by_key_ties_take_a_first():
    for seed in range(200):
        na = seed % 7
        nb = min(12 - na, (seed // 7) % 7)
        a = np.sort((oracle.gen(np.uint32, na, seed) % 5).astype(np.int32))
        b = np.sort((oracle.gen(np.uint32, nb, seed + 1) % 5).astype(np.int32))
        av = np.arange(na, dtype=np.int32)
        bv = np.arange(100, 100 + nb, dtype=np.int32)
        gk, gv = R.group_merge_by_key(a, av, b, bv)
        wk, wv = oracle.merge(a, b, av, bv)
        assert np.array_equal(gk, wk) and np.array_equal(gv, wv), seed
