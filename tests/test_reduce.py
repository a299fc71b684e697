"""GPU parity of bk_reduce_* against the oracle (reduce.cu:58-97 semantics).

Integer results are bit-exact (wrapping); float sums stay within
|err| <= 2*ceil(log2 n)*eps*sum|x| of the long-double oracle.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import bulk_b200
import oracle
from tests.gpu_util import NP, assert_within_bound, dev, gen, host
from tests.sizes import EDGE_SIZES, reference_sizes

pytestmark = pytest.mark.gpu
TAGS = ["i32", "u32", "i64", "u64", "f32", "f64"]


def _check(tag, op, x, init, got):
    if tag in ("f32", "f64") and op == "sum":
        ref, mag = oracle.reduce(x, NP[tag](init))
        assert_within_bound(got, ref, mag, max(x.size, 1), NP[tag], f"reduce {tag} n={x.size}")
    else:
        assert got == oracle.reduce(x, NP[tag](init), op), f"reduce_{op}_{tag} n={x.size}"


def test_known_answer_sequence_init13(cuda):
    # reduce.cu:132-148: thrust::sequence over n = 123456789 ints, init 13
    n = 123456789
    x = torch.arange(n, dtype=torch.int32, device=cuda)
    got = int(bulk_b200.reduce(x, 13).item())
    want = (13 + n * (n - 1) // 2) % (1 << 32)
    assert got == (want - (1 << 32) if want >= (1 << 31) else want)


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("op", ["sum", "min", "max"])
def test_edge_sizes(cuda, tag, op):
    for i, n in enumerate(EDGE_SIZES):
        x = gen(tag, n, 100 + i)
        init = NP[tag](7 if tag not in ("f32", "f64") else 0.25)
        got = host(bulk_b200.reduce(dev(x), init, op))[0]
        _check(tag, op, x, init, got)


@pytest.mark.parametrize("tag", ["i32", "f32", "f64"])
def test_reference_size_schedule(cuda, tag):
    for n in reference_sizes():
        x = gen(tag, n, n)
        got = host(bulk_b200.reduce(dev(x), NP[tag](13)))[0]
        _check(tag, "sum", x, 13, got)


@pytest.mark.parametrize("tag", ["i32", "f32", "i64", "f64"])
@pytest.mark.parametrize("offset", [1, 2, 3])
def test_misaligned_input(cuda, tag, offset):
    n = 100000
    x = gen(tag, n + offset, 9)
    d = dev(x)[offset:]
    got = host(bulk_b200.reduce(d, NP[tag](0)))[0]
    _check(tag, "sum", x[offset:], 0, got)


def test_float_result_is_reproducible(cuda):
    x = dev(gen("f32", (1 << 24) + 123, 4))
    a = [host(bulk_b200.reduce(x, np.float32(0)))[0] for _ in range(5)]
    assert len({float(v).hex() for v in a}) == 1
    assert bulk_b200.workspace_status() == 0


@pytest.mark.slow
@pytest.mark.parametrize("tag", ["i32", "f32", "f64"])
def test_full_size_2_28(cuda, tag):
    # the benchmark configuration: N = 2^28, f32/f64 U[-1,1], i32 U[-100,100]
    n = 1 << 28
    x = dev(gen(tag, n, 0))
    got = host(bulk_b200.reduce(x, NP[tag](0)))[0]
    if tag == "i32":
        want = int(x.to(torch.int64).sum().item()) % (1 << 32)
        assert int(np.int64(got)) % (1 << 32) == want
    else:
        ref = float(x.double().sum().item())
        mag = float(x.double().abs().sum().item())
        assert_within_bound(got, ref, mag, n, NP[tag], "2^28")
    assert bulk_b200.workspace_status() == 0
