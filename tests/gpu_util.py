"""Helpers shared by the GPU parity tests (host <-> device copies and the
floating-point tolerance check)."""
from __future__ import annotations

import numpy as np
import torch

import oracle

NP = {"i32": np.int32, "u32": np.uint32, "i64": np.int64, "u64": np.uint64, "f32": np.float32, "f64": np.float64}


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy()


def gen(tag: str, n: int, seed: int) -> np.ndarray:
    """Inputs in the ranges of the benchmark configurations."""
    dt = NP[tag]
    if tag == "i32":
        return oracle.gen(dt, n, seed, -100, 100)
    if tag == "i64":
        return oracle.gen(np.int32, n, seed, -(1 << 30), 1 << 30).astype(np.int64) * 4099
    if tag == "u32":
        return oracle.gen(np.uint32, n, seed)
    if tag == "u64":
        return oracle.gen(np.uint64, n, seed)
    return oracle.gen(dt, n, seed, -1.0, 1.0)


def assert_within_bound(got, ref, abs_sum, n, dtype, what=""):
    """|got - ref| <= 2*ceil(log2 n)*eps*sum|x| elementwise (the stated tolerance)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    bound = oracle.fp_bound(n, dtype, abs_sum)
    err = np.abs(got - ref)
    bad = np.flatnonzero(err > bound)
    assert bad.size == 0, (f"{what}: {bad.size} elements beyond 2*ceil(log2 n)*eps*sum|x|; first at "
                           f"{bad[0]}: got {got.flat[bad[0]]!r} ref {ref.flat[bad[0]]!r} bound {np.broadcast_to(bound, err.shape).flat[bad[0]]!r}")
