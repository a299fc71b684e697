"""Size schedules of the reference drivers' validation loops.

scan.cu:214-229, merge_sort_by_key.cu:365-380 and reduce_by_key.cu:405-420 test
n = 1, 2, 4, ..., 2^20 and then 20 sizes ``rng() % (1 << 20)`` drawn from a
default-constructed ``thrust::default_random_engine`` (minstd_rand: the
Lehmer generator x <- 48271 * x mod (2^31 - 1), seed 1).
"""
from __future__ import annotations


def minstd_rand(count: int, seed: int = 1) -> list[int]:
    out, x = [], seed
    for _ in range(count):
        x = (48271 * x) % 2147483647
        out.append(x)
    return out


def reference_sizes(max_log2: int = 20, include_random: bool = True, cap: int | None = None) -> list[int]:
    sizes = [1 << i for i in range(max_log2 + 1)]
    if include_random:
        sizes += [r % (1 << 20) for r in minstd_rand(20)]
    if cap is not None:
        sizes = [s for s in sizes if s <= cap]
    return sizes


EDGE_SIZES = [0, 1, 2, 3, 4, 5, 7, 8, 15, 16, 17, 31, 32, 33, 255, 256, 257, 1023, 1024, 1025,
              2047, 2048, 2049, 4095, 4096, 4097, 8191, 8192, 8193, 65535, 65536, 65537,
              (1 << 20) - 1, (1 << 20) + 1]
