"""Generate tests/golden/reference_outputs.json from the reference itself.

Runs the reference's own algorithms compiled for the host
(oracle/_ref/libbulkref.so, built by oracle/ref/build_ref.py from the
reference sources) on the reference drivers' known-answer inputs and records
their outputs: scalars as values, arrays as SHA-256 digests of their bytes
(inputs are regenerated from the recorded recipe, so nothing large is stored).

Usage (needs the reference sources to build the library):
    python oracle/ref/build_ref.py && python tests/golden/gen_golden.py
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import reference as R  # noqa: E402
from tests.sizes import reference_sizes  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_outputs.json"


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libbulkref.so is missing: run oracle/ref/build_ref.py first")
    g = {"generator": "tests/golden/gen_golden.py", "reference": "jaredhoberock/bulk compiled for the host"}
    # reduce.cu:132-148 -- sequence(0..n-1), init 13 (int wraps)
    g["reduce_sequence_init13"] = [{"n": n, "out": int(R.cpu_reduce(np.arange(n, dtype=np.int32), 13))}
                                   for n in (1, 1000, 123456789)]
    # scan.cu:158-184 -- all ones, init 13, the drivers' size schedule (device-style three-pass scan)
    g["scan_ones_init13"] = [{"n": n, "sha256": digest(R.cpu_inclusive_scan(np.ones(n, np.int32), 13))}
                             for n in reference_sizes()]
    # reduce + scan of i32 U[-1000,1000] (oracle.gen seed = n) through the group algorithms
    g["group_reduce_scan_i32"] = []
    for n in (1, 5, 12, 13, 1000, 4097):
        x = oracle.gen(np.int32, n, n, -1000, 1000)
        g["group_reduce_scan_i32"].append({"n": n, "seed": n, "init": 13, "reduce": int(R.group_reduce(x, 13)),
                                           "scan_sha256": digest(R.group_inclusive_scan(x, 13))})
    # merge.cu:258-278 -- hash-filled halves, each sorted, merged
    g["merge_hash_fill"] = []
    for n in (2, 1000, 123457, 1 << 20):
        a = np.sort(oracle.ref_hash_fill_i32(n // 2), kind="stable")
        g["merge_hash_fill"].append({"n": n, "sha256": digest(R.merge(a, a.copy()))})
    # reduce_by_key.cu:364-402 -- keys = values = hash(i) % 10
    g["reduce_by_key_hash_mod10"] = []
    for n in (1, 2, 13, 1024, 19999, 40000):
        k = oracle.ref_hash_fill_i32(n, 10)
        rk, rv = R.group_reduce_by_key(k, k)
        g["reduce_by_key_hash_mod10"].append({"n": n, "count": int(rk.size), "keys_sha256": digest(rk),
                                              "values_sha256": digest(rv)})
    # the bounded group block sort and merge_by_key on small tiles (stability, A-first ties)
    g["group_sort_tiles"] = []
    for seed in range(40):
        n = 1 + seed % 12
        keys = (oracle.gen(np.uint32, n, seed) % 4).astype(np.int32)
        gk, gv = R.group_stable_sort_by_key(keys, np.arange(n, dtype=np.int32))
        g["group_sort_tiles"].append({"keys": keys.tolist(), "sorted_keys": gk.tolist(), "sorted_vals": gv.tolist()})
    g["group_merge_tiles"] = []
    for seed in range(40):
        na, nb = seed % 7, min(12 - seed % 7, (seed // 7) % 7)
        a = np.sort((oracle.gen(np.uint32, na, seed) % 5).astype(np.int32))
        b = np.sort((oracle.gen(np.uint32, nb, seed + 1) % 5).astype(np.int32))
        gk, gv = R.group_merge_by_key(a, np.arange(na, dtype=np.int32), b, np.arange(100, 100 + nb, dtype=np.int32))
        g["group_merge_tiles"].append({"a": a.tolist(), "b": b.tolist(), "keys": gk.tolist(), "vals": gv.tolist()})
    OUT.write_text(json.dumps(g, indent=1) + "\n")
    print(OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
