"""Measure the launch-shape table the library compiles in (bulk_b200/csrc/tuning_table.inc).

For each op, element size and size class, every candidate shape is set
through bk_tune_override, the op is timed on one B200 with CUDA events
(median of 5 after 2 warm-up calls; a size class is represented by one n:
2^15, 2^19, 2^23 and 2^26 elements), and the fastest shape is kept when it
beats the op's default shape by more than 3 % (otherwise the default stays:
smaller differences are run-to-run noise).  The
table and the timings behind it go to bulk_b200/csrc/tuning_table.inc (C++
initialisers, compiled into libbulkb200.so) and bulk_b200/tuning_table.json
(provenance: device, date, every candidate's time).  Rebuild the library
afterwards (python bulk_b200/build.py).

Usage (on a GPU machine): python bulk_b200/tune.py [--quick]
        python bulk_b200/tune.py --from-json   (rewrite the .inc from the recorded timings)
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys
import time
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

OPS = {"reduce": 0, "scan": 1, "reduce_by_key": 2, "merge": 3, "sort": 4}
# the library's defaults (bk_tune.hpp default_knobs)
DEFAULT = {"reduce": (4, 0), "scan": (2, 0), "reduce_by_key": (3, 0), "merge": (3, 0), "sort": (1, 1)}
# the kernel caps reduce_by_key at two CTAs per SM unless key and value are 4 bytes each
DEFAULT_FOR = {("reduce_by_key", 12): (2, 0)}
MARGIN = 0.03


def choose(op, res, default=None):
    """The fastest shape if it beats the default by more than MARGIN, else the default."""
    default = default or DEFAULT[op]
    best = min(res, key=lambda r: r[1])
    dflt = [t for shape, t in res if shape == default]
    if dflt and best[1] > dflt[0] * (1.0 - MARGIN):
        return default
    return best[0]
CLASS_N = [1 << 15, 1 << 19, 1 << 23, 1 << 26]
# (op, label, element bytes, candidate (ctas_per_sm, prefetch) shapes)
PLAN = [
    ("reduce", "f32", 4, [(1, 0), (2, 0), (4, 0), (8, 0)]),
    ("reduce", "f64", 8, [(1, 0), (2, 0), (4, 0), (8, 0)]),
    ("scan", "f32", 4, [(1, 0), (2, 0)]),
    ("scan", "f64", 8, [(1, 0), (2, 0)]),
    ("reduce_by_key", "i32/f32", 8, [(1, 0), (2, 0), (3, 0)]),
    ("reduce_by_key", "i32/f64", 12, [(1, 0), (2, 0)]),
    ("merge", "f32/u32", 8, [(1, 0), (2, 0), (3, 0)]),
    ("sort", "u32/u32", 8, [(1, 0), (1, 1), (1, 2)]),
    ("sort", "u64/u32", 12, [(1, 0), (1, 1), (1, 2)]),
]


def _inputs(op, label, n, dev):
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    if op in ("reduce", "scan"):
        dt = torch.float32 if label == "f32" else torch.float64
        x = torch.rand(n, generator=g, device=dev, dtype=dt)
        return {"x": x, "out": torch.empty_like(x), "r": torch.empty(1, dtype=dt, device=dev)}
    if op == "reduce_by_key":
        dt = torch.float32 if label.endswith("f32") else torch.float64
        keys = torch.sort(torch.randint(0, max(1, n // 16), (n,), generator=g, device=dev, dtype=torch.int32)).values
        vals = torch.rand(n, generator=g, device=dev, dtype=dt)
        return {"k": keys, "v": vals, "ok": torch.empty(n, dtype=torch.int32, device=dev),
                "ov": torch.empty(n, dtype=dt, device=dev), "c": torch.empty(1, dtype=torch.int64, device=dev)}
    if op == "merge":
        a = torch.sort(torch.rand(n // 2, generator=g, device=dev)).values
        b = torch.sort(torch.rand(n - n // 2, generator=g, device=dev)).values
        av = torch.arange(a.numel(), dtype=torch.int32, device=dev)
        bv = torch.arange(b.numel(), dtype=torch.int32, device=dev)
        return {"a": a, "b": b, "av": av, "bv": bv, "o": torch.empty(n, device=dev),
                "ov": torch.empty(n, dtype=torch.int32, device=dev)}
    kt = torch.int32 if label.startswith("u32") else torch.int64
    k0 = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=dev, dtype=torch.int32).to(kt)
    return {"k0": k0, "v0": torch.arange(n, dtype=torch.int32, device=dev), "k": k0.clone(),
            "v": torch.zeros(n, dtype=torch.int32, device=dev)}


def _call(op, d):
    import bulk_b200
    if op == "reduce":
        bulk_b200.reduce(d["x"], 0, out=d["r"])
    elif op == "scan":
        bulk_b200.inclusive_scan(d["x"], 0, out=d["out"])
    elif op == "reduce_by_key":
        bulk_b200.reduce_by_key(d["k"], d["v"], d["ok"], d["ov"], d["c"], sync=False)
    elif op == "merge":
        bulk_b200.merge(d["a"], d["b"], d["av"], d["bv"], out=d["o"], out_vals=d["ov"])
    else:
        d["k"].copy_(d["k0"])
        d["v"].copy_(d["v0"])
        bulk_b200.stable_sort_by_key(d["k"], d["v"])


def _time(op, d, reps, inner):
    import torch
    for _ in range(2):
        _call(op, d)
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(inner):
            _call(op, d)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / inner)
    return statistics.median(times)


def tune(quick=False):
    import torch

    import bulk_b200
    from bulk_b200 import _lib
    lib = bulk_b200.lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    entries, record = [], []
    for op, label, eb, cands in PLAN:
        for sc, n in enumerate(CLASS_N):
            if quick and sc != 3:
                continue
            d = _inputs(op, label, n, dev)
            inner = 20 if n <= (1 << 19) else 1
            res = []
            for c, pf in cands:
                _lib.check(lib.bk_tune_override(OPS[op], eb, sc, c, pf), "bk_tune_override")
                res.append(((c, pf), _time(op, d, 5, inner)))
            _lib.check(lib.bk_tune_override(OPS[op], eb, sc, 0, 0), "bk_tune_override")
            best = choose(op, res, DEFAULT_FOR.get((op, eb)))
            entries.append((OPS[op], eb, sc, best))
            record.append({"op": op, "dtype": label, "elem_bytes": eb, "size_class": sc, "n": n,
                           "candidates_ms": {f"ctas{c}_pf{pf}": t for (c, pf), t in res},
                           "chosen": {"ctas_per_sm": best[0], "prefetch": best[1]}})
            print(f"{op:14s} {label:8s} n=2^{n.bit_length() - 1:<2d} " +
                  " ".join(f"{c}/{pf}:{t:.4f}" for (c, pf), t in res) + f"  -> {best}", flush=True)
            del d
            torch.cuda.empty_cache()
    props = torch.cuda.get_device_properties(dev)
    prov = {"device": props.name, "sms": props.multi_processor_count,
            "date_utc": time.strftime("%Y-%m-%d %H:%M", time.gmtime()),
            "procedure": ("bulk_b200/tune.py: median of 5 timed calls (CUDA events) after 2 warm-up calls per "
                          f"shape; the default shape stays unless another is more than {MARGIN:.0%} faster"),
            "cells": record}
    write_table(prov, entries)
    return entries


def write_table(prov, entries):
    names = {v: k for k, v in OPS.items()}
    lines = ["// Launch-shape table: {op, element bytes, size class, {ctas_per_sm, prefetch}}.",
             f"// Measured by bulk_b200/tune.py on {prov['device']} ({prov['sms']} SMs), "
             f"{prov['date_utc']} UTC; timings in bulk_b200/tuning_table.json."]
    for op, eb, sc, (c, pf) in entries:
        lines.append(f"{{bk::tune::k{''.join(w.capitalize() for w in names[op].split('_'))}, {eb}, {sc}, {{{c}, {pf}}}}},")
    (PKG / "csrc" / "tuning_table.inc").write_text("\n".join(lines) + "\n")
    (PKG / "tuning_table.json").write_text(json.dumps(prov, indent=1) + "\n")


def from_json():
    """Re-choose every cell from the recorded candidate timings and rewrite both files."""
    prov = json.loads((PKG / "tuning_table.json").read_text())
    entries = []
    for cell in prov["cells"]:
        res = []
        for key, t in cell["candidates_ms"].items():
            c, pf = key.replace("ctas", "").split("_pf")
            res.append(((int(c), int(pf)), t))
        best = choose(cell["op"], res, DEFAULT_FOR.get((cell["op"], cell["elem_bytes"])))
        cell["chosen"] = {"ctas_per_sm": best[0], "prefetch": best[1]}
        entries.append((OPS[cell["op"]], cell["elem_bytes"], cell["size_class"], best))
    prov["procedure"] = ("bulk_b200/tune.py: median of 5 timed calls (CUDA events) after 2 warm-up calls per "
                         f"shape; the default shape stays unless another is more than {MARGIN:.0%} faster")
    write_table(prov, entries)
    return entries


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--quick", action="store_true", help="the largest size class only")
    ap.add_argument("--from-json", action="store_true", help="rewrite the table from the recorded timings")
    a = ap.parse_args(argv)
    if a.from_json:
        from_json()
    else:
        tune(a.quick)
    return 0


if __name__ == "__main__":
    sys.exit(main())
