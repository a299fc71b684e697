"""The reference's own GPU benchmarks beside the library's, on one GPU.

Runs the reference's five drivers (built for sm_100a by
baseline/build_ref_gpu.py into baseline/_ref/gpu/), reads the times each
prints for its bulk implementation ("My time") and for Thrust ("Thrust's
time"), and times the library's public Python API on the same configuration:
the same element types and sizes, inputs of the same distributions (seeded
torch generators, not the drivers' hash: uniform keys for the sorts and
merges, sorted for the merge inputs, zeros for reduce and scan as the drivers
use, keys uniform in 0..9 for reduce_by_key as the drivers' hash mod 10
gives), and the drivers' timing: the mean of 50 calls (20 for the sort)
issued back to back between two CUDA events.  The library's calls leave
their results on the device; the reference's reduce and reduce_by_key read a
result back to the host in every call, by design of their interface.

Prints one JSON object: per configuration the three times in ms and the
library's speed-up over each.  Usage (on a GPU machine, after
python baseline/build_ref_gpu.py): python baseline/compare_gpu.py
"""
from __future__ import annotations

import json
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "baseline" / "_ref" / "gpu"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

TIME_RE = re.compile(r"^\s*(Thrust's time|My time):\s*([0-9.eE+-]+)\s*ms")


def run_driver(name: str, timeout: float = 900.0) -> str:
    p = subprocess.run([str(BIN / name)], capture_output=True, text=True, timeout=timeout, cwd=str(BIN))
    if p.returncode != 0:
        raise RuntimeError(f"{name} exited {p.returncode}: {p.stderr[-400:]}")
    return p.stdout


def parse(text: str) -> dict:
    """{label: {"thrust_ms": t, "reference_ms": m}}; a label is the section
    headings in force (e.g. "Large input / int", "64b float / N=134217728")."""
    out: dict = {}
    heads: list[str] = []
    for line in text.splitlines():
        s = line.strip()
        m = TIME_RE.match(line)
        if m:
            key = " / ".join(heads)
            out.setdefault(key, {})["thrust_ms" if m.group(1).startswith("Thrust") else "reference_ms"] = \
                float(m.group(2))
            continue
        if s.endswith(":") and not s.startswith("Testing"):
            label = s[:-1]
            if label in ("Large input", "Small input"):
                heads = [label]
            else:
                heads = [h for h in heads if h in ("Large input", "Small input")] + [label]
        elif s.startswith("N: "):
            heads = [h for h in heads if not h.startswith("N=")] + [f"N={s[3:]}"]
    return out


def _mean_ms(fn, calls: int) -> float:
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(calls):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / calls


def ours() -> dict:
    import torch
    import bulk_b200
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    res = {}
    for label, dt in (("int", torch.int32), ("long int", torch.int64), ("float", torch.float32),
                      ("double", torch.float64)):
        x = torch.zeros(1 << 28, dtype=dt, device=dev)
        o = torch.empty(1, dtype=dt, device=dev)
        res[f"reduce / {label}"] = _mean_ms(lambda: bulk_b200.reduce(x, 0, out=o), 50)
        del x
    for label, dt in (("32b int", torch.int32), ("64b float", torch.float64)):
        x = torch.zeros(1 << 27, dtype=dt, device=dev)
        res[f"scan / {label} / N={1 << 27}"] = _mean_ms(lambda: bulk_b200.inclusive_scan(x, 13, out=x), 50)
        del x
    n = 123456789
    for label, dt in (("int", torch.int32), ("float", torch.float32), ("double", torch.float64)):
        def sorted_half():
            if dt.is_floating_point:
                return torch.sort(torch.rand(n // 2, generator=g, device=dev, dtype=dt)).values
            return torch.sort(torch.randint(-(1 << 31), (1 << 31) - 1, (n // 2,), generator=g, device=dev,
                                            dtype=dt)).values
        a, b = sorted_half(), sorted_half()
        c = torch.empty(a.numel() + b.numel(), dtype=dt, device=dev)
        res[f"merge / Large input / {label}"] = _mean_ms(lambda: bulk_b200.merge(a, b, out=c), 50)
        del a, b, c
    n = 12345678
    for label, kdt, vdt in (("int", torch.int32, torch.int32), ("float", torch.float32, torch.int32),
                            ("double", torch.float64, torch.int64)):
        if kdt.is_floating_point:
            k0 = torch.rand(n, generator=g, device=dev, dtype=kdt)
        else:
            k0 = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=dev, dtype=kdt)
        v0 = torch.randint(-(1 << 31), (1 << 31) - 1, (n,), generator=g, device=dev, dtype=torch.int32).to(vdt)
        k, v = torch.empty_like(k0), torch.empty_like(v0)
        res[f"merge_sort_by_key / Large input / {label}"] = _mean_ms(
            lambda: bulk_b200.stable_sort_by_key_copy_batch([k0], [v0], [k], [v]), 20)
        del k0, v0, k, v
    for size_label, n in (("Large input", 12345678), ("Small input", 19999)):
        keys = torch.randint(0, 10, (n,), generator=g, device=dev, dtype=torch.int32)
        vals = torch.randint(0, 10, (n,), generator=g, device=dev, dtype=torch.int32)
        ok, ov = torch.empty_like(keys), torch.empty_like(vals)
        cnt = torch.empty(1, dtype=torch.int64, device=dev)
        res[f"reduce_by_key / {size_label} / int"] = _mean_ms(
            lambda: bulk_b200.reduce_by_key(keys, vals, ok, ov, cnt, sync=False), 50)
        del keys, vals, ok, ov
    return res


def main() -> int:
    ref = {}
    for name in ("reduce", "scan", "merge", "merge_sort_by_key", "reduce_by_key"):
        for label, t in parse(run_driver(name)).items():
            ref[f"{name} / {label}"] = t
    mine = ours()
    rows = {}
    for key, ms in mine.items():
        r = ref.get(key, {})
        row = {"ours_ms": ms, "reference_ms": r.get("reference_ms"), "thrust_ms": r.get("thrust_ms")}
        if row["reference_ms"]:
            row["speedup_vs_reference"] = row["reference_ms"] / ms
        if row["thrust_ms"]:
            row["speedup_vs_thrust"] = row["thrust_ms"] / ms
        rows[key] = row
    import torch
    print(json.dumps({"device": torch.cuda.get_device_name(0), "configs": rows,
                      "reference_sections": ref}, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
