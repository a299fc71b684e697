"""Build the reference's own device-wide drivers for sm_100a (the optional GPU
baseline: the reference's kernels on the same B200 as the library's).

The reference ships five benchmark drivers -- reduce.cu, scan.cu, merge.cu,
merge_sort_by_key.cu and reduce_by_key.cu -- each of which validates its bulk
implementation against Thrust and then prints "Thrust's time" and "My time"
(its bulk implementation) per configuration.  This recipe copies them, the
bulk/ tree and the helper headers from the reference checkout into
baseline/_ref/gpu/src (a build folder, git-ignored) and compiles each with
nvcc for sm_100a into baseline/_ref/gpu/<driver>.  Changes to the copy, all
needed to compile with CUDA 12.9 / Thrust 2.8, none to an algorithm:

* bulk/malloc.hpp: three lines hold their statement twice (a merge artefact;
  the second `void *result` is a redefinition), kept once;
* bulk/algorithm/detail/stable_merge_sort.hpp: the three barriers the block
  merge sort lacks (between reading the stage and overwriting it, and between
  writing values and gathering them), as for the host build of the oracle;
* merge.cu, merge_sort_by_key.cu: the comparison with moderngpu (the
  `sean_*` functions and their timing lines) is removed -- moderngpu is not
  vendored and not installed;
* merge_sort_by_key.cu: `locate_merge_path` initialises its
  `thrust::detail::wrapped_function` member with braces (the type is an
  aggregate in Thrust 2.8, with no converting constructor);
* compat headers written into baseline/_ref/gpu/shim: Thrust headers that
  newer Thrust renamed or dropped (forwarding headers), `thrust::detail::
  enable_if` and `remove_reference`, `__thrust_forceinline__`, and
  <thrust/host_vector.h>, which older Thrust pulled in with
  <thrust/device_vector.h>.

Usage: python baseline/build_ref_gpu.py [--force]   (nvcc only; no GPU needed)
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
OUT = ROOT / "baseline" / "_ref" / "gpu"
SRC = OUT / "src"
SHIM = OUT / "shim"
# the reference checkout: $BULK_REFERENCE, else the "reference" directory beside this repository
REFERENCE = Path(os.environ.get("BULK_REFERENCE", str(ROOT.parent / "reference")))
NVCC = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"
DRIVERS = ["reduce", "scan", "merge", "merge_sort_by_key", "reduce_by_key"]
HEADERS = ["decomposition.hpp", "head_flags.hpp", "tail_flags.hpp", "reduce_intervals.hpp", "join_iterator.hpp",
           "time_invocation_cuda.hpp"]

SORT_BARRIERS = [
    ("  bulk::copy_n(bulk::bound<grainsize>(g.this_exec), stage.keys + local_offset, local_size, local_keys);\n",
     "  bulk::copy_n(bulk::bound<grainsize>(g.this_exec), stage.keys + local_offset, local_size, local_keys);\n"
     "  g.wait();\n"),
    ("                       gather_indices,\n                       comp);\n",
     "                       gather_indices,\n                       comp);\n    g.wait();\n"),
    ("    bulk::copy_n(bulk::bound<grainsize>(g.this_exec), local_values, local_size, stage.vals + local_offset);\n",
     "    bulk::copy_n(bulk::bound<grainsize>(g.this_exec), local_values, local_size, stage.vals + local_offset);\n"
     "    g.wait();\n"),
]

SHIM_FILES = {
    "compat_gpu.h": """#pragma once
#include <cuda_runtime_api.h>
#include <thrust/detail/config.h>
#include <thrust/host_vector.h>
#include <type_traits>
#ifndef __thrust_forceinline__
#define __thrust_forceinline__ __forceinline__
#endif
THRUST_NAMESPACE_BEGIN
namespace detail {
template <bool B, class T = void>
struct enable_if : std::enable_if<B, T> {};
template <class T>
struct remove_reference : std::remove_reference<T> {};
}  // namespace detail
THRUST_NAMESPACE_END
""",
    "thrust/detail/swap.h": "#pragma once\n#include <thrust/swap.h>\n",
    "thrust/detail/util/blocking.h": "#pragma once\n#include <thrust/detail/config/compiler_fence.h>\n",
    "thrust/detail/cstdint.h": "#pragma once\n#include <cstdint>\n",
    "thrust/system/cuda/detail/guarded_cuda_runtime_api.h": "#pragma once\n#include <cuda_runtime_api.h>\n",
    "thrust/detail/type_traits/function_traits.h": """#pragma once
#include <thrust/detail/type_traits.h>
#include <thrust/detail/type_traits/has_nested_type.h>
#include <thrust/detail/type_traits/is_commutative.h>
THRUST_NAMESPACE_BEGIN
namespace detail {
__THRUST_DEFINE_HAS_NESTED_TYPE(has_result_type, result_type)
template <class F>
struct result_type { typedef typename F::result_type type; };
}  // namespace detail
THRUST_NAMESPACE_END
""",
    "thrust/iterator/detail/is_trivial_iterator.h": """#pragma once
#include <thrust/type_traits/is_contiguous_iterator.h>
THRUST_NAMESPACE_BEGIN
namespace detail {
template <class T>
struct is_trivial_iterator : thrust::is_contiguous_iterator<T> {};
}  // namespace detail
THRUST_NAMESPACE_END
""",
}


def available() -> bool:
    return (REFERENCE / "bulk" / "bulk.hpp").exists() and all((REFERENCE / f"{d}.cu").exists() for d in DRIVERS)


def _replace_once(path: Path, old: str, new: str):
    text = path.read_text()
    if text.count(old) != 1:
        raise RuntimeError(f"patch anchor not found exactly once in {path.name}: {old[:60]!r}")
    path.write_text(text.replace(old, new))


def _dedupe_doubled_lines(path: Path) -> int:
    """Lines that hold the same statement twice, tab-separated, keep one copy."""
    fixed = 0
    out = []
    for line in path.read_text().split("\n"):
        parts = [p for p in line.split("\t") if p.strip()]
        if "\t\t" in line and len(parts) == 2 and parts[0].strip() == parts[1].strip():
            line = parts[0]
            fixed += 1
        out.append(line)
    path.write_text("\n".join(out))
    return fixed


def _strip_moderngpu(path: Path):
    text = path.read_text()
    text = text.replace("#include <moderngpu.cuh>\n", "")
    # the sean_* comparison functions, then every line that times or prints them
    text, k = re.subn(r"template<typename T>\nvoid sean_\w+\(.*?\n}\n", "", text, flags=re.S)
    if k != 1:
        raise RuntimeError(f"expected one sean_* function in {path.name}, found {k}")
    text = "\n".join(l for l in text.split("\n") if "sean_" not in l and "Sean" not in l)
    path.write_text(text)


def prepare():
    if SRC.exists():
        shutil.rmtree(SRC)
    SRC.mkdir(parents=True)
    shutil.copytree(REFERENCE / "bulk", SRC / "bulk")
    for f in HEADERS + [f"{d}.cu" for d in DRIVERS]:
        shutil.copy2(REFERENCE / f, SRC / f)
    for p in SRC.rglob("*"):
        if p.is_file():
            p.chmod(0o644)
    if _dedupe_doubled_lines(SRC / "bulk" / "malloc.hpp") != 3:
        raise RuntimeError("expected three doubled lines in bulk/malloc.hpp")
    for old, new in SORT_BARRIERS:
        _replace_once(SRC / "bulk" / "algorithm" / "detail" / "stable_merge_sort.hpp", old, new)
    for d in ("merge", "merge_sort_by_key"):
        _strip_moderngpu(SRC / f"{d}.cu")
    # thrust::detail::wrapped_function is an aggregate now: brace-initialise it
    _replace_once(SRC / "merge_sort_by_key.cu", "      comp(comp)\n  {}", "      comp{comp}\n  {}")
    if SHIM.exists():
        shutil.rmtree(SHIM)
    for rel, text in SHIM_FILES.items():
        p = SHIM / rel
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_text(text)


def build(force: bool = False) -> list[Path]:
    """Compile every driver; returns the binaries (empty when the reference is absent)."""
    bins = [OUT / d for d in DRIVERS]
    if all(b.exists() for b in bins) and not force:
        return bins
    if not available():
        return [b for b in bins if b.exists()]
    OUT.mkdir(parents=True, exist_ok=True)
    prepare()
    flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-w", f"-I{SHIM}", f"-I{SRC}",
             "-include", "compat_gpu.h", "-D__bulk_exec_check_disable__="]
    procs = [(d, subprocess.Popen([str(NVCC), *flags, str(SRC / f"{d}.cu"), "-o", str(OUT / d)]))
             for d in DRIVERS]
    failed = [d for d, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    return bins


if __name__ == "__main__":
    for b in build(force="--force" in sys.argv):
        print(b)
