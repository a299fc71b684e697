"""Build oracle/_ref/libbulkref.so: the reference's own algorithms compiled
for the host (TEST INFRASTRUCTURE ONLY -- the checker and the timed CPU
baseline; nothing in the product loads it).

The recipe compiles the reference's headers where they lie (the reference checkout,
read-only) after copying its bulk/ tree and decomposition.hpp into
oracle/_ref/src (a build folder, kept out of git) and applying two patches to
that copy:

* bulk/malloc.hpp: `extern __shared__ int s_data_segment_begin[]` becomes a
  plain `extern` declaration (the host harness defines the array);
* bulk/algorithm/detail/stable_merge_sort.hpp: the three barriers the block
  merge sort lacks (between reading the stage and overwriting it, and between
  writing values and gathering them) are added, without which a real
  thread-per-agent run corrupts keys.

Everything else is compiled as shipped, with g++ against the CUDA 12.9 Thrust
headers and a small compat shim (oracle/ref/shim) for Thrust names that newer
versions dropped.  Usage: python oracle/ref/build_ref.py [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ORACLE = HERE.parent
OUT = ORACLE / "_ref"
SRC = OUT / "src"
LIB = OUT / "libbulkref.so"
# the reference checkout: $BULK_REFERENCE, else the "reference" directory beside this repository
REFERENCE = Path(os.environ.get("BULK_REFERENCE", str(ORACLE.parent.parent / "reference")))
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

PATCHES = [
    ("bulk/malloc.hpp", "extern __shared__ int s_data_segment_begin[];", "extern int s_data_segment_begin[];"),
    ("bulk/algorithm/detail/stable_merge_sort.hpp",
     "  bulk::copy_n(bulk::bound<grainsize>(g.this_exec), stage.keys + local_offset, local_size, local_keys);\n",
     "  bulk::copy_n(bulk::bound<grainsize>(g.this_exec), stage.keys + local_offset, local_size, local_keys);\n"
     "  g.wait();\n"),
    ("bulk/algorithm/detail/stable_merge_sort.hpp",
     "                       gather_indices,\n                       comp);\n",
     "                       gather_indices,\n                       comp);\n    g.wait();\n"),
    ("bulk/algorithm/detail/stable_merge_sort.hpp",
     "    bulk::copy_n(bulk::bound<grainsize>(g.this_exec), local_values, local_size, stage.vals + local_offset);\n",
     "    bulk::copy_n(bulk::bound<grainsize>(g.this_exec), local_values, local_size, stage.vals + local_offset);\n"
     "    g.wait();\n"),
]


def available() -> bool:
    return (REFERENCE / "bulk" / "bulk.hpp").exists()


def _prepare_sources():
    if SRC.exists():
        shutil.rmtree(SRC)
    SRC.mkdir(parents=True)
    shutil.copytree(REFERENCE / "bulk", SRC / "bulk")
    shutil.copy2(REFERENCE / "decomposition.hpp", SRC / "decomposition.hpp")
    for rel, old, new in PATCHES:
        p = SRC / rel
        p.chmod(0o644)
        text = p.read_text()
        if text.count(old) != 1:
            raise RuntimeError(f"patch anchor not found exactly once in {rel}: {old[:60]!r}")
        p.write_text(text.replace(old, new))


def build(force: bool = False) -> Path | None:
    """Build the library; returns its path, or None when the reference is absent."""
    deps = [HERE / "ref_agent.cpp", HERE / "ref_group.cpp", Path(__file__)] + sorted((HERE / "shim").rglob("*.h"))
    if LIB.exists() and not force and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps):
        return LIB
    if not available():
        return LIB if LIB.exists() else None
    OUT.mkdir(exist_ok=True)
    _prepare_sources()
    common = ["g++", "-std=c++20", "-O2", "-fPIC", "-fvisibility=hidden", "-w",
              f"-I{HERE / 'shim'}", f"-I{SRC}", f"-I{CUDA / 'include'}", "-D__bulk_exec_check_disable__="]
    objs = []
    for name, extra in (("ref_agent", ["-include", "compat.h"]), ("ref_group", ["-include", "host_shared.h"])):
        obj = OUT / f"{name}.o"
        subprocess.run(common + extra + ["-c", str(HERE / f"{name}.cpp"), "-o", str(obj)], check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-shared", "-o", str(tmp), *objs, f"-L{CUDA / 'lib64'}", "-lcudart", "-lpthread",
                    f"-Wl,-rpath,{CUDA / 'lib64'}"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
