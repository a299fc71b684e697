"""Build the oracle (test infrastructure) into oracle/lib/liboracle.so with gcc.

The oracle is the CPU restatement used by tests/, smoke() and bench.py's CPU
baseline to check the CUDA library; the product never loads it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle.so"
SRC = [HERE / "oracle.c"]


def build(force: bool = False) -> Path:
    LIB.parent.mkdir(exist_ok=True)
    deps = SRC + [HERE / "oracle.h", Path(__file__)]
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [os.environ.get("CC", "gcc"), "-O2", "-std=gnu11", "-fPIC", "-shared", "-Wall",
           "-o", str(tmp), *map(str, SRC), "-lm", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
