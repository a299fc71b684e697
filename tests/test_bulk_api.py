"""The bulk:: C++ interface (include/bulk/*.hpp).

Without a GPU: every header compiles on its own for sm_100a, and the API
program tests/bulk_api/api_check.cu (the reference drivers' usage patterns plus
every agent- and group-level algorithm) compiles.  On a GPU: the program runs
and each of its checks against std:: algorithms passes.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
INCLUDE = ROOT / "include"
PROGRAM = ROOT / "tests" / "bulk_api" / "api_check.cu"
HEADERS = ["execution_policy.hpp", "future.hpp", "malloc.hpp", "async.hpp", "algorithm.hpp",
           "iterator.hpp", "uninitialized.hpp", "bulk.hpp"]
NVCC_FLAGS = ["-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-I", str(INCLUDE)]

needs_nvcc = pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not found")


def _nvcc(args, cwd):
    r = subprocess.run(["nvcc", *NVCC_FLAGS, *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


@pytest.fixture(scope="module")
def api_binary(tmp_path_factory):
    out = tmp_path_factory.mktemp("bulk_api") / "api_check"
    _nvcc(["-o", str(out), str(PROGRAM)], cwd=out.parent)
    return out


@needs_nvcc
@pytest.mark.parametrize("header", HEADERS)
def test_header_compiles_alone(header, tmp_path):
    src = tmp_path / "one.cu"
    src.write_text(f"#include <bulk/{header}>\nint main() {{ return 0; }}\n")
    _nvcc(["-c", "-o", str(tmp_path / "one.o"), str(src)], cwd=tmp_path)


@needs_nvcc
def test_api_program_compiles(api_binary):
    assert api_binary.exists()


@pytest.mark.gpu
@needs_nvcc
def test_api_program_runs(api_binary):
    r = subprocess.run([str(api_binary)], capture_output=True, text=True, timeout=180)
    lines = r.stdout.splitlines()
    failures = [ln for ln in lines if ln.startswith("FAIL")]
    assert not failures, "\n".join(failures) + "\n" + r.stderr
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert lines and lines[-1].startswith("PASSED")
    # every family of the interface was exercised
    text = r.stdout
    for name in ["hello_world", "saxpy", "sum con(512)", "futures", "choose_sizes default grid",
                 "default grid launches", "grid<128,4>", "group reduce n=",
                 "non-commutative", "group inclusive_scan", "group exclusive_scan", "group copy_n", "gather",
                 "scatter_if", "for_each_n", "adjacent_difference", "strided_iterator", "group merge na=",
                 "merge_by_key", "inplace_merge", "stable_sort_by_key", "group stable_sort n=",
                 "group reduce_by_key", "group malloc", "uninitialized", "agent bounded reduce",
                 "agent bounded merge_by_key", "cluster group reduce (4 CTAs", "cluster group reduce non-commutative",
                 "grid of clusters reduce", "block in the peer CTA's shared memory (DSMEM)",
                 "errors raise thrust::system_error"]:
        assert name in text, name
