"""The per-device set-up cache behind every kernel's shared-memory opt-in
(bulk_b200/csrc/bk_host_cache.hpp), checked on the CPU: set-up runs once per
(device, call site), a second device is set up again, failures are not
cached, and concurrent first calls run set-up once."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_per_device_cache(tmp_path):
    exe = tmp_path / "host_cache_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", f"-I{ROOT / 'bulk_b200' / 'csrc'}",
                    str(ROOT / "tests" / "host" / "host_cache_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
