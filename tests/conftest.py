"""Shared pytest configuration.

Markers: ``gpu`` = needs a CUDA device (B200).  ``-m "not gpu"`` runs the oracle
checks, host logic and C-ABI export checks on a CPU-only machine.
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# Build the library in-tree when it is missing and nvcc is available (CPU
# container); on a GPU machine the prebuilt library is used as shipped.
_lib = ROOT / "bulk_b200" / "lib" / "libbulkb200.so"
if not _lib.exists() and shutil.which("nvcc"):
    import importlib.util
    _spec = importlib.util.spec_from_file_location("bulk_b200_build_script", ROOT / "bulk_b200" / "build.py")
    _mod = importlib.util.module_from_spec(_spec)
    _spec.loader.exec_module(_mod)
    _mod.build()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size (2^26-2^28 element) property tests")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
