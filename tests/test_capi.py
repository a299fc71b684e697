"""The C-ABI library loads on a CPU-only machine and exports every declared entry point."""
from __future__ import annotations

import ctypes
import re
import subprocess

import bulk_b200
from bulk_b200 import _lib


def test_header_parses_and_every_symbol_is_exported():
    decls = _lib.parse_header()
    assert len(decls) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s(bk_\w+)", out))
    missing = sorted(set(decls) - exported)
    assert not missing, f"declared but not exported: {missing}"
    extra = sorted(n for n in exported - set(decls))
    assert not extra, f"exported but not declared in include/bulk_b200.h: {extra}"


def test_ctypes_binding_matches_header():
    for name, (res, args) in _lib.DECLS.items():
        fn = getattr(bulk_b200.lib, name)
        assert fn.argtypes == args, name


def test_status_strings_and_version():
    lib = bulk_b200.lib
    assert lib.bk_version() >= 10000
    for code in (0, -1, -2, -3, -4, -5, -6):
        assert lib.bk_status_string(code)
    assert lib.bk_status_string(-3) == b"device-side wait timed out"


def test_workspace_sizes_are_sane_without_a_device():
    ws = bulk_b200.workspace_bytes
    # scan: 256-byte header + one 8-byte status word per 8192-element tile
    assert ws("inclusive_scan", "f32", None, 1 << 28) == 256 + (1 << 28) // 8192 * 8
    assert ws("inclusive_scan", "f64", None, 1 << 28) > ws("inclusive_scan", "f32", None, 1 << 28)
    assert ws("reduce", "f32", None, 1 << 28) >= 256
    assert ws("reduce", "f32", "u32", 10) == 0          # reduce has no payload
    assert bulk_b200.lib.bk_workspace_bytes(99, 1, 0, 10) == 0


def test_invalid_workspace_init_is_rejected():
    assert bulk_b200.lib.bk_workspace_init(None, 1024, None) == _lib.BK_ERR_INVALID_ARGUMENT
    assert bulk_b200.lib.bk_workspace_status(None, 1024, None) == _lib.BK_ERR_INVALID_ARGUMENT
