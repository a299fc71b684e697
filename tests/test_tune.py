"""The launch-shape table (bulk_b200/csrc/bk_tune.hpp, tuning_table.inc) and
its selection logic, through the C-ABI on the CPU: size classes, table cells,
defaults for missing cells, overrides and their bounds."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

import bulk_b200
from bulk_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
TABLE = ROOT / "bulk_b200" / "csrc" / "tuning_table.inc"
OPS = {"kReduce": 0, "kScan": 1, "kReduceByKey": 2, "kMerge": 3, "kSort": 4}
DEFAULTS = {0: (4, 0), 1: (2, 0), 2: (3, 0), 3: (3, 0), 4: (1, 1)}
CLASS_N = [1, (1 << 16) - 1, 1 << 16, (1 << 20) - 1, 1 << 20, (1 << 24) - 1, 1 << 24, 1 << 30]
CLASS_OF = [0, 0, 1, 1, 2, 2, 3, 3]


def lookup(op, eb, n):
    c, p = ctypes.c_int32(), ctypes.c_int32()
    st = bulk_b200.lib.bk_tune_lookup(op, eb, n, ctypes.byref(c), ctypes.byref(p))
    assert st == _lib.BK_OK
    return c.value, p.value


def table():
    cells = {}
    for m in re.finditer(r"\{bk::tune::(k\w+), (\d+), (\d), \{(\d+), (\d+)\}\},", TABLE.read_text()):
        cells[(OPS[m.group(1)], int(m.group(2)), int(m.group(3)))] = (int(m.group(4)), int(m.group(5)))
    return cells


def test_lookup_follows_the_table_and_defaults():
    cells = table()
    assert cells, "the table has at least one cell"
    for op in range(5):
        for eb in (4, 8, 12, 16):
            for n, sc in zip(CLASS_N, CLASS_OF):
                assert lookup(op, eb, n) == cells.get((op, eb, sc), DEFAULTS[op]), (op, eb, n)


def test_override_wins_then_clears():
    lib = bulk_b200.lib
    before = lookup(0, 4, 1 << 20)
    assert lib.bk_tune_override(0, 4, 2, 8, 0) == _lib.BK_OK
    assert lookup(0, 4, 1 << 20) == (8, 0)
    assert lookup(0, 4, 1 << 24) != (8, 0) or table().get((0, 4, 3)) == (8, 0)  # other cells untouched
    assert lib.bk_tune_override(0, 4, 2, 0, 0) == _lib.BK_OK
    assert lookup(0, 4, 1 << 20) == before


@pytest.mark.parametrize("args", [(5, 4, 0, 1, 0), (-1, 4, 0, 1, 0), (0, 17, 0, 1, 0), (0, 4, 4, 1, 0),
                                  (1, 4, 0, 3, 0), (2, 8, 0, 4, 0), (3, 8, 0, 4, 0), (4, 8, 0, 2, 0),
                                  (0, 4, 0, 1, 5)])
def test_override_bounds(args):
    assert bulk_b200.lib.bk_tune_override(*args) == _lib.BK_ERR_INVALID_ARGUMENT


def test_lookup_rejects_bad_op():
    c, p = ctypes.c_int32(), ctypes.c_int32()
    assert bulk_b200.lib.bk_tune_lookup(9, 4, 10, ctypes.byref(c), ctypes.byref(p)) == _lib.BK_ERR_INVALID_ARGUMENT
