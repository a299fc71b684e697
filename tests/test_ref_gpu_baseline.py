"""CPU checks of the optional GPU baseline's host logic: the parser that reads
the reference drivers' printed times, and the recipe's text patches (on
synthetic text)."""
from __future__ import annotations

import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _load(name):
    spec = importlib.util.spec_from_file_location(name, ROOT / "baseline" / f"{name}.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_parser_reads_each_section():
    c = _load("compare_gpu")
    text = "\n".join([
        "Testing n = 1", "my_result: 13",
        "int: ", "Thrust's time: 1.5 ms", "My time:       2.5 ms", "Performance relative to Thrust: 0.6",
        "double: ", "Thrust's time: 3 ms", "My time:       4e-1 ms",
    ])
    got = c.parse(text)
    assert got == {"int": {"thrust_ms": 1.5, "reference_ms": 2.5}, "double": {"thrust_ms": 3.0, "reference_ms": 0.4}}
    text = "\n".join([
        "32b int:", "N: 1", "  Thrust's time:  0.01 ms", "  My time:  0.02 ms", "",
        "N: 134217728", "  Thrust's time:  1 ms", "  My time:  2 ms",
        "64b float:", "N: 134217728", "  Thrust's time:  3 ms", "  My time:  4 ms",
    ])
    got = c.parse(text)
    assert got["32b int / N=134217728"] == {"thrust_ms": 1.0, "reference_ms": 2.0}
    assert got["64b float / N=134217728"] == {"thrust_ms": 3.0, "reference_ms": 4.0}
    assert "32b int / N=1" in got
    text = "\n".join([
        "Large input: ", "int: ", "Thrust's time: 1 ms", "My time: 2 ms", "Output ratio: 0.9",
        "Small input: ", "int: ", "Thrust's time: 5 ms", "My time: 6 ms",
    ])
    got = c.parse(text)
    assert got == {"Large input / int": {"thrust_ms": 1.0, "reference_ms": 2.0},
                   "Small input / int": {"thrust_ms": 5.0, "reference_ms": 6.0}}


def test_recipe_patches(tmp_path):
    b = _load("build_ref_gpu")
    p = tmp_path / "h.hpp"
    p.write_text("a;\n  int x = 1;\t\t    int x = 1;\nb;\t\t    c;\n")
    assert b._dedupe_doubled_lines(p) == 1
    assert p.read_text() == "a;\n  int x = 1;\nb;\t\t    c;\n"
    p = tmp_path / "d.cu"
    p.write_text("#include <moderngpu.cuh>\n#include <x>\n\ntemplate<typename T>\nvoid sean_go(int a)\n{\n  f(a);\n}\n"
                 "\nint main()\n{\n  sean_go(1);\n  g();\n  std::cout << \"Sean's time\";\n}\n")
    b._strip_moderngpu(p)
    t = p.read_text()
    assert "moderngpu" not in t and "sean_" not in t and "Sean" not in t and "g();" in t and "#include <x>" in t
    with pytest.raises(RuntimeError):
        b._replace_once(p, "no such text", "x")
