"""The C-ABI library loads without a GPU and exports every entry point that
include/tnbp_b200.h declares; state calls fail loudly (no CPU fallback)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "tnbp_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(tnbp_[a-z0-9_]+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(ROOT, "tnbp_b200", "libtnbp_b200.so"))
    names = _declared()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_state_calls_fail_loudly_without_gpu():
    tb = pytest.importorskip("tnbp_b200")
    if tb.device_available():
        pytest.skip("a device is visible")
    with pytest.raises(tb.TnbpError) as e:
        tb.State([(0, 1)])
    assert e.value.code == tb.ENOGPU


def test_no_oracle_on_the_product_path():
    """The product package never imports or links the oracle."""
    pkg = os.path.join(ROOT, "tnbp_b200")
    for dp, _, fs in os.walk(pkg):
        for f in fs:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                txt = open(os.path.join(dp, f), errors="ignore").read()
                assert "bp_numpy" not in txt and "gqten_cpu" not in txt, f
