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


def test_footprint_estimate_host_only():
    """tnbp_footprint_estimate (the server's admission figure) runs without a
    device: exact on a one-edge graph, smallest for complex64 storage,
    growing with D; the sweep scratch counts one wave (of at most the wave
    budget, 96 MiB by default) rather than every site's slots."""
    tb = pytest.importorskip("tnbp_b200")
    one = tb.footprint_estimate([(0, 1)], [1], tb.C128)
    # two degree-1 sites of 2 elements x (4 x 16 B); one edge: arenas 128 B,
    # truncation 128 B, Gram partials 512 B; x 1.1 plus 8 MiB
    assert one == int((2 * 2 * 64 + 128 + 128 + 512) * 1.1) + (8 << 20)
    e = tb.bond_square_lattice(6, 6)
    f = {p: tb.footprint_estimate(e, [16] * len(e), p) for p in (tb.C64, tb.MIXED, tb.C128)}
    assert f[tb.C64] < f[tb.MIXED] and f[tb.C64] < f[tb.C128]
    # 36 sites at D = 16: all tree slots would be ~270 MB of complex128; one wave is 96 MiB
    assert f[tb.C128] < 36 * 16**4 * 2 * 16 * 4 + (200 << 20)
    assert tb.footprint_estimate(e, [32] * len(e), tb.MIXED) > 8 * f[tb.MIXED]
    with pytest.raises(tb.TnbpError):
        tb.footprint_estimate(e, [0] * len(e), tb.MIXED)
