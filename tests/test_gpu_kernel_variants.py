"""Every leg-contraction kernel of the reduced-precision sweeps against the
numpy oracle.

The engine picks the kernel of each task by its shape; three switches, read
once per process, change that choice: TNBP_LEG_BULK=1 routes the eligible
complex64 tasks to the bulk-staged tcgen05 kernel (cp.async.bulk tiles),
TNBP_DISABLE_TCGEN05=1 routes every task to the CUDA-core kernels, and
TNBP_LEG_GRAM=1 runs each target's last absorption and its Gram in the fused
tcgen05 kernel (k_leg_gram_tc) instead of the separate kernels (the
default), and TNBP_GRAM_PERSIST chooses between the two forms of the tcgen05
Gram (k_gram_tc, one CTA per split-K chunk, and k_gram_tc_persist, one CTA
per SM), which must agree bit for bit.  Each
variant runs in its own process here, on a 3x3 patch at D = 32 (all three
tree levels and all tile layouts of the bulk kernel: L = 1, 32, 1024) and on
uneven dims 2..9, with the message tolerance of the other reduced-precision
tests (5e-5 per element of a normalized message).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

SCRIPT = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {oracle!r}]
import tnbp_b200 as tb, bp_numpy as bn
assert tb.device_available()
worst = 0.0
for L, dims_kind in ((3, "d32"), (3, "uneven")):
    rng = np.random.default_rng(17)
    edges = tb.bond_square_lattice(L, L)
    dims = [32] * len(edges) if dims_kind == "d32" else [int(x) for x in rng.integers(2, 10, size=len(edges))]
    sites = bn.sites_of(edges)
    V = []
    for s in sites:
        sh = [dims[m] for m in bn.bonds_of(edges, s)] + [2]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    E = []
    for m in range(2 * len(edges)):
        D = dims[m % len(edges)]
        A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
        M = A @ A.conj().T
        E.append(M / np.linalg.norm(M))
    F = bn.bp_sweep(edges, V, E)
    for prec in (tb.MIXED, tb.C64):
        with tb.State(edges, prec) as st:
            st.set_state(V, E)
            tb.BeliefPropagation(st)
            for m in range(2 * len(edges)):
                worst = max(worst, float(np.max(np.abs(st.get_message(m) - F[m]))))
print("WORST", worst)
"""


SWITCHES = ("TNBP_LEG_BULK", "TNBP_DISABLE_TCGEN05", "TNBP_LEG_GRAM", "TNBP_GRAM_PERSIST")


@pytest.mark.parametrize("env", [{"TNBP_LEG_BULK": "1"}, {"TNBP_DISABLE_TCGEN05": "1"}, {"TNBP_LEG_GRAM": "1"},
                                 {"TNBP_GRAM_PERSIST": "0"}, {"TNBP_GRAM_PERSIST": "1"}, {}],
                         ids=["bulk-staged", "cuda-core", "fused-leg-gram", "gram-per-chunk", "gram-persistent",
                              "default"])
def test_leg_kernel_variant_matches_oracle(env):
    code = SCRIPT.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"))
    full_env = {k: v for k, v in os.environ.items() if k not in SWITCHES}
    full_env.update(env)
    r = subprocess.run([sys.executable, "-c", code], env=full_env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    worst = float(r.stdout.split("WORST")[-1])
    assert worst <= 5e-5, worst


# The two Gram kernels on the same messages: every BP message of a mixed and
# a complex64 sweep (3x3 at D = 32, where every Gram is a tcgen05 task with
# chunks of an odd number of 64-row blocks at the corners, and a 4x4 lattice
# of uneven dims) must be the same bits.
BITS = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {oracle!r}]
import tnbp_b200 as tb, bp_numpy as bn
out = []
for L, dims_kind in ((3, "d32"), (4, "uneven")):
    rng = np.random.default_rng(29)
    edges = tb.bond_square_lattice(L, L)
    dims = [32] * len(edges) if dims_kind == "d32" else [int(x) for x in rng.integers(3, 33, size=len(edges))]
    V = []
    for s in bn.sites_of(edges):
        sh = [dims[m] for m in bn.bonds_of(edges, s)] + [2]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    E = []
    for m in range(2 * len(edges)):
        D = dims[m % len(edges)]
        A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
        M = A @ A.conj().T
        E.append(M / np.linalg.norm(M))
    for prec in (tb.MIXED, tb.C64):
        with tb.State(edges, prec) as st:
            st.set_state(V, E)
            tb.BeliefPropagation(st)
            out += [np.asarray(st.get_message(m)).ravel() for m in range(2 * len(edges))]
np.save({path!r}, np.concatenate(out))
"""


def test_gram_kernels_agree_bitwise(tmp_path):
    got = []
    for flag in ("0", "1"):
        path = str(tmp_path / f"msgs{flag}.npy")
        code = BITS.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"), path=path)
        env = {k: v for k, v in os.environ.items() if k not in SWITCHES}
        env["TNBP_GRAM_PERSIST"] = flag
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        got.append(np.load(path))
    assert got[0].shape == got[1].shape
    assert np.array_equal(got[0], got[1])
