"""Every leg-contraction kernel of the reduced-precision sweeps against the
numpy oracle.

The engine picks the kernel of each task by its shape; three switches, read
once per process, change that choice: TNBP_LEG_BULK=1 routes the eligible
complex64 tasks to the bulk-staged tcgen05 kernel (cp.async.bulk tiles),
TNBP_DISABLE_TCGEN05=1 routes every task to the CUDA-core kernels, and
TNBP_LEG_GRAM=1 runs each target's last absorption and its Gram in the fused
tcgen05 kernel (k_leg_gram_tc) instead of the separate kernels (the
default).  Each
variant runs in its own process here, on a 3x3 patch at D = 32 (all three
tree levels and all tile layouts of the bulk kernel: L = 1, 32, 1024) and on
uneven dims 2..9, with the message tolerance of the other reduced-precision
tests (5e-5 per element of a normalized message).
"""
import os
import subprocess
import sys

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


@pytest.mark.parametrize("env", [{"TNBP_LEG_BULK": "1"}, {"TNBP_DISABLE_TCGEN05": "1"}, {"TNBP_LEG_GRAM": "1"}, {}],
                         ids=["bulk-staged", "cuda-core", "fused-leg-gram", "default"])
def test_leg_kernel_variant_matches_oracle(env):
    code = SCRIPT.format(root=ROOT, oracle=os.path.join(ROOT, "oracle"))
    full_env = dict(os.environ)
    full_env.pop("TNBP_LEG_BULK", None)
    full_env.pop("TNBP_DISABLE_TCGEN05", None)
    full_env.pop("TNBP_LEG_GRAM", None)
    full_env.update(env)
    r = subprocess.run([sys.executable, "-c", code], env=full_env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    worst = float(r.stdout.split("WORST")[-1])
    assert worst <= 5e-5, worst
