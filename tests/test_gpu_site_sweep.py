"""The site-resident sweep kernel (k_site_sweep) against the numpy oracle.

By default (TNBP_SITE_SWEEP=0 turns it off) every site whose tensor, work
buffers, messages and Gram partials fit the kernel's shared memory is swept
whole by one CTA (every
outgoing message, its normalization and its distance to the stored message),
the other sites by the per-level kernels in the same sweep.  Each case runs
in its own process (the switch is read once per process): one sweep of
uneven and uniform dims on lattices and a chain, all three precisions,
against bp_numpy's sweep (complex128 1e-12; the reduced-precision paths read
complex64 site tensors, 5e-5 per element as the other reduced-precision
tests); and a short kicked-Ising solve whose value must equal the per-level
path's (1e-10 on complex128, where lattice sites at D <= 4 are small and the
edges' sites of later steps are not).
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SWITCHES = ("TNBP_LEG_BULK", "TNBP_DISABLE_TCGEN05", "TNBP_LEG_GRAM", "TNBP_SITE_SWEEP")

SWEEP = r"""
import sys
import numpy as np
sys.path[:0] = [{root!r}, {oracle!r}]
import tnbp_b200 as tb, bp_numpy as bn
assert tb.device_available()
cases = [("lattice", 3, "uniform4"), ("lattice", 4, "uneven"), ("lattice", 3, "mixed_big"), ("chain", 6, "uneven")]
worst = {{}}
for kind, L, dims_kind in cases:
    rng = np.random.default_rng(41)
    if kind == "lattice":
        edges = tb.bond_square_lattice(L, L)
    else:
        edges = [(i, i + 1) for i in range(L - 1)]
    ne = len(edges)
    if dims_kind == "uniform4":
        dims = [4] * ne
    elif dims_kind == "uneven":
        dims = [int(x) for x in rng.integers(2, 7, size=ne)]
    else:  # the centre site too large for one CTA, the others small
        dims = [int(x) for x in rng.integers(2, 5, size=ne)]
        for m, (a, b) in enumerate(edges):
            if 4 in (a, b):
                dims[m] = 12
    V = []
    for s in bn.sites_of(edges):
        sh = [dims[m] for m in bn.bonds_of(edges, s)] + [2]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    E = []
    for m in range(2 * ne):
        D = dims[m % ne]
        A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
        M = A @ A.conj().T
        E.append(M / np.linalg.norm(M))
    F = bn.bp_sweep(edges, V, E)
    for name, prec in (("c128", tb.C128), ("mixed", tb.MIXED), ("c64", tb.C64)):
        with tb.State(edges, prec) as st:
            st.set_state(V, E)
            tb.BeliefPropagation(st)
            w = max(float(np.max(np.abs(st.get_message(m) - F[m]))) for m in range(2 * ne))
        worst[name] = max(worst.get(name, 0.0), w)
print("WORST", worst["c128"], worst["mixed"], worst["c64"])
"""

SOLVE = r"""
import math, sys
import numpy as np
sys.path[:0] = [{root!r}]
import tnbp_b200 as tb
edges = tb.bond_square_lattice(4, 4)
layer = tb.KickedIsingTPO(edges, -math.pi / 8, 0.0, 0.4, 1.0)
out = []
for prec in (tb.C128, tb.MIXED):
    with tb.State(edges, prec) as st:
        t = st.tpo(layer)
        for _ in range(4):
            tb.AbsorbTPO(st, t)
            tb.BeliefPropagationLoop(st, 1e-10, 50)
            tb.Truncation(st, 4, 1e-10)
        out.append(tb.Measure(st, [5], [np.diag([1.0, -1.0]).astype(complex)])[0])
print("VALS", out[0].real, out[0].imag, out[1].real, out[1].imag)
"""


def _run(code, flag):
    env = {k: v for k, v in os.environ.items() if k not in SWITCHES}
    env["TNBP_SITE_SWEEP"] = flag
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def test_site_sweep_matches_oracle():
    out = _run(SWEEP.format(root=ROOT, oracle=os.path.join(ROOT, "oracle")), "1")
    c128, mixed, c64 = (float(x) for x in out.split("WORST")[-1].split())
    assert c128 <= 1e-12, c128
    assert mixed <= 5e-5 and c64 <= 5e-5, (mixed, c64)


def test_site_sweep_solve_equals_per_level_path():
    code = SOLVE.format(root=ROOT)
    on = [float(x) for x in _run(code, "1").split("VALS")[-1].split()]
    off = [float(x) for x in _run(code, "0").split("VALS")[-1].split()]
    assert abs(complex(on[0], on[1]) - complex(off[0], off[1])) <= 1e-10, (on, off)
    assert abs(complex(on[2], on[3]) - complex(off[2], off[3])) <= 1e-6, (on, off)
