"""tnbp_estimator (tnbp_b200/apps/estimator.cc): the estimator app's loop as
C++ host code over the C ABI.

Run with the reference app's command line on the golden circuits, its printed
one- and two-site expectation values must equal the reference estimator's
(the fixtures hold the values the reference printed) to 1e-9, as in
test_gpu_parity.py's end-to-end test; --precision mixed must stay within
1e-6 of them.  The same holds with --do_opt_tpo 1.
"""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

from records import load_probe  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
APP = os.path.join(os.path.dirname(HERE), "tnbp_b200", "tnbp_estimator")
ONE = re.compile(r"Expectation value of single site operator at site (\d+) (\S+)")
TWO = re.compile(r"Expectation value of two site operator at sites \((\d+),(\d+)\) (\S+)")


def _run(name, meta, precision, extra=()):
    if not os.path.exists(APP):
        pytest.fail(f"{APP} is not built: run `python tnbp_b200/build.py`")
    cmd = [APP, "--circuit", os.path.join(HERE, "golden", "inputs", f"{name}.qasm"),
           "--sparse_pauli", os.path.join(HERE, "golden", "inputs", f"{name}.txt"),
           "--max_bond_dim", str(meta["chi"]), "--bp_tolerance", repr(meta["tol"]),
           "--max_bp_iterations", str(meta["maxit"]), "--sv_min", repr(meta["sv_min"]),
           "--precision", precision, "--sum", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    one = [float(m.group(2)) for m in ONE.finditer(r.stdout)]
    two = [float(m.group(3)) for m in TWO.finditer(r.stdout)]
    return one, two, r.stdout


@pytest.mark.parametrize("name", ["ki3x3", "rc3x3", "chain6"])
@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("mixed", 1e-6)])
def test_estimator_app_prints_the_reference_values(name, precision, tol):
    R, meta = load_probe(os.path.join(HERE, "golden", f"probe_{name}.npz"))
    one, two, out = _run(name, meta, precision)
    ref_one = [float(v.real) for v in R["meas1/values"]]
    ref_two = [float(v.real) for v in R["meas2/values"]]
    assert len(one) == len(ref_one), out
    assert len(two) >= len(ref_two), out
    for a, b in zip(one, ref_one):
        assert abs(a - b) <= tol, (a, b)
    for a, b in zip(two, ref_two):
        assert abs(a - b) <= tol, (a, b)
    assert "Sum of c_k <P_k>" in out


@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("mixed", 1e-6)])
def test_estimator_app_with_opt_tpo(precision, tol):
    """--do_opt_tpo 1 (OptTPObySVD on every layer, optsvdtpo.h:86-214): a
    kicked-Ising circuit with ZZ compiled as cx rz cx; the fixture holds what
    the reference estimator printed with the same flags."""
    import json
    ref = json.load(open(os.path.join(HERE, "golden", "opt_optzz3x3.json")))
    one, two, out = _run("optzz3x3", ref, precision,
                         ("--do_opt_tpo", "1", "--eps_opt_tpo", repr(ref["eps_opt_tpo"])))
    assert out.count("optimization of tpo for layer") == 3
    if precision == "c128":
        # step 0 leaves a product state: its second singular values are
        # rounding noise at the sv_min = 1e-8 cut, which the reduced-precision
        # sweeps may leave just above it (an extra ~1e-8 direction)
        assert [int(v) for v in re.findall(r"bond dim = (\d+)", out)] == ref["bond_dims"]
    assert len(one) == len(ref["one"]) and len(two) == len(ref["two"]), out
    for a, b in zip(one + two, ref["one"] + ref["two"]):
        assert abs(a - b) <= tol, (a, b)


def test_estimator_app_measures_cluster_terms():
    """--measure_clusters: the rows the reference drops, measured on their
    tree clusters.  On the chain (a tree, no truncation) they are exact; the
    oracle's cluster contraction of the reference's own final state gives
    the same values (a gauge-invariant quantity, 1e-9)."""
    import numpy as np

    import bp_numpy as bn
    R, meta = load_probe(os.path.join(HERE, "golden", "probe_chain6.npz"))
    one, two, out = _run("chain6", meta, "c128", ("--measure_clusters",))
    rows = re.findall(r"Expectation value of cluster operator in row (\d+) (\S+)", out)
    assert rows, out
    pauli = open(os.path.join(HERE, "golden", "inputs", "chain6.txt")).read()
    ed = R["edges"].real.astype(int)
    edges = [(int(ed[0, i]), int(ed[1, i])) for i in range(ed.shape[1])]
    t = int(R["n_layers"].real) - 1
    V = [R[f"step/{t}/trunc/V/{s}"] for s in range(len(bn.sites_of(edges)))]
    E = [R[f"step/{t}/trunc/E/{m}"] for m in range(2 * len(edges))]
    lines = [l.strip() for l in pauli.splitlines()]
    lines = [l for l in lines if l and not l.startswith("#") and not l.startswith("//")]
    for r, v in rows:
        ps = lines[int(r)].split()[-1].upper()
        qs = [i for i in range(len(ps)) if ps[len(ps) - 1 - i] != "I"]
        ls = [ps[len(ps) - 1 - q] for q in qs]
        want = bn.measure_cluster(edges, V, E, qs, ls)
        assert abs(float(v) - want.real) <= 1e-9, (r, v, want)
    assert "Sum of c_k <P_k> over all terms" in out


@pytest.mark.parametrize("precision,tol", [("c128", 1e-9), ("mixed", 1e-6)])
def test_estimator_app_with_num_gates(precision, tol):
    """--num_gates (manual gate-number layering, qasmtotpo.h:709-738) on a
    barrier-free kicked-Ising program split inside its Floquet steps; the
    fixture holds what the reference app printed with the same flags."""
    import json
    ref = json.load(open(os.path.join(HERE, "golden", "count_kinb3x3.json")))
    one, two, out = _run("kinb3x3", ref, precision, ("--num_gates", ",".join(str(n) for n in ref["num_gates"])))
    if precision == "c128":
        assert [int(v) for v in re.findall(r"bond dim = (\d+)", out)] == ref["bond_dims"]
    assert len(one) == len(ref["one"]) and len(two) == len(ref["two"]), out
    for a, b in zip(one + two, ref["one"] + ref["two"]):
        assert abs(a - b) <= tol, (a, b)


@pytest.mark.parametrize("precision,tol", [("c128", 1e-10), ("mixed", 1e-6)])
def test_estimator_app_full_size_random_circuit(precision, tol):
    """The benchmark's random-circuit workload at full size (10x10 qubits, 12
    layers of U3 on every qubit and CZ on one edge colouring, chi 32, the
    64-term observable): every value the reference estimator app printed
    (tests/golden/est_rc10x10.json, made by make_golden.py --only est_rc10)
    against the engine's app on the same files and flags."""
    import json
    ref = json.load(open(os.path.join(HERE, "golden", "est_rc10x10.json")))
    one, two, out = _run("rc10x10", ref, precision)
    got_one = [(int(m.group(1)), float(m.group(2))) for m in ONE.finditer(out)]
    assert [s for s, _ in got_one] == [s for s, _ in ref["one"]], out
    for (_, a), (_, b) in zip(got_one, ref["one"]):
        assert abs(a - b) <= tol, (a, b)
    got_two = [(int(m.group(1)), int(m.group(2)), float(m.group(3))) for m in TWO.finditer(out)]
    assert [(a, b) for a, b, _ in got_two[: len(ref["two"])]] == [(a, b) for a, b, _ in ref["two"]]
    for (_, _, a), (_, _, b) in zip(got_two, ref["two"]):
        assert abs(a - b) <= tol, (a, b)
