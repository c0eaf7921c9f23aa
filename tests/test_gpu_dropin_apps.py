"""tnbp's own apps running unchanged on the GPU engine.

apps/estimator/main.cc and apps/kicked_ising_lattice/main.cc from the
reference tree are compiled, unmodified, against the drop-in tensor backend
(include/tnbp_dropin/gqten/gqten.h) and the GPU overloads of tnbp's hot-path
functions (tnbp_b200/dropin/device_overloads.cpp) by build()
(tnbp_b200/build.py build_dropin) into tnbp_b200/apps/_dropin/.  Their
printed values must equal the values the reference apps printed on the CPU
(the fixtures): the 4x4 kicked-Ising workload (both apps; steps 0-3 to 1e-10,
step 4 to 1e-7, where the reference's own BP loop ends after 50 sweeps with a
growing condition), the golden circuits (1e-9, as the other end-to-end
tests) and the full-size random-circuit workload (1e-10).
"""
import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

from records import load_probe  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
BIN = os.path.join(os.path.dirname(HERE), "tnbp_b200", "apps", "_dropin")
ONE = re.compile(r"Expectation value of single site operator at site (\d+) (\S+)")
TWO = re.compile(r"Expectation value of two site operator at sites \((\d+),(\d+)\) (\S+)")


def _app(name):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} is built only where the reference sources are (build() on the build machine)")
    return exe


def _estimator(qasm, pauli, chi, tol, maxit, sv_min):
    r = subprocess.run([_app("estimator"), "--circuit", qasm, "--sparse_pauli", pauli, "--max_bond_dim", str(chi),
                        "--bp_tolerance", repr(tol), "--max_bp_iterations", str(maxit), "--sv_min", repr(sv_min)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return ([(int(m.group(1)), float(m.group(2))) for m in ONE.finditer(r.stdout)],
            [(int(m.group(1)), int(m.group(2)), float(m.group(3))) for m in TWO.finditer(r.stdout)], r.stdout)


def test_dropin_kicked_ising_lattice_config1():
    ref = json.load(open(os.path.join(G, "config1.json")))["kicked_ising_lattice"]
    r = subprocess.run([_app("kicked_ising_lattice"), "--lattice", "square", "--L", "4", "--dt", "0.25", "--Jz", "-1",
                        "--hz", "0", "--hx", repr(ref["hx"]), "--num_steps", "5", "--max_bond_dim", "4",
                        "--bp_tolerance", "1e-10", "--max_bp_iterations", "50"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = {}
    for m in re.finditer(r"measurement of (Z|X) at site (\d+) time step (\d+) = (\S+)", r.stdout):
        got[(m.group(1), f"{m.group(3)}/{m.group(2)}")] = float(m.group(4))
    for m in re.finditer(r"measurement of ZZ at sites \((\d+),(\d+)\) time step (\d+) = (\S+)", r.stdout):
        got[("ZZ", f"{m.group(3)}/{m.group(1)},{m.group(2)}")] = float(m.group(4))
    n = 0
    for kind in ("Z", "X", "ZZ"):
        for key, want in ref[kind].items():
            step = int(key.split("/")[0])
            tol = 1e-7 if step >= 4 else 1e-10
            assert abs(got[(kind, key)] - want) <= tol, (kind, key, got[(kind, key)], want)
            n += 1
    assert n > 100


def test_dropin_estimator_config1():
    ref = json.load(open(os.path.join(G, "config1.json")))["estimator"]
    one, _, out = _estimator(os.path.join(G, "inputs", "config1.qasm"), os.path.join(G, "inputs", "config1.txt"),
                             4, 1e-10, 50, 1e-8)
    assert one and one[0][0] == 5
    assert abs(one[0][1] - ref["Z5"]) <= 1e-7, (one, ref["Z5"])
    dims = [int(v) for v in re.findall(r"bond dim = (\d+)", out)]
    assert dims == ref["bond_dims"]


@pytest.mark.parametrize("name", ["ki3x3", "rc3x3", "chain6"])
def test_dropin_estimator_golden_circuits(name):
    R, meta = load_probe(os.path.join(G, f"probe_{name}.npz"))
    one, two, _ = _estimator(os.path.join(G, "inputs", f"{name}.qasm"), os.path.join(G, "inputs", f"{name}.txt"),
                             meta["chi"], meta["tol"], meta["maxit"], meta["sv_min"])
    ref_one = [float(v.real) for v in R["meas1/values"]]
    ref_two = [float(v.real) for v in R["meas2/values"]]
    assert len(one) == len(ref_one)
    for (_, a), b in zip(one, ref_one):
        assert abs(a - b) <= 1e-9, (a, b)
    for (_, _, a), b in zip(two, ref_two):
        assert abs(a - b) <= 1e-9, (a, b)


def test_dropin_estimator_full_size_random_circuit():
    ref = json.load(open(os.path.join(G, "est_rc10x10.json")))
    one, two, _ = _estimator(os.path.join(G, "inputs", "rc10x10.qasm"), os.path.join(G, "inputs", "rc10x10.txt"),
                             ref["chi"], ref["tol"], ref["maxit"], ref["sv_min"])
    assert [s for s, _ in one] == [s for s, _ in ref["one"]]
    for (_, a), (_, b) in zip(one, ref["one"]):
        assert abs(a - b) <= 1e-10, (a, b)
    for (_, _, a), (_, _, b) in zip(two, ref["two"]):
        assert abs(a - b) <= 1e-10, (a, b)
