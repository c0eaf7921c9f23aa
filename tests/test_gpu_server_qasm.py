"""Served estimator requests from QASM programs (tnbp_server_submit_qasm): the
estimator app's workload (apps/estimator/main.cc:105-238) -- EdgesFromQasm,
QasmToTPO, optional OptTPObySVD, per layer AbsorbTPO / BP loop / Truncation,
then Σ c_k <P_k> -- batched with kicked-Ising requests in the same sweeps,
and the server's TPO cache.

* Each QASM request gives the same result alone and in a mix with
  kicked-Ising requests of other lattices (1e-12).
* Complex128 served results equal the plain per-job path (1e-10) and the sum
  of the reference estimator's own per-term values (1e-9); with
  do_opt_tpo the reference app's values from --do_opt_tpo 1 (1e-9).
* Requests naming the same program share one set of device TPO layers.
"""
import json
import os

import numpy as np
import pytest

import bp_numpy as bn
from records import load_probe
from test_gpu_server import REQUESTS, THETA_J, observable

pytestmark = pytest.mark.gpu
tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
NAMES = ["ki3x3", "rc3x3", "chain6"]


def _case(name):
    R, meta = load_probe(os.path.join(G, f"probe_{name}.npz"))
    src = open(os.path.join(G, "inputs", f"{name}.qasm")).read()
    pauli = open(os.path.join(G, "inputs", f"{name}.txt")).read()
    return R, meta, src, pauli


def _serve(items, precision, max_active=64, stagger=0):
    """items: ("qasm", name, do_opt) or ("ki", request tuple); returns results."""
    srv = tb.Server(precision, 0, max_active)
    try:
        ids, pending, steps = [], list(items), 0
        while pending or any(srv.result(i) is None for i in ids):
            if pending and (stagger == 0 or steps % stagger == 0):
                it = pending.pop(0)
                if it[0] == "qasm":
                    _, meta, src, pauli = _case(it[1]) if it[1] in NAMES else (None, it[3], it[4], it[5])
                    ids.append(srv.submit_qasm(src, pauli, meta["chi"], meta["tol"], meta["maxit"], meta["sv_min"],
                                               do_opt_tpo=it[2]))
                else:
                    L, chi, nst, th, seed = it[1]
                    ids.append(srv.submit_kicked_ising(L, chi, nst, THETA_J, th, observable(L, seed)))
                if stagger == 0:
                    continue
            srv.step()
            steps += 1
            assert steps < 100000
        return [srv.result(i) for i in ids], srv.tpo_cache_stats()
    finally:
        srv.close()


def _plain(name, precision=tb.C128):
    _, meta, src, pauli = _case(name)
    edges = tb.EdgesFromQasm(src)
    with tb.State(edges, precision) as st:
        for layer in tb.QasmToTPO(src, edges):
            tb.AbsorbTPO(st, layer)
            tb.BeliefPropagationLoop(st, meta["tol"], meta["maxit"])
            tb.Truncation(st, meta["chi"], meta["sv_min"])
        total, _ = tb.MeasurePauliSum(st, tb.load_sparse_pauli(pauli, edges))
    return total


def _reference_sum(terms, one, two):
    """Σ c_k <P_k> from the values the reference printed (one-site terms in
    file order, then two-site terms in file order); None if the reference
    printed fewer two-site values than there are terms."""
    k1 = [t for t in terms if t[0] == 1]
    k2 = [t for t in terms if t[0] == 2]
    if len(k1) != len(one) or len(k2) != len(two):
        return None
    return sum(t[3] * v for t, v in zip(k1 + k2, list(one) + list(two)))


@pytest.mark.parametrize("precision", [tb.MIXED, tb.C128])
def test_qasm_requests_alone_and_in_a_mix(precision):
    qasm = [("qasm", n, False) for n in NAMES]
    ki = [("ki", r) for r in REQUESTS[:4]]
    alone = [_serve([q], precision)[0][0] for q in qasm]
    mixed, _ = _serve([ki[0], qasm[0], ki[1], qasm[1], ki[2], qasm[2], ki[3]], precision, stagger=2)
    together = [mixed[1], mixed[3], mixed[5]]
    for a, b in zip(alone, together):
        assert abs(a - b) <= 1e-12, (a, b)


def test_qasm_c128_server_equals_plain_path_and_reference():
    served, _ = _serve([("qasm", n, False) for n in NAMES], tb.C128, stagger=1)
    checked = 0
    for name, s in zip(NAMES, served):
        p = _plain(name)
        assert abs(s - p) <= 1e-10, (name, s, p)
        R, _, src, pauli = _case(name)
        terms, _ = bn.parse_pauli_text(pauli, tb.EdgesFromQasm(src))
        ref = _reference_sum(terms, R["meas1/values"], R["meas2/values"])
        if ref is not None:
            assert abs(s - ref) <= 1e-9, (name, s, ref)
            checked += 1
    assert checked >= 1


def test_qasm_request_with_opt_tpo_matches_the_reference_app():
    ref = json.load(open(os.path.join(G, "opt_optzz3x3.json")))
    src = open(os.path.join(G, "inputs", "optzz3x3.qasm")).read()
    pauli = open(os.path.join(G, "inputs", "optzz3x3.txt")).read()
    served, stats = _serve([("qasm", "optzz3x3", True, ref, src, pauli)], tb.C128)
    terms, _ = bn.parse_pauli_text(pauli, tb.EdgesFromQasm(src))
    want = _reference_sum(terms, ref["one"], ref["two"])
    assert want is not None
    assert abs(served[0] - want) <= 1e-9, (served[0], want)


def test_requests_on_one_program_share_its_tpo_layers():
    _, meta, src, pauli = _case("rc3x3")
    srv = tb.Server(tb.C128, 0, 8)
    try:
        ids = [srv.submit_qasm(src, pauli, meta["chi"], meta["tol"], meta["maxit"], meta["sv_min"]) for _ in range(3)]
        ids.append(srv.submit_qasm(src, pauli, meta["chi"], meta["tol"], meta["maxit"], meta["sv_min"],
                                   do_opt_tpo=True))
        ids.append(srv.submit_kicked_ising(3, 4, 2, THETA_J, 0.5, observable(3, 1)))
        ids.append(srv.submit_kicked_ising(3, 8, 3, THETA_J, 0.5, observable(3, 2)))
        hits, misses, entries = srv.tpo_cache_stats()
        assert (hits, misses, entries) == (3, 3, 3)
        while any(srv.result(i) is None for i in ids):
            srv.step()
        r = [srv.result(i) for i in ids]
        assert r[0] == r[1] == r[2]
        assert abs(r[3] - r[0]) <= 1e-8  # the compressed TPO is the same operator
    finally:
        srv.close()


def test_qasm_submit_errors():
    srv = tb.Server(tb.MIXED, 0, 4)
    try:
        with pytest.raises(tb.TnbpError) as e:
            srv.submit_qasm("OPENQASM 2.0;\nqreg q[2];\ncx q[0] q[1];\n", "1.0 ZZ\n", 4)
        assert e.value.code == tb.EPARSE
        src = "OPENQASM 2.0;\ninclude \"qelib1.inc\";\nqreg q[3];\ncx q[0],q[1];\n"
        with pytest.raises(tb.TnbpError) as e:
            srv.submit_qasm(src, "1.0 ZII\n", 4)  # qubit 2: no two-qubit gate touches it
        assert e.value.code == tb.EINVAL
        rid = srv.submit_qasm(src, "1.0 IZZ\n0.5 IIZ\n", 4)
        while srv.result(rid) is None:
            srv.step()
        assert abs(srv.result(rid) - 1.5) <= 1e-12  # |00>: <Z0 Z1> = <Z0> = 1
    finally:
        srv.close()
