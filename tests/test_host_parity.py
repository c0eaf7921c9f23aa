"""Bit-exact parity of the engine's host-side builders with the reference's
own code (fixtures from oracle/ref_hostparity.cc, tests/golden/host_*.json):
lattice edges, greedy BP layers, leg order, BFS paths, parsed QASM
(op, qubits, params to the last bit), EdgesFromQasm, TPO layer shapes and
Pauli-term classification.  Runs on the CPU (no device needed)."""
import glob
import json
import os

import numpy as np
import pytest

import bp_numpy as bn
from reference_root import reference_file, reference_root

tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
HOSTS = sorted(glob.glob(os.path.join(G, "host_*.json")))


def _graph_checks(edges, ref):
    assert [tuple(e) for e in ref["edges"]] == edges
    assert [[tuple(e) for e in l] for l in ref["layers"]] == tb.GreedyEdgeLayering(edges)
    sites = tb.GetSiteIndexFromBond(edges)
    assert sites == ref["sites"]
    for s, b in zip(sites, ref["bonds"]):
        assert tb.GetSurroundingBondIndex(s, edges) == b
    for src, dst, path in ref["paths"]:
        assert tb.FindShortestPath(edges, src, dst) == path


@pytest.mark.parametrize("path", HOSTS, ids=[os.path.basename(p) for p in HOSTS])
def test_host_builders_bit_exact(path):
    ref = json.load(open(path))
    name = os.path.basename(path)[5:-5]
    if name.startswith("lattice"):
        Lx, Ly = map(int, name[7:].split("x"))
        _graph_checks(tb.bond_square_lattice(Lx, Ly), ref)
        return
    if name in ("kobe", "ising_circuit"):
        pytest.skip("input lives in the reference tree") if not os.path.exists(reference_root()) else None
        base = reference_file("apps", "estimator/kicked_ising.qasm" if name == "kobe" else "qasm_tpo/ising_circuit.qasm")
        src = open(base).read()
        ptxt = open(reference_file("apps", "estimator", "H_ising_kobe.txt")).read() if name == "kobe" else None
    else:
        src = open(os.path.join(G, "inputs", f"{name}.qasm")).read()
        pp = os.path.join(G, "inputs", f"{name}.txt")
        ptxt = open(pp).read() if os.path.exists(pp) else None
    ins = tb.qasm_instructions(src)
    assert len(ins) == len(ref["instructions"])
    for (op, qs, ps, nq), (rop, rqs, rps) in zip(ins, ref["instructions"]):
        assert op == rop
        if nq <= 4:
            assert qs == rqs
        else:
            assert nq == len(rqs)
        assert len(ps) == len(rps)
        for a, b in zip(ps, rps):
            assert a == b  # same grammar and evaluation order: identical doubles
    edges = tb.EdgesFromQasm(src) if name != "pass2x3" else tb.bond_square_lattice(3, 2)
    _graph_checks(edges, ref)
    if "tpo_shapes" in ref:
        layers = tb.QasmToTPO(src, edges)
        assert len(layers) == len(ref["tpo_shapes"])
        for layer, shapes in zip(layers, ref["tpo_shapes"]):
            for si, sh in enumerate(shapes):
                assert list(layer.site_op(edges, si).shape) == sh
    if ptxt is not None:
        terms = tb.load_sparse_pauli(ptxt, edges)
        ones = [(int(q), l) for k, q, l in zip(terms.kind, terms.q0, terms.letters[0::2].decode()) if k == 1]
        assert [q for q, _ in ones] == [r[0] for r in ref["pauli_one"]]
        for (q, l), r in zip(ones, ref["pauli_one"]):
            op = np.array([complex(*x) for x in r[1]]).reshape((2, 2), order="F")
            assert np.array_equal(op, bn.pauli_op(l))
        twos = [(int(a), int(b), terms.letters[2 * i:2 * i + 2].decode())
                for i, (k, a, b) in enumerate(zip(terms.kind, terms.q0, terms.q1)) if k == 2]
        assert [(a, b) for a, b, _ in twos] == [(r[0], r[1]) for r in ref["pauli_two"]]
        for (a, b, ls), r in zip(twos, ref["pauli_two"]):
            op = np.array([complex(*x) for x in r[2]]).reshape((2, 2, 2, 2), order="F")
            assert np.array_equal(op, bn.pauli_two(ls[0], ls[1]))
        rows = list(terms.row)
        coeffs = [complex(*ref["pauli_coeffs"][i]) for i in range(len(ref["pauli_coeffs"]))]
        kept_coeffs = [c for c in terms.coeff]
        # coefficients of kept terms appear in file order
        it = iter(coeffs)
        for c in kept_coeffs:
            assert any(c == x for x in it)
        assert terms.dropped + len(terms) == len(coeffs)
        assert rows == sorted(rows)


def test_qasm_errors_are_reported_not_fatal():
    with pytest.raises(tb.TnbpError) as e:
        tb.qasm_instructions("OPENQASM 2.0;\nqreg q[2];\ncx q[0];\n")
    assert e.value.code == tb.EPARSE
    with pytest.raises(tb.TnbpError):
        tb.qasm_instructions("OPENQASM 2.0;\nqreg q[2];\nrx(foo) q[0];\n")
    with pytest.raises(tb.TnbpError) as e:
        tb.QasmToTPO("OPENQASM 2.0;\nqreg q[2];\ncx q[0],q[1];\nmeasure q[0] -> c[0];\n", [(0, 1)])
    with pytest.raises(tb.TnbpError) as e:
        tb.load_sparse_pauli("1.0 XQ\n", [(0, 1)])
    assert e.value.code == tb.EPARSE


def test_kicked_ising_tpo_is_the_floquet_step():
    """Contracting the kicked-Ising TPO of a 2-site chain over its bond gives
    Ux Uz exp(-i dt Jz ZZ) (apps/kicked_ising_lattice/circuit.h:43-102)."""
    Jz, hz, hx, dt = -0.7, 0.3, 1.1, 0.4
    layer = tb.KickedIsingTPO([(0, 1)], Jz, hz, hx, dt)
    A = layer.site_op([(0, 1)], 0)  # (r, in, out)
    B = layer.site_op([(0, 1)], 1)
    # U[(a_out, b_out), (a_in, b_in)] = sum_k A[k, a_in, a_out] B[k, b_in, b_out]
    U = np.einsum("kia,kjb->abij", A, B).reshape(4, 4, order="F")
    Z = np.diag([1, -1])
    X = np.array([[0, 1], [1, 0]])
    zz = np.kron(Z, Z)
    from scipy.linalg import expm
    one = expm(-1j * dt * hx * X) @ expm(-1j * dt * hz * Z)
    want = np.kron(one, one) @ expm(-1j * dt * Jz * zz)
    # kron order: little-endian index a + 2 b -> np.kron(b-part, a-part)
    np.testing.assert_allclose(U, want, atol=1e-14)
