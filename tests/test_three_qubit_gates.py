"""Three-qubit gates (ccx, cswap) in QASM -> TPO (the reference's branch is
include/tnbp/parser/qasmtotpo.h:439-698).  The engine splits the 8 x 8 gate
into three factors by two truncated SVDs and joins them along shortest paths
with identity pass-through tensors.  Each layer's operator, contracted over
its bonds into a dense 2^n x 2^n matrix, must equal the dense product of the
layer's gates (built here independently from the gate definitions), for
triples on a path of adjacent sites, on an L shape, at distance two, with
paths that share an edge, in every qubit order, and composed with one- and
two-qubit gates.  Runs on the CPU."""
import itertools
import math

import numpy as np
import pytest

import tnbp_b200 as tb

LX, LY = 3, 2  # qubits ix + 3 iy


def lattice_cz():
    lines = []
    for iy in range(LY):
        for ix in range(LX):
            s = ix + LX * iy
            if ix + 1 < LX:
                lines.append(f"cz q[{s}],q[{s + 1}];")
            if iy + 1 < LY:
                lines.append(f"cz q[{s}],q[{s + LX}];")
    return lines


def embed(n, qubits, fn):
    """Dense 2^n x 2^n operator of a classical-reversible gate: fn maps the
    gate qubits' bits to new bits (index = sum_q bit_q 2^q)."""
    U = np.zeros((2 ** n, 2 ** n), complex)
    for i in range(2 ** n):
        bits = [(i >> q) & 1 for q in range(n)]
        new = fn([bits[q] for q in qubits])
        for q, b in zip(qubits, new):
            bits[q] = b
        U[sum(b << q for q, b in enumerate(bits)), i] = 1.0
    return U


def ccx(n, a, b, c):
    return embed(n, (a, b, c), lambda x: [x[0], x[1], x[2] ^ (x[0] & x[1])])


def cswap(n, a, b, c):
    return embed(n, (a, b, c), lambda x: [x[0], x[2], x[1]] if x[0] else x)


def rx_on(n, q, t):
    u = np.array([[math.cos(t / 2), -1j * math.sin(t / 2)], [-1j * math.sin(t / 2), math.cos(t / 2)]])
    return np.kron(np.kron(np.eye(2 ** (n - q - 1)), u), np.eye(2 ** q))


def dense_layer(edges, layer):
    """Contract the layer's site operators O[bonds..., in, out] over bonds."""
    sites = tb.GetSiteIndexFromBond(edges)
    n = len(sites)
    letters = iter("abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ")
    bond = {m: next(letters) for m in range(len(edges))}
    pin = [next(letters) for _ in range(n)]
    pout = [next(letters) for _ in range(n)]
    ops, subs = [], []
    for si in range(n):
        ops.append(layer.site_op(edges, si))
        subs.append("".join(bond[m] for m in tb.GetSurroundingBondIndex(sites[si], edges)) + pin[si] + pout[si])
    # result index order: out_{n-1} .. out_0, in_{n-1} .. in_0 (qubit 0 least significant)
    res = "".join(reversed(pout)) + "".join(reversed(pin))
    D = np.einsum(",".join(subs) + "->" + res, *ops)
    return D.reshape(2 ** n, 2 ** n)


CASES = [("ccx", (0, 1, 2)), ("ccx", (2, 0, 1)), ("ccx", (0, 1, 4)), ("ccx", (4, 0, 1)), ("ccx", (0, 2, 4)),
         ("ccx", (3, 2, 0)), ("cswap", (3, 4, 5)), ("cswap", (1, 5, 3)), ("cswap", (5, 0, 2)), ("ccx", (0, 5, 2))]


@pytest.mark.parametrize("gate,qs", CASES, ids=[f"{g}{''.join(map(str, q))}" for g, q in CASES])
def test_three_qubit_gate_layer_is_the_dense_gate(gate, qs):
    n = LX * LY
    src = "\n".join(["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];", *lattice_cz(), "barrier q;",
                     f"{gate} q[{qs[0]}],q[{qs[1]}],q[{qs[2]}];", "barrier q;",
                     f"rx(0.3) q[{qs[0]}];", f"{gate} q[{qs[0]}],q[{qs[1]}],q[{qs[2]}];",
                     f"cz q[{qs[1]}],q[{qs[1] + 1 if qs[1] % LX < LX - 1 else qs[1] - 1}];", f"rx(0.7) q[{qs[2]}];"]) + "\n"
    edges = tb.EdgesFromQasm(src)
    layers = tb.QasmToTPO(src, edges)
    assert len(layers) == 3
    G = (ccx if gate == "ccx" else cswap)(n, *qs)
    np.testing.assert_allclose(dense_layer(edges, layers[1]), G, atol=1e-12)
    # composed layer: rx, the gate, a cz on an edge, rx -- in program order
    b = qs[1]
    nb = b + 1 if b % LX < LX - 1 else b - 1
    cz = np.diag([(-1.0 if ((i >> b) & 1 and (i >> nb) & 1) else 1.0) for i in range(2 ** n)])
    want = rx_on(n, qs[2], 0.7) @ cz @ G @ rx_on(n, qs[0], 0.3)
    np.testing.assert_allclose(dense_layer(edges, layers[2]), want, atol=1e-12)
    # the operator bonds stay small: each split keeps at most 4
    assert max(int(r) for r in layers[1].edge_rank) <= 16


def test_three_qubit_gate_on_disconnected_qubits_is_refused():
    src = "OPENQASM 2.0;\nqreg q[5];\ncz q[0],q[1];\ncz q[3],q[4];\nccx q[0],q[1],q[3];\n"
    with pytest.raises(tb.TnbpError):
        tb.QasmToTPO(src, tb.EdgesFromQasm(src))
