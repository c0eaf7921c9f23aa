"""The numpy oracle (oracle/bp_numpy.py) against the reference's own outputs.

Fixtures come from the reference's unchanged headers compiled into
oracle/_ref/ (tests/golden/make_golden.py).  Every stage starts from the
reference's own input for that stage, so the comparisons are exact up to
FP64 rounding: AbsorbTPO, one BP sweep, the BP loop with its conditions,
truncation (bond dims, errors, diag(S) messages) and the one- and two-site
expectation values.
"""
import glob
import os

import numpy as np
import pytest

import bp_numpy as bn
from records import load_probe

HERE = os.path.dirname(os.path.abspath(__file__))
PROBES = sorted(glob.glob(os.path.join(HERE, "golden", "probe_*.npz")))


def _edges(R):
    ed = R["edges"].real.astype(int)
    return [(int(ed[0, i]), int(ed[1, i])) for i in range(ed.shape[1])]


@pytest.mark.parametrize("path", PROBES, ids=[os.path.basename(p) for p in PROBES])
def test_oracle_matches_reference_stages(path):
    R, meta = load_probe(path)
    edges = _edges(R)
    ns, ne = len(bn.sites_of(edges)), len(edges)
    V, E = bn.init_state(edges)
    for t in range(int(R["n_layers"].real)):
        P = f"step/{t}/"
        O = [R[f"tpo/{t}/{s}"] for s in range(ns)]
        V1, E1 = bn.absorb_tpo(edges, V, E, O)
        for s in range(ns):
            np.testing.assert_allclose(V1[s], R[P + f"absorb/V/{s}"], atol=1e-13, rtol=0)
        for m in range(2 * ne):
            np.testing.assert_allclose(E1[m], R[P + f"absorb/E/{m}"], atol=1e-13, rtol=0)
        Va = [R[P + f"absorb/V/{s}"] for s in range(ns)]
        Ea = [R[P + f"absorb/E/{m}"] for m in range(2 * ne)]
        F = bn.bp_sweep(edges, Va, Ea)
        for m in range(2 * ne):
            np.testing.assert_allclose(F[m], R[P + f"sweep0/E/{m}"], atol=1e-12, rtol=0)
        Eb, conds = bn.bp_run(edges, Va, Ea, meta["tol"], meta["maxit"])
        ref_iters = int(R[P + "bp_iters"].real)
        assert len(conds) == ref_iters
        for k, c in enumerate(conds):
            rc = float(R[P + f"cond/{k}"].real)
            assert abs(c - rc) <= 1e-12 + 1e-8 * abs(rc)
        for m in range(2 * ne):
            np.testing.assert_allclose(Eb[m], R[P + f"bp/E/{m}"], atol=1e-12, rtol=0)
        Ebr = [R[P + f"bp/E/{m}"] for m in range(2 * ne)]
        Vt, Et, dims, errs = bn.truncate(edges, Va, Ebr, meta["chi"], meta["sv_min"])
        assert dims == [int(x) for x in R[P + "trunc/dims"].real]
        np.testing.assert_allclose(errs, R[P + "trunc/errs"].real, atol=1e-12, rtol=0)
        for m in range(2 * ne):
            np.testing.assert_allclose(Et[m], R[P + f"trunc/E/{m}"], atol=1e-12, rtol=0)
        V = [R[P + f"trunc/V/{s}"] for s in range(ns)]
        E = [R[P + f"trunc/E/{m}"] for m in range(2 * ne)]
    sites1 = R["meas1/sites"].real.astype(int)
    for i, s in enumerate(sites1):
        v = bn.measure_1site(edges, V, E, int(s), R[f"meas1/op/{i}"])
        assert abs(v - R["meas1/values"][i]) < 1e-12
    pr = R["meas2/pairs"].real.astype(int)
    for i in range(pr.shape[1]):
        v = bn.measure_2site(edges, V, E, (int(pr[0, i]), int(pr[1, i])), R[f"meas2/op/{i}"])
        assert abs(v - R["meas2/values"][i]) < 1e-12


def test_chain_is_exact_against_statevector():
    """An open chain is a tree: BP is exact, and with no truncation the BP
    expectation values equal the statevector ones (known-answer test)."""
    rng = np.random.default_rng(7)
    n = 6
    edges = [(i, i + 1) for i in range(n - 1)]
    V, E = bn.init_state(edges)
    gates = []
    # brick-wall of random 2-qubit unitaries, built as TPO layers by SVD split
    for layer in range(3):
        O = [np.zeros((1,) * len(bn.bonds_of(edges, s)) + (2, 2), complex) for s in range(n)]
        for s in range(n):
            O[s][(0,) * len(bn.bonds_of(edges, s)) + (0, 0)] = 1
            O[s][(0,) * len(bn.bonds_of(edges, s)) + (1, 1)] = 1
        ops = [list(o) for o in O]
        # one-qubit random unitaries then CZ on alternating bonds
        Us = []
        for s in range(n):
            q, _ = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
            Us.append(q)
            gates.append((q, [s]))
        cz_bonds = list(range(layer % 2, n - 1, 2))
        for b in cz_bonds:
            gates.append((np.diag([1, 1, 1, -1]).astype(complex), [b, b + 1]))
        O = []
        for s in range(n):
            bonds = bn.bonds_of(edges, s)
            shape = [2 if (m in cz_bonds) else 1 for m in bonds]
            o = np.zeros(shape + [2, 2], complex)
            # CZ = P0 (x) I + P1 (x) Z = sum_k A_k (x) B_k
            for idx in np.ndindex(*shape):
                op = Us[s].copy()
                for k, m in enumerate(bonds):
                    if m in cz_bonds:
                        first = edges[m][0] == s
                        if first:
                            A = np.diag([1, 0]) if idx[k] == 0 else np.diag([0, 1])
                        else:
                            A = np.eye(2) if idx[k] == 0 else np.diag([1, -1])
                        op = A @ op
                o[idx] = op.T  # reference layout O[..., in, out] = U[out][in]
            O.append(o)
        V, E = bn.absorb_tpo(edges, V, E, O)
        E, conds = bn.bp_run(edges, V, E, 1e-14, 50)
        V, E, dims, errs = bn.truncate(edges, V, E, 64, 1e-14)
    terms = [(1, (2,), ("Z",), 1.0), (2, (1, 2), ("X", "Y"), 1.0), (1, (5,), ("X",), 1.0)]
    ref = bn.statevector_expect(n, gates, terms)
    _, vals = bn.pauli_sum(edges, V, E, terms)
    np.testing.assert_allclose(np.array(vals), np.array(ref), atol=1e-10)
    # products ClassifyOps drops, on their tree clusters: exact on a chain
    cl = [((0, 3), ("X", "Z")), ((4, 1), ("Y", "X")), ((1, 2, 4), ("Z", "Y", "X")),
          ((5, 0, 2, 3), ("X", "Z", "Y", "Z")), ((3, 5), ("Z", "Z"))]
    ref = bn.statevector_expect(n, gates, [(3, q, l, 1.0) for q, l in cl])
    got = [bn.measure_cluster(edges, V, E, q, l) for q, l in cl]
    np.testing.assert_allclose(np.array(got), np.array(ref), atol=1e-10)


@pytest.mark.parametrize("path", PROBES, ids=[os.path.basename(p) for p in PROBES])
def test_cluster_of_an_adjacent_pair_is_the_two_site_measurement(path):
    """The tree cluster of an adjacent pair is the pair itself: the cluster
    contraction equals measure.h's two-site value on the reference's final
    (loopy-BP) state."""
    R, meta = load_probe(path)
    edges = _edges(R)
    ns, ne = len(bn.sites_of(edges)), len(edges)
    t = int(R["n_layers"].real) - 1
    V = [R[f"step/{t}/trunc/V/{s}"] for s in range(ns)]
    E = [R[f"step/{t}/trunc/E/{m}"] for m in range(2 * ne)]
    for (a, b) in edges:
        for la, lb in (("X", "Z"), ("Y", "Y"), ("Z", "X")):
            v2 = bn.measure_2site(edges, V, E, (a, b), bn.pauli_two(la, lb))
            vc = bn.measure_cluster(edges, V, E, (b, a), (lb, la))
            assert abs(v2 - vc) < 1e-12


def test_oracle_shortest_paths_are_the_reference_paths():
    """FindShortestPath restated in the oracle against the reference's own
    paths (oracle/ref_hostparity.cc fixtures)."""
    import json
    n = 0
    for p in sorted(glob.glob(os.path.join(HERE, "golden", "host_*.json"))):
        H = json.load(open(p))
        if "paths" not in H:
            continue
        edges = [tuple(e) for e in H["edges"]]
        for src, dst, path in H["paths"]:
            assert bn.shortest_path(edges, src, dst) == path
            n += 1
    assert n > 50
