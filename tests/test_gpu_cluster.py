"""Pauli products the reference drops (non-adjacent pairs, three or more
qubits; paulitotpo.h:111-132), measured on the device on their tree
clusters (tnbp_measure_cluster / tnbp_measure_pauli_text).

Parity is against the numpy oracle's cluster contraction on the same state
(the reference's final state of each probe, uploaded), which tests/
test_oracle_golden.py pins to the statevector on a tree graph and to the
reference's two-site measurement for adjacent pairs:
* complex128 storage (TNBP_C128, TNBP_MIXED): 1e-10;
* complex64 storage (TNBP_C64): 1e-5;
* an adjacent pair through the cluster path equals the two-site measurement
  of tnbp_measure_pauli_sum (1e-12);
* tnbp_measure_pauli_text: kept rows as tnbp_measure_pauli_sum, dropped rows
  as tnbp_measure_cluster, identity rows as 1.
"""
import glob
import os

import numpy as np
import pytest

import bp_numpy as bn
from records import load_probe

pytestmark = pytest.mark.gpu
tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
PROBES = sorted(glob.glob(os.path.join(HERE, "golden", "probe_*.npz")))


def _final_state(path):
    R, _ = load_probe(path)
    ed = R["edges"].real.astype(int)
    edges = [(int(ed[0, i]), int(ed[1, i])) for i in range(ed.shape[1])]
    ns, ne = len(bn.sites_of(edges)), len(edges)
    t = int(R["n_layers"].real) - 1
    V = [R[f"step/{t}/trunc/V/{s}"] for s in range(ns)]
    E = [R[f"step/{t}/trunc/E/{m}"] for m in range(2 * ne)]
    return edges, V, E


def _terms(edges, seed, n=12):
    """Random products on 2 to 4 distinct qubits, none an adjacent pair."""
    rng = np.random.default_rng(seed)
    sites = bn.sites_of(edges)
    eset = {tuple(e) for e in edges} | {(b, a) for a, b in edges}
    out = []
    while len(out) < n:
        k = int(rng.integers(2, min(5, len(sites) + 1)))
        q = [int(x) for x in rng.choice(sites, size=k, replace=False)]
        if k == 2 and (q[0], q[1]) in eset:
            continue
        out.append((q, "".join(rng.choice(list("XYZ"), size=k))))
    return out


@pytest.mark.parametrize("path", PROBES, ids=[os.path.basename(p) for p in PROBES])
@pytest.mark.parametrize("prec,tol", [(tb.C128, 1e-10), (tb.MIXED, 1e-10), (tb.C64, 1e-5)])
def test_cluster_terms_match_the_oracle(path, prec, tol):
    edges, V, E = _final_state(path)
    terms = _terms(edges, 11)
    coeffs = np.linspace(-1.0, 1.0, len(terms)) + 0.25j
    with tb.State(edges, prec) as st:
        st.set_state(V, E)
        vals, total = tb.MeasureCluster(st, terms, coeffs)
    want = [bn.measure_cluster(edges, V, E, q, tuple(l)) for q, l in terms]
    for got, w in zip(vals, want):
        assert abs(got - w) <= tol, (got, w)
    assert abs(total - sum(c * w for c, w in zip(coeffs, want))) <= tol * len(terms)


@pytest.mark.parametrize("path", PROBES, ids=[os.path.basename(p) for p in PROBES])
def test_adjacent_pair_through_the_cluster_path(path):
    edges, V, E = _final_state(path)
    with tb.State(edges, tb.C128) as st:
        st.set_state(V, E)
        pairs = [((a, b), "XZ") for a, b in edges] + [((b, a), "YY") for a, b in edges]
        vals, _ = tb.MeasureCluster(st, pairs)
        lines = [f"1.0 {_string(len(bn.sites_of(edges)), q, l)}" for q, l in pairs]
        kept = tb.load_sparse_pauli("\n".join(lines) + "\n", edges)
        _, per = tb.MeasurePauliSum(st, kept)
    assert len(per) == len(pairs)
    for a, b in zip(vals, per):
        assert abs(a - b) <= 1e-12, (a, b)


def _string(n, qubits, letters):
    s = ["I"] * (max(qubits) + 1 if n <= max(qubits) else n)
    for q, l in zip(qubits, letters):
        s[len(s) - 1 - q] = l
    return "".join(s)


def test_measure_pauli_text_rows():
    path = os.path.join(HERE, "golden", "probe_rc3x3.npz")
    edges, V, E = _final_state(path)
    n = len(bn.sites_of(edges))
    cl = _terms(edges, 5, n=5)
    rows = [("0.5", [4], "Z"), ("-1.25", [0, 1], "XY"), ("2.0", [], ""), ("0.75", cl[0][0], cl[0][1]),
            ("1.5", cl[1][0], cl[1][1]), ("0.3", [8], "X"), ("-0.7", cl[2][0], cl[2][1])]
    text = "\n".join(f"{c} {_string(n, q, l) if q else 'I' * n}" for c, q, l in rows) + "\n"
    with tb.State(edges, tb.C128) as st:
        st.set_state(V, E)
        total, vals, kinds = tb.MeasurePauliText(st, text, clusters=True)
        total0, vals0, _ = tb.MeasurePauliText(st, text, clusters=False)
        kept = tb.load_sparse_pauli(text, edges)
        ksum, kper = tb.MeasurePauliSum(st, kept)
        cvals, _ = tb.MeasureCluster(st, [(q, l) for _, q, l in rows if len(q) > 1 and (len(q) > 2 or tuple(q) not in
                                                                                          {tuple(e) for e in edges})])
    assert list(kinds) == [1, 2, 0, 3, 3, 1, 3]
    assert abs(total0 - ksum) <= 1e-12
    assert vals[2] == 1.0
    assert np.isnan(vals0[3].real) and np.isnan(vals0[4].real) and np.isnan(vals0[6].real)
    k = [i for i, kd in enumerate(kinds) if kd in (1, 2)]
    for i, v in zip(k, kper):
        assert abs(vals[i] - v) <= 1e-12
    c = [i for i, kd in enumerate(kinds) if kd == 3]
    for i, v in zip(c, cvals):
        assert abs(vals[i] - v) <= 1e-12
    want = sum(float(rows[i][0]) * vals[i] for i in range(len(rows)))
    assert abs(total - want) <= 1e-10
