"""OptTPObySVD (include/tnbp/ptns/function/optsvdtpo.h:86-214): the engine's
host implementation (tnbp_opt_tpo_svd, OptTPObySVD in Python) and the numpy
oracle against the reference's own OptTPObySVD (fixtures
tests/golden/opttpo_*, made by oracle/ref_hostparity.cc).

An SVD fixes its singular vectors only up to a unitary on each operator bond,
so the checks are on what such a gauge leaves unchanged: the bond dimensions
(exact), the full operator of a small lattice (all site operators contracted,
within 1e-12) and the singular values of every bond-leg unfolding of every
site operator (within 1e-12).  Runs on the CPU (no device needed)."""
import ctypes as C
import json
import os
import string

import numpy as np
import pytest

import bp_numpy as bn
from reference_root import reference_file, reference_root

tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
KOBE = reference_file("apps", "estimator", "kicked_ising.qasm")
SMALL = [("zzcx3x3", "eps1e-08"), ("zzcx3x3", "eps1000"), ("optmix2x3", "eps1e-08")]


def _fixture(name, tag):
    z = np.load(os.path.join(G, f"opttpo_{name}.npz"))
    edges = [tuple(int(v) for v in e) for e in z["edges"]]
    ns = len(bn.sites_of(edges))
    stages = {}
    for stage in ("before", "after"):
        layers = []
        while f"{tag}/{stage}/{len(layers)}/0" in z:
            l = len(layers)
            layers.append([z[f"{tag}/{stage}/{l}/{s}"] for s in range(ns)])
        stages[stage] = layers
    eps = float(tag[3:])
    return edges, stages["before"], stages["after"], eps


def full_operator(edges, ops):
    """<out|O|in> of the whole layer: every bond contracted, rows = outputs,
    columns = inputs, qubit 0 the least significant bit."""
    sites = bn.sites_of(edges)
    letters = iter(string.ascii_letters)
    bond = {m: next(letters) for m in range(len(edges))}
    lin = {s: next(letters) for s in sites}
    lout = {s: next(letters) for s in sites}
    terms = ["".join(bond[m] for m in bn.bonds_of(edges, s)) + lin[s] + lout[s] for s in sites]
    spec = (",".join(terms) + "->" + "".join(lout[s] for s in reversed(sites))
            + "".join(lin[s] for s in reversed(sites)))
    n = len(sites)
    return np.einsum(spec, *ops, optimize=True).reshape(2 ** n, 2 ** n)


def leg_spectra(t):
    return [np.linalg.svd(np.moveaxis(t, k, 0).reshape(t.shape[k], -1), compute_uv=False)
            for k in range(t.ndim - 2)]


def _same_up_to_bond_gauge(edges, got, ref, full=True):
    assert [t.shape for t in got] == [t.shape for t in ref]
    for a, b in zip(got, ref):
        for sa, sb in zip(leg_spectra(a), leg_spectra(b)):
            np.testing.assert_allclose(sa, sb, rtol=0, atol=1e-12)
    if full:
        np.testing.assert_allclose(full_operator(edges, got), full_operator(edges, ref), rtol=0, atol=1e-12)


def _engine(edges, ops, eps):
    layer = tb.OptTPObySVD(edges, tb.TPOLayer.from_ops(edges, ops), eps)
    return [layer.site_op(edges, si) for si in range(len(ops))]


@pytest.mark.parametrize("name,tag", SMALL)
def test_oracle_matches_reference(name, tag):
    """Pins the numpy restatement to the reference's OptTPObySVD."""
    edges, before, after, eps = _fixture(name, tag)
    assert before and len(before) == len(after)
    for b, a in zip(before, after):
        _same_up_to_bond_gauge(edges, bn.opt_tpo_svd(edges, b, eps), a)


@pytest.mark.parametrize("name,tag", SMALL)
def test_engine_matches_reference(name, tag):
    edges, before, after, eps = _fixture(name, tag)
    for b, a in zip(before, after):
        _same_up_to_bond_gauge(edges, _engine(edges, b, eps), a)


@pytest.mark.parametrize("name,lattice", [("zzcx3x3", None), ("optmix2x3", (3, 2))])
def test_engine_on_its_own_qasm_tpo(name, lattice):
    """QasmToTPO then OptTPObySVD, all in the engine, from the QASM text."""
    edges, _, after, eps = _fixture(name, "eps1e-08")
    src = open(os.path.join(G, "inputs", f"{name}.qasm")).read()
    if lattice is None:
        assert tb.EdgesFromQasm(src) == edges
    for l, layer in enumerate(tb.QasmToTPO(src, edges)):
        tb.OptTPObySVD(edges, layer, eps)
        got = [layer.site_op(edges, si) for si in range(len(after[l]))]
        _same_up_to_bond_gauge(edges, got, after[l])


def test_compression_is_exact_and_shrinks_the_bonds():
    """cx rz cx on every bond: operator rank 4 -> 2, the operator unchanged
    (the discarded singular values are rounding noise)."""
    edges, before, after, eps = _fixture("zzcx3x3", "eps1e-08")
    for b in before:
        got = _engine(edges, b, eps)
        assert all(t.shape[:-2] == (4,) * (t.ndim - 2) for t in b)
        assert all(t.shape[:-2] == (2,) * (t.ndim - 2) for t in got)
        np.testing.assert_allclose(full_operator(edges, got), full_operator(edges, b), rtol=0, atol=1e-12)


def test_large_eps_keeps_one_singular_value():
    edges, before, after, eps = _fixture("zzcx3x3", "eps1000")
    assert eps > 1
    for b, a in zip(before, after):
        got = _engine(edges, b, eps)
        assert all(t.shape[:-2] == (1,) * (t.ndim - 2) for t in got)
        assert [t.shape for t in got] == [t.shape for t in a]


@pytest.mark.skipif(not os.path.exists(KOBE), reason="input lives in the reference tree")
def test_reference_kicked_ising_qasm():
    """The reference's own 156-qubit kicked_ising.qasm (ZZ as cx u cx):
    bond dimensions and per-leg spectra of every compressed site operator."""
    ref = json.load(open(os.path.join(G, "opttpo_kobe.json")))
    edges = [tuple(e) for e in ref["edges"]]
    src = open(KOBE).read()
    assert tb.EdgesFromQasm(src) == edges
    layers = tb.QasmToTPO(src, edges)
    want = ref["eps1e-08"]["layers"]
    assert len(layers) == len(want)
    for layer, wl in zip(layers, want):
        tb.OptTPObySVD(edges, layer, 1e-8)
        for si, w in enumerate(wl):
            t = layer.site_op(edges, si)
            assert list(t.shape) == w["shape"]
            assert abs(np.linalg.norm(t) - w["norm"]) <= 1e-12 * max(1.0, w["norm"])
            for s, ws in zip(leg_spectra(t), w["legs"]):
                np.testing.assert_allclose(s, ws, rtol=0, atol=1e-12)


def test_abi_errors_and_in_place_repacking():
    edges, before, _, _ = _fixture("zzcx3x3", "eps1e-08")
    layer = tb.TPOLayer.from_ops(edges, before[0])
    e = np.ascontiguousarray(np.array(edges, np.int32))
    rank = layer.edge_rank.copy()
    off = layer.op_offset.copy()
    n_in = layer.op_data.size
    data = np.zeros(2 * n_in + 8, np.float64)
    data[: 2 * n_in] = layer.op_data.view(np.float64)
    guard = data[2 * n_in:].copy()
    i32, i64, f64 = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)
    nel = C.c_int64()
    args = lambda r, o, d: (e.ctypes.data_as(i32), len(edges), 1e-8, r, o, d, C.byref(nel))  # noqa: E731
    assert tb.lib.tnbp_opt_tpo_svd(*args(None, off.ctypes.data_as(i64), data.ctypes.data_as(f64))) == tb.EINVAL
    bad = rank.copy()
    bad[0] = 0
    assert tb.lib.tnbp_opt_tpo_svd(*args(bad.ctypes.data_as(i32), off.ctypes.data_as(i64),
                                         data.ctypes.data_as(f64))) == tb.EINVAL
    neg = off.copy()
    neg[1] = -1
    assert tb.lib.tnbp_opt_tpo_svd(*args(rank.ctypes.data_as(i32), neg.ctypes.data_as(i64),
                                         data.ctypes.data_as(f64))) == tb.EINVAL
    # failed calls leave the caller's buffers as they were
    np.testing.assert_array_equal(data[: 2 * n_in], layer.op_data.view(np.float64))
    assert tb.lib.tnbp_opt_tpo_svd(*args(rank.ctypes.data_as(i32), off.ctypes.data_as(i64),
                                         data.ctypes.data_as(f64))) == tb.OK
    assert 0 < nel.value < n_in
    assert off[0] == 0 and np.all(np.diff(off) > 0) and off[-1] < nel.value
    np.testing.assert_array_equal(data[2 * n_in:], guard)


def test_manual_gate_number_layering_matches_reference():
    """QasmToTPO with num_gates (qasmtotpo.h:709-738) against the reference's
    own overload (tests/golden/tpocount_kinb3x3.npz): layer shapes exact, each
    layer's full operator within 1e-12 -- splits on step boundaries, inside
    steps, and with a partly filled last layer."""
    z = np.load(os.path.join(G, "tpocount_kinb3x3.npz"))
    edges = [tuple(int(v) for v in e) for e in z["edges"]]
    src = open(os.path.join(G, "inputs", "kinb3x3.qasm")).read()
    ns = len(bn.sites_of(edges))
    k = 0
    while f"split{k}" in z:
        split = [int(v) for v in z[f"split{k}"]]
        layers = tb.QasmToTPOByCount(src, edges, split)
        nl = 0
        while f"split{k}/{nl}/0" in z:
            nl += 1
        assert len(layers) == nl
        for l, layer in enumerate(layers):
            ref = [z[f"split{k}/{l}/{s}"] for s in range(ns)]
            got = [layer.site_op(edges, s) for s in range(ns)]
            assert [t.shape for t in got] == [t.shape for t in ref]
            np.testing.assert_allclose(full_operator(edges, got), full_operator(edges, ref), rtol=0, atol=1e-12)
        k += 1
    assert k == 4


def test_manual_gate_number_layering_errors():
    src = open(os.path.join(G, "inputs", "kinb3x3.qasm")).read()
    edges = tb.EdgesFromQasm(src)
    for split, code in (([21, 20], tb.EINVAL),        # more instructions than the counts cover
                        ([21, 21, 5], tb.EINVAL),     # a layer that receives nothing
                        ([0, 42], tb.EINVAL),         # a count < 1
                        ([], tb.EINVAL)):
        with pytest.raises(tb.TnbpError) as e:
            tb.QasmToTPOByCount(src, edges, split)
        assert e.value.code == code, split
    with pytest.raises(tb.TnbpError) as e:  # barriers are gates there: "matrix for this op not implemented"
        tb.QasmToTPOByCount(open(os.path.join(G, "inputs", "ki3x3.qasm")).read(),
                            tb.EdgesFromQasm(open(os.path.join(G, "inputs", "ki3x3.qasm")).read()), [500])
    assert e.value.code == tb.EUNSUPPORTED
