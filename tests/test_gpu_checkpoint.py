"""Checkpoint / resume of the device state (tnbp_save_state / tnbp_load_state,
the SaveTPS / LoadTPS of include/tnbp/ptns/function/iotps.h:37-105 as the
reference's apps/estimator_restart uses them).

* A checkpoint the reference app saved after one pass of a 3x3 kicked-Ising
  circuit, loaded into a job and run through a second pass on the device,
  gives the values the reference app printed after the same restart
  (1e-9 complex128; 5e-6 mixed: BP restarts far from its fixed point here --
  first condition 1e-3, about 11 sweeps per layer -- and the reduced-precision
  stop at a condition of 1e-7 leaves ~1.5e-6 on some terms) and, in
  complex128, the same bond dimensions.
* Save, load into a fresh job and continue: identical to the job that was
  never interrupted (bit for bit, complex128).
* A file that does not belong to the job's lattice is refused and leaves
  the job's state as it was.
"""
import json
import os

import numpy as np
import pytest

import bp_numpy as bn

pytestmark = pytest.mark.gpu
tb = pytest.importorskip("tnbp_b200")
HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden")
NAME = "ki3x3r"


def _inputs():
    src = open(os.path.join(G, "inputs", f"{NAME}.qasm")).read()
    pauli = open(os.path.join(G, "inputs", f"{NAME}.txt")).read()
    meta = json.load(open(os.path.join(G, f"ckpt_{NAME}.json")))
    return src, pauli, meta


def _pass(st, layers, meta):
    dims = []
    for layer in layers:
        tb.AbsorbTPO(st, layer)
        tb.BeliefPropagationLoop(st, meta["tol"], meta["maxit"])
        d, _ = tb.Truncation(st, meta["chi"], meta["sv_min"])
        dims += [int(x) for x in d]
    return dims


def _reference_order(pauli, edges, per):
    """Per-term values in the order the restart app prints them: one-site
    terms, then two-site terms, each in file order."""
    ref_terms, _ = bn.parse_pauli_text(pauli, edges)
    k1 = [i for i, t in enumerate(ref_terms) if t[0] == 1]
    k2 = [i for i, t in enumerate(ref_terms) if t[0] == 2]
    return [per[i].real for i in k1], [per[i].real for i in k2]


@pytest.mark.parametrize("prec,tol", [(tb.C128, 1e-9), (tb.MIXED, 5e-6)])
def test_resume_from_the_reference_checkpoint(prec, tol):
    src, pauli, meta = _inputs()
    edges = tb.EdgesFromQasm(src)
    layers = tb.QasmToTPO(src, edges)
    with tb.State(edges, prec) as st:
        st.load(os.path.join(G, f"ckpt_{NAME}000000.dat"))
        assert max(st.bond_dims()) == 4
        dims = _pass(st, layers, meta)
        _, per = tb.MeasurePauliSum(st, tb.load_sparse_pauli(pauli, edges))
    if prec == tb.C128:
        assert dims == meta["bond_dims"]
    one, two = _reference_order(pauli, edges, per)
    assert len(one) == len(meta["one"])
    assert len(two) >= len(meta["two"])
    for a, b in zip(one + two[: len(meta["two"])], meta["one"] + meta["two"]):
        assert abs(a - b) <= tol, (a, b)


def test_save_load_continue_is_bit_identical(tmp_path):
    src, pauli, meta = _inputs()
    edges = tb.EdgesFromQasm(src)
    layers = tb.QasmToTPO(src, edges)
    terms = tb.load_sparse_pauli(pauli, edges)
    path = str(tmp_path / "ck.dat")
    with tb.State(edges, tb.C128) as a, tb.State(edges, tb.C128) as b:
        _pass(a, layers, meta)
        a.save(path)
        # the file holds exactly the device state
        V, E = tb.LoadTPS(path, edges)
        for x, y in zip(V + E, a.get_V() + a.get_E()):
            np.testing.assert_array_equal(x, y)
        b.load(path)
        for x, y in zip(a.get_V() + a.get_E(), b.get_V() + b.get_E()):
            np.testing.assert_array_equal(x, y)
        da = _pass(a, layers, meta)
        db = _pass(b, layers, meta)
        assert da == db
        ta, pa = tb.MeasurePauliSum(a, terms)
        tb_, pb = tb.MeasurePauliSum(b, terms)
        np.testing.assert_array_equal(pa, pb)
        assert ta == tb_


def test_load_refuses_another_lattice_and_keeps_the_state(tmp_path):
    src, pauli, meta = _inputs()
    edges = tb.EdgesFromQasm(src)
    layers = tb.QasmToTPO(src, edges)
    other = tb.bond_square_lattice(4, 3)
    path = str(tmp_path / "other.dat")
    with tb.State(other, tb.C128) as o:
        o.save(path)
    with tb.State(edges, tb.C128) as st:
        tb.AbsorbTPO(st, layers[0])
        before = st.get_V() + st.get_E()
        with pytest.raises(tb.TnbpError):
            st.load(path)
        for x, y in zip(before, st.get_V() + st.get_E()):
            np.testing.assert_array_equal(x, y)
        tb.BeliefPropagationLoop(st, meta["tol"], meta["maxit"])
