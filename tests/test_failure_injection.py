"""Failures injected on the host, none of which may reach the device: a
non-finite gate angle (the reference's strtod turns "1e400" into inf and
builds NaN operators silently), non-finite Floquet parameters, a NaN in a
TPO layer handed to OptTPObySVD, an out-of-range coefficient in an
observable, and state calls without a device.  Each ends in a status code
(TnbpError), not a crash.  Runs on the CPU."""
import numpy as np
import pytest

tb = pytest.importorskip("tnbp_b200")

SRC = 'OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg q[2];\ncx q[0],q[1];\nrx({}) q[0];\n'


def test_non_finite_gate_angle_is_refused():
    edges = tb.EdgesFromQasm(SRC.format("0.3"))
    assert len(tb.QasmToTPO(SRC.format("0.3"), edges)) == 1
    ins = tb.qasm_instructions(SRC.format("1e400"))  # parsing keeps the reference's value
    assert any(np.isinf(p) for i in ins for p in i[2])
    with pytest.raises(tb.TnbpError) as e:
        tb.QasmToTPO(SRC.format("1e400"), edges)
    assert e.value.code == tb.EINVAL and "non-finite" in str(e.value)


def test_non_finite_floquet_parameters_are_refused():
    edges = tb.bond_square_lattice(2, 2)
    with pytest.raises(tb.TnbpError) as e:
        tb.KickedIsingTPO(edges, float("nan"), 0.0, 0.4, 1.0)
    assert e.value.code == tb.EINVAL


def test_nan_operator_element_is_refused_by_opt_tpo():
    edges = tb.EdgesFromQasm(SRC.format("0.3"))
    layer = tb.QasmToTPO(SRC.format("0.3"), edges)[0]
    layer.op_data = layer.op_data.copy()
    layer.op_data[3] = complex("nan")
    with pytest.raises(tb.TnbpError) as e:
        tb.OptTPObySVD(edges, layer, 1e-8)
    assert e.value.code == tb.EINVAL


def test_out_of_range_coefficient_is_a_parse_error():
    with pytest.raises(tb.TnbpError) as e:
        tb.load_sparse_pauli("1e400 ZZ\n", [(0, 1)])
    assert e.value.code == tb.EPARSE


def test_device_calls_fail_loudly_without_a_device():
    if tb.device_available():
        pytest.skip("a device is visible")
    for make in (lambda: tb.State([(0, 1)]), lambda: tb.Server(tb.MIXED, 0, 4)):
        with pytest.raises(tb.TnbpError) as e:
            make()
        assert e.value.code == tb.ENOGPU
