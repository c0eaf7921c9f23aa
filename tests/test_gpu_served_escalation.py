"""Requests whose BP does not converge, on the mixed path and in the server.

When a BP loop stops at its iteration limit (apps/estimator/main.cc:131-157
with the condition still above the tolerance), the messages it keeps depend
on every rounding of the sweeps before it, amplified: on the 8x8, chi 8,
12-step kicked-Ising request below, moving theta_h by one part in 1e13 moves
the complex128 result by ~1e-10, and the mixed path's ~1e-7 rounding moves it
by ~3e-4.  A mixed server with escalation on restarts such a request in
complex128, so its result is the plain path's (1e-10); a request that
converges stays on the mixed path (1e-6).  A non-converging request whose
value the rounding does not move (8x8, chi 16, 8 steps) stays within 1e-6
on the mixed path itself.  With an escalation threshold, only requests with
a BP loop whose condition never came below it are restarted.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

tb = pytest.importorskip("tnbp_b200")

THETA_J = -math.pi / 4
TOL_PLAIN = 1e-10
TOL_MIXED = 1e-6

NONCONV = (8, 8, 12, 1.1, 11)      # BP stops at 50 sweeps from step 5 on
NONCONV_OK = (8, 16, 8, 1.1, 12)   # BP stops at 50 sweeps; rounding not amplified past 1e-6
CONV = (8, 16, 6, 1.1, 13)         # every BP loop converges


def observable(L, seed, n_terms=8):
    """Random 1- to 4-qubit Pauli terms (X/Y/Z letters, N(0,1) coefficients)
    plus one single-site Z and one nearest-neighbour ZZ, so that terms of both
    kinds survive the reference's classification."""
    rng = np.random.default_rng(seed)
    n = L * L
    lines = []
    for _ in range(n_terms):
        k = int(rng.integers(1, 5))
        qs = rng.choice(n, size=k, replace=False)
        s = ["I"] * n
        for q, c in zip(qs, rng.choice(list("XYZ"), size=k)):
            s[n - 1 - int(q)] = str(c)
        lines.append(f"{float(rng.normal())!r} " + "".join(s))
    for coeff, qs in ((0.5, (0,)), (-0.25, (0, 1))):
        s = ["I"] * n
        for q in qs:
            s[n - 1 - q] = "Z"
        lines.append(f"{coeff} " + "".join(s))
    return tb.load_sparse_pauli("\n".join(lines) + "\n", tb.bond_square_lattice(L, L))


def plain(req, precision):
    """The plain per-job path; returns (sum, every BP loop converged)."""
    L, chi, nst, th, seed = req
    edges = tb.bond_square_lattice(L, L)
    layer = tb.KickedIsingTPO(edges, THETA_J / 2, 0.0, th / 2, 1.0)
    conv = True
    with tb.State(edges, precision) as st:
        t = st.tpo(layer)
        for _ in range(nst):
            tb.AbsorbTPO(st, t)
            _, c = tb.BeliefPropagationLoop(st, 1e-8, 50)
            conv = conv and c < 1e-8
            tb.Truncation(st, chi, 1e-8)
        total, _ = tb.MeasurePauliSum(st, observable(L, seed))
    return total, conv


def serve(reqs, escalate, threshold=0.0):
    srv = tb.Server(tb.MIXED, 0, 8)
    try:
        srv.set_escalation(escalate)
        srv.set_escalation_threshold(threshold)
        ids = [srv.submit_kicked_ising(L, chi, n, THETA_J, th, observable(L, seed)) for L, chi, n, th, seed in reqs]
        steps = 0
        while any(srv.result(i) is None for i in ids):
            srv.step()
            steps += 1
            assert steps < 100000
        return [srv.result(i) for i in ids], [srv.info(i) for i in ids]
    finally:
        srv.close()


def _run(info):
    return {k: info[k] for k in ("precision", "escalated", "bp_converged")}


def _need_gpu():
    if not tb.device_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")


def test_escalated_request_equals_the_plain_path():
    _need_gpu()
    p_non, conv_non = plain(NONCONV, tb.C128)
    p_conv, conv_conv = plain(CONV, tb.C128)
    assert not conv_non and conv_conv
    (v_non, v_conv), (i_non, i_conv) = serve([NONCONV, CONV], escalate=True)
    assert _run(i_non) == {"precision": tb.C128, "escalated": True, "bp_converged": False}
    assert _run(i_conv) == {"precision": tb.MIXED, "escalated": False, "bp_converged": True}
    assert i_conv["unconverged_loops"] == 0 and i_conv["worst_min_cond"] == 0.0
    assert abs(v_non - p_non) <= TOL_PLAIN, (v_non, p_non)
    assert abs(v_conv - p_conv) <= TOL_MIXED, (v_conv, p_conv)


def test_without_escalation_the_request_is_flagged_and_stays_mixed():
    _need_gpu()
    (v_non,), (i_non,) = serve([NONCONV], escalate=False)
    assert _run(i_non) == {"precision": tb.MIXED, "escalated": False, "bp_converged": False}
    assert i_non["unconverged_loops"] >= 1 and i_non["worst_final_cond"] >= i_non["worst_min_cond"] > 0
    assert math.isfinite(v_non.real) and math.isfinite(v_non.imag)


def test_nonconverging_request_within_1e6_on_the_mixed_path():
    _need_gpu()
    p, conv_p = plain(NONCONV_OK, tb.C128)
    m, conv_m = plain(NONCONV_OK, tb.MIXED)
    assert not conv_p and not conv_m
    assert abs(m - p) <= TOL_MIXED, (m, p)


def test_escalation_threshold_picks_the_ill_conditioned_loops():
    """With a threshold, only requests with a BP loop whose condition never
    fell below it are restarted (tnbp_server_set_escalation_threshold): the
    escalated set is exactly the one the non-escalating run's statistics
    name, and every value is within the mixed tolerance of the plain path
    (the escalated ones within the plain tolerance)."""
    _need_gpu()
    reqs = [NONCONV, NONCONV_OK, CONV]
    thr = 1e-2
    _, infos = serve(reqs, escalate=False)
    want = [i["worst_min_cond"] > thr for i in infos]
    assert want[0] and not want[2]
    vals, infos_e = serve(reqs, escalate=True, threshold=thr)
    assert [i["escalated"] for i in infos_e] == want
    for req, v, esc in zip(reqs, vals, want):
        p, _ = plain(req, tb.C128)
        assert abs(v - p) <= (TOL_PLAIN if esc else TOL_MIXED), (req, v, p)
