"""The served estimator path (continuous batching, tnbp_server_*).

Requests of different lattice sides, bond dimensions and depths share every
batched BP sweep launch.  Each task of a batched launch is computed from its
own job's data with a fixed reduction order, and the kernel that runs a task
depends only on that task's dimensions, so a request's result must not
depend on what it was batched with: the tests below require the result of
every request in a mix (staggered arrivals, a queue behind a slot limit) to
equal its result alone to 1e-12 absolute, and the complex128 server to equal
the plain per-job path (InitTensorProductState / AbsorbTPO /
BeliefPropagationLoop / Truncation / Measure) to 1e-10.  The mixed
(TNBP_MIXED) server is within 1e-6 of the complex128 path, the
complex64-storage server within 1e-5.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

tb = pytest.importorskip("tnbp_b200")

THETA_J = -math.pi / 4
TOL_MIX = 1e-12  # alone vs in the mix (the same arithmetic on the same data)
TOL_PLAIN = 1e-10  # complex128 server vs the plain per-job path
TOL_MIXED = 1e-6  # mixed server (complex128 state) vs the complex128 path
# complex64 storage rounds the state about three times per Floquet step;
# per-term errors reach ~1e-6 here, so that mode is held to 1e-5
TOL_C64 = 1e-5

# (L, chi, steps, theta_h, seed of the observable); the chi = 32 request
# reaches BP at D = 64 in its last step, so the batches mix the D <= 32 and
# the 32 < D <= 64 tensor-core kernels with the CUDA-core ones
REQUESTS = [(4, 4, 4, 0.55, 1), (3, 8, 5, 0.30, 2), (5, 2, 3, 0.90, 3), (4, 8, 3, 1.10, 4),
            (6, 4, 3, 0.70, 5), (3, 2, 6, 0.40, 6), (3, 32, 6, 0.45, 7)]


def observable(L, seed, n_terms=8):
    """8-term random observable: 1 to 4 distinct qubits, letters in {X,Y,Z},
    coefficients N(0,1), plus one single-site Z and one nearest-neighbour ZZ
    so that every request keeps terms of both kinds after the reference's
    classification drops non-adjacent and >2-qubit terms."""
    rng = np.random.default_rng(seed)
    n = L * L
    lines = []
    for _ in range(n_terms):
        k = int(rng.integers(1, 5))
        qs = rng.choice(n, size=k, replace=False)
        letters = rng.choice(list("XYZ"), size=k)
        s = ["I"] * n
        for q, c in zip(qs, letters):
            s[n - 1 - int(q)] = str(c)
        lines.append(f"{float(rng.normal())!r} " + "".join(s))
    s = ["I"] * n
    s[n - 1 - 0] = "Z"
    lines.append("0.5 " + "".join(s))
    s = ["I"] * n
    s[n - 1 - 0] = "Z"
    s[n - 1 - 1] = "Z"
    lines.append("-0.25 " + "".join(s))
    edges = tb.bond_square_lattice(L, L)
    return tb.load_sparse_pauli("\n".join(lines) + "\n", edges)


def run_server(reqs, precision, max_active=64, stagger=0):
    """Submit `reqs` (arriving `stagger` server steps apart) and step until
    all are done; returns the results in submission order."""
    srv = tb.Server(precision, 0, max_active)
    try:
        ids, pending = [], list(reqs)
        steps = 0
        while pending or any(srv.result(i) is None for i in ids):
            if pending and (stagger == 0 or steps % stagger == 0):
                L, chi, nst, th, seed = pending.pop(0)
                ids.append(srv.submit_kicked_ising(L, chi, nst, THETA_J, th, observable(L, seed)))
                if stagger == 0:
                    continue
            srv.step()
            steps += 1
            assert steps < 100000
        return [srv.result(i) for i in ids]
    finally:
        srv.close()


def plain(req, precision=tb.C128):
    L, chi, nst, th, seed = req
    edges = tb.bond_square_lattice(L, L)
    layer = tb.KickedIsingTPO(edges, THETA_J / 2, 0.0, th / 2, 1.0)
    with tb.State(edges, precision) as st:
        t = st.tpo(layer)
        for _ in range(nst):
            tb.AbsorbTPO(st, t)
            tb.BeliefPropagationLoop(st, 1e-8, 50)
            tb.Truncation(st, chi, 1e-8)
        total, _ = tb.MeasurePauliSum(st, observable(L, seed))
    return total


def _need_gpu():
    if not tb.device_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")


@pytest.mark.parametrize("precision", [tb.MIXED, tb.C64, tb.C128])
def test_each_result_is_the_same_alone_and_in_the_mix(precision):
    _need_gpu()
    alone = [run_server([r], precision)[0] for r in REQUESTS]
    together = run_server(REQUESTS, precision)
    staggered = run_server(REQUESTS, precision, stagger=3)
    queued = run_server(REQUESTS, precision, max_active=2, stagger=1)
    for a, b, c, d in zip(alone, together, staggered, queued):
        assert abs(a - b) <= TOL_MIX and abs(a - c) <= TOL_MIX and abs(a - d) <= TOL_MIX, (a, b, c, d)


def test_c128_server_equals_plain_path_and_mixed_is_within_1e6():
    _need_gpu()
    served128 = run_server(REQUESTS, tb.C128, stagger=2)
    served_mixed = run_server(REQUESTS, tb.MIXED, stagger=2)
    served64 = run_server(REQUESTS, tb.C64, stagger=2)
    for r, s128, sm, s64 in zip(REQUESTS, served128, served_mixed, served64):
        p = plain(r)
        assert abs(s128 - p) <= TOL_PLAIN, (r, s128, p)
        assert abs(sm - p) <= TOL_MIXED, (r, sm, p)
        assert abs(s64 - p) <= TOL_C64, (r, s64, p)


def test_admission_rejects_a_request_larger_than_the_budget():
    _need_gpu()
    srv = tb.Server(tb.MIXED, 64 << 20, 4)  # 64 MiB budget
    try:
        with pytest.raises(tb.TnbpError) as e:
            srv.submit_kicked_ising(12, 32, 4, THETA_J, 0.5, observable(12, 1))
        assert e.value.code == tb.ENOMEM
    finally:
        srv.close()


def test_cancelled_requests_leave_the_others_unchanged():
    """tnbp_server_cancel between steps: a queued request and an admitted one
    are cancelled (TNBP_ECANCELED); the remaining request's result equals its
    result alone, and the freed slot admits the next queued request."""
    _need_gpu()
    keep, drop_active, drop_queued, later = REQUESTS[0], REQUESTS[1], REQUESTS[2], REQUESTS[4]
    alone = run_server([keep], tb.MIXED)[0]
    alone_later = run_server([later], tb.MIXED)[0]
    srv = tb.Server(tb.MIXED, 0, 2)
    try:
        ids = []
        for L, chi, nst, th, seed in (keep, drop_active, drop_queued, later):
            ids.append(srv.submit_kicked_ising(L, chi, nst, THETA_J, th, observable(L, seed)))
        srv.step()
        srv.step()  # two admitted (slot limit 2), two queued
        srv.cancel(ids[1])
        srv.cancel(ids[2])
        steps = 0
        while srv.result(ids[0]) is None or srv.result(ids[3]) is None:
            srv.step()
            steps += 1
            assert steps < 100000
        for i in (1, 2):
            with pytest.raises(tb.TnbpError) as e:
                srv.result(ids[i])
            assert e.value.code == tb.ECANCELED
        assert abs(srv.result(ids[0]) - alone) <= TOL_MIX
        assert abs(srv.result(ids[3]) - alone_later) <= TOL_MIX
        srv.cancel(ids[0])  # finished: no-op
        assert abs(srv.result(ids[0]) - alone) <= TOL_MIX
    finally:
        srv.close()
