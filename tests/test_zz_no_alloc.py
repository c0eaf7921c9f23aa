"""tnbp_bp_message_noalloc: one BP message with no device allocation.

Callers that may not allocate device memory (a framework that owns the whole
HBM budget, or a stream-ordered pipeline that cannot take cudaMalloc's
implicit synchronization) pass device pointers for the site tensor, the
incoming messages and the output; the entry point uses only its static
scratch array.  Its output must equal the message the allocating sweep
(tnbp_bp_sweep) computes, to the 1e-12 of the complex128 sweep tests, on two
calls in a row over every (site, leg) of an uneven lattice.

This file is collected last so that a run stopping at the first failure has
run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

tb = pytest.importorskip("tnbp_b200")
torch = pytest.importorskip("torch")
import bp_numpy as bn  # noqa: E402

_fn = tb.lib.tnbp_bp_message_noalloc
_fn.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(C.c_void_p), C.c_void_p,
                C.c_void_p]
_fn.restype = C.c_int


def _dev(a):
    flat = np.ascontiguousarray(np.asarray(a, np.complex128).reshape(-1, order="F"))
    return torch.from_numpy(flat).to("cuda")


def _call(site_t, shape, target, msg_ts, out_t, stream):
    sh = (C.c_int32 * len(shape))(*shape)
    ptrs = (C.c_void_p * (len(shape) - 1))(*[(m.data_ptr() if m is not None else None) for m in msg_ts])
    return _fn(site_t.data_ptr(), sh, len(shape), target, ptrs, out_t.data_ptr(), stream)


def test_no_alloc_message_matches_sweep_on_two_calls():
    if not tb.device_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")
    rng = np.random.default_rng(42)
    edges = tb.bond_square_lattice(3, 3)
    dims = [int(x) for x in rng.integers(2, 17, size=len(edges))]
    sites = bn.sites_of(edges)
    V, E = [], []
    for s in sites:
        sh = [dims[m] for m in bn.bonds_of(edges, s)] + [2]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    for m in range(2 * len(edges)):
        D = dims[m % len(edges)]
        A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
        E.append(A @ A.conj().T / np.linalg.norm(A) ** 2)
    with tb.State(edges, tb.C128) as st:
        st.set_state(V, E)
        tb.BeliefPropagation(st)  # the allocating path
        F = st.get_E()
    stream = torch.cuda.current_stream().cuda_stream
    V_t = [_dev(v) for v in V]
    E_t = [_dev(e) for e in E]
    jobs = []
    for si, s in enumerate(sites):
        bonds = bn.bonds_of(edges, s)
        for t, m in enumerate(bonds):
            msgs = [None if k == t else E_t[bn.in_msg(edges, s, bonds[k])] for k in range(len(bonds))]
            jobs.append((si, list(V[si].shape), t, msgs, bn.out_msg(edges, s, m)))
    for order in (jobs, jobs[::-1]):  # two calls in a row over every message
        for si, shape, t, msgs, mo in order:
            out = torch.zeros(shape[t] * shape[t], dtype=torch.complex128, device="cuda")
            rc = _call(V_t[si], shape, t, msgs, out, stream)
            assert rc == 0, tb.lib.tnbp_last_error().decode()
            torch.cuda.synchronize()
            got = out.cpu().numpy().reshape(shape[t], shape[t], order="F")
            assert np.max(np.abs(got - F[mo])) <= 1e-12


def test_no_alloc_rejects_oversize_site_before_gpu_work():
    if not tb.device_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")
    shape = [64, 64, 64, 4, 2]  # 2,097,152 elements > TNBP_NOALLOC_MAX_SITE_ELEMS
    dummy = torch.zeros(4, dtype=torch.complex128, device="cuda")
    rc = _call(dummy, shape, 0, [None, dummy, dummy, dummy], dummy, torch.cuda.current_stream().cuda_stream)
    assert rc == tb.EINVAL
    assert "exceeds the no-allocation limit" in tb.lib.tnbp_last_error().decode()


def test_no_alloc_wide_and_rank2_back_to_back_allocates_nothing():
    """A 3-site chain with bond dimension 128 on both bonds: the middle site
    [128, 128, 2] (both targets, the widest dims the entry point takes) and
    the end sites [128, 2] (rank 2: no leg contraction, the Gram of the site
    with itself).  Every message is queued on one stream with no
    synchronization between the calls, then compared with the allocating
    sweep; the device's free memory is the same before and after the queued
    calls (the first call, which loads the kernels, comes before)."""
    if not tb.device_available():
        pytest.fail("no CUDA device: the GPU tests need a B200")
    rng = np.random.default_rng(7)
    edges = [(0, 1), (1, 2)]
    D = 128
    sites = bn.sites_of(edges)
    V, E = [], []
    for s in sites:
        sh = [D for _ in bn.bonds_of(edges, s)] + [2]
        V.append(rng.normal(size=sh) + 1j * rng.normal(size=sh))
    for m in range(2 * len(edges)):
        A = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
        E.append(A @ A.conj().T / np.linalg.norm(A) ** 2)
    with tb.State(edges, tb.C128) as st:
        st.set_state(V, E)
        tb.BeliefPropagation(st)
        F = st.get_E()
    stream = torch.cuda.current_stream().cuda_stream
    V_t = [_dev(v) for v in V]
    E_t = [_dev(e) for e in E]
    jobs = []
    for si, s in enumerate(sites):
        bonds = bn.bonds_of(edges, s)
        for t, m in enumerate(bonds):
            msgs = [None if k == t else E_t[bn.in_msg(edges, s, bonds[k])] for k in range(len(bonds))]
            jobs.append((si, list(V[si].shape), t, msgs, bn.out_msg(edges, s, m)))
    assert sorted(len(j[1]) for j in jobs) == [2, 2, 3, 3]
    outs = [torch.zeros(j[1][j[2]] ** 2, dtype=torch.complex128, device="cuda") for j in jobs * 2]
    warm = torch.zeros(D * D, dtype=torch.complex128, device="cuda")
    mid = next(j for j in jobs if len(j[1]) == 3)
    assert _call(V_t[mid[0]], mid[1], mid[2], mid[3], warm, stream) == 0, tb.lib.tnbp_last_error().decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k, (si, shape, t, msgs, mo) in enumerate(jobs + jobs[::-1]):
        rc = _call(V_t[si], shape, t, msgs, outs[k], stream)
        assert rc == 0, tb.lib.tnbp_last_error().decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for k, (si, shape, t, msgs, mo) in enumerate(jobs + jobs[::-1]):
        got = outs[k].cpu().numpy().reshape(shape[t], shape[t], order="F")
        # each call overwrites the shared scratch; the output buffers are the
        # caller's, so every queued result stays intact
        assert np.max(np.abs(got - F[mo])) <= 1e-12
