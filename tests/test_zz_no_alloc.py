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
