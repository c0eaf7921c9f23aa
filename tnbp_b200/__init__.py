"""tnbp_b200: B200-native (sm_100a) loopy-BP PEPS expectation-value engine.

Python face of the C ABI in include/tnbp_b200.h (libtnbp_b200.so, built
in-tree by tnbp_b200.build).  The functions below carry the names and the
argument meaning of r-ccs-cms/tnbp's estimator entry points
(include/tnbp/ptns/function/*.h); the state they act on lives on the GPU
inside a `State` handle instead of caller-owned std::vectors.

There is no CPU path: loading the library without a CUDA device works (for
the host-side builders), but every state call raises `TnbpError` with code
TNBP_ENOGPU, and importing without a built library raises ImportError.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtnbp_b200.so")

C128, C64, MIXED = 0, 1, 2
OK, EINVAL, ECUDA, ENOMEM, ENOTCONV, EPARSE, EUNSUPPORTED, ENOGPU, ECANCELED = 0, -1, -2, -3, -4, -5, -6, -7, -8


class TnbpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `python tnbp_b200/build.py` (nvcc, sm_100a)")
    return C.CDLL(LIB_PATH)


lib = _load()
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p
lib.tnbp_last_error.restype = C.c_char_p
lib.tnbp_version.restype = C.c_char_p

_SIGS = {
    "tnbp_device_available": [],
    "tnbp_square_lattice": [C.c_int32, C.c_int32, _i32p, C.c_int64, _i64p],
    "tnbp_greedy_layering": [_i32p, C.c_int64, _i32p, _i32p],
    "tnbp_surrounding_bonds": [_i32p, C.c_int64, C.c_int32, _i32p, C.c_int32, _i32p],
    "tnbp_shortest_path": [_i32p, C.c_int64, C.c_int32, C.c_int32, _i32p, C.c_int32, _i32p],
    "tnbp_qasm_edges": [C.c_char_p, _i32p, C.c_int64, _i64p],
    "tnbp_qasm_instructions": [C.c_char_p, _i32p, _i32p, _i32p, _i32p, _f64p, C.c_int64, _i64p],
    "tnbp_pauli_terms": [C.c_char_p, _i32p, C.c_int64, _i32p, _i32p, _i32p, C.c_char_p, _f64p, _i32p,
                         C.c_int64, _i64p, _i64p],
    "tnbp_qasm_tpo": [C.c_char_p, _i32p, C.c_int64, _i32p, _i64p, _f64p, C.c_int64, _i32p, _i64p],
    "tnbp_qasm_tpo_counts": [C.c_char_p, _i32p, C.c_int64, _i32p, C.c_int32, _i32p, _i64p, _f64p, C.c_int64, _i32p,
                             _i64p],
    "tnbp_kicked_ising_tpo": [_i32p, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, _i32p, _i64p,
                              _f64p, C.c_int64, _i64p],
    "tnbp_opt_tpo_svd": [_i32p, C.c_int64, C.c_double, _i32p, _i64p, _f64p, _i64p],
    "tnbp_tps_write": [C.c_char_p, _i32p, C.c_int64, _i32p, _i32p, _f64p, _f64p],
    "tnbp_tps_read": [C.c_char_p, _i32p, C.c_int64, _i32p, _i32p, _f64p, C.c_int64, _f64p, C.c_int64, _i64p,
                      _i64p],
    "tnbp_save_state": [_vp, C.c_char_p],
    "tnbp_load_state": [_vp, C.c_char_p],
    "tnbp_job_create": [_i32p, C.c_int64, _i32p, C.c_int32, _vp, C.c_uint64, C.POINTER(_vp)],
    "tnbp_job_destroy": [_vp],
    "tnbp_job_info": [_vp, _i64p, _i64p, _i32p],
    "tnbp_job_device_bytes": [_vp, _u64p],
    "tnbp_footprint_estimate": [_i32p, C.c_int64, _i32p, C.c_int32, _u64p],
    "tnbp_bond_dims": [_vp, _i32p],
    "tnbp_site_shape": [_vp, C.c_int64, _i32p, C.c_int32, _i32p],
    "tnbp_download_site": [_vp, C.c_int64, _f64p, C.c_int64],
    "tnbp_upload_site": [_vp, C.c_int64, _i32p, C.c_int32, _f64p],
    "tnbp_download_message": [_vp, C.c_int64, _f64p, C.c_int64, _i32p],
    "tnbp_upload_message": [_vp, C.c_int64, C.c_int32, _f64p],
    "tnbp_tpo_create": [_vp, _i32p, _i64p, _f64p, C.POINTER(_vp)],
    "tnbp_tpo_destroy": [_vp],
    "tnbp_absorb_tpo": [_vp, _vp],
    "tnbp_bp_sweep": [_vp],
    "tnbp_bp_condition": [_vp, _f64p],
    "tnbp_bp_run": [_vp, C.c_double, C.c_int32, _i32p, _f64p],
    "tnbp_truncate": [_vp, C.c_int32, C.c_double, _i32p, _f64p],
    "tnbp_measure_1site": [_vp, C.c_int64, _i64p, _f64p, _f64p],
    "tnbp_measure_2site": [_vp, C.c_int64, _i32p, _f64p, _f64p],
    "tnbp_measure_pauli_sum": [_vp, C.c_int64, _i32p, _i32p, _i32p, C.c_char_p, _f64p, _f64p, _f64p],
    "tnbp_measure_cluster": [_vp, C.c_int64, _i32p, _i32p, C.c_char_p, _f64p, _f64p, _f64p],
    "tnbp_measure_pauli_text": [_vp, C.c_char_p, C.c_int32, _f64p, _i32p, C.c_int64, _i64p, _f64p],
    "tnbp_sweep_stats": [_vp, _f64p, _f64p, _f64p],
    "tnbp_sweep_totals": [_vp, _f64p, _f64p, _f64p, _i64p],
    "tnbp_server_create": [C.c_int32, C.c_uint64, C.c_int32, C.POINTER(_vp)],
    "tnbp_server_destroy": [_vp],
    "tnbp_server_submit_kicked_ising": [_vp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                        C.c_double, C.c_int32, C.c_double, C.c_int64, _i32p, _i32p, _i32p,
                                        C.c_char_p, _f64p, _i64p],
    "tnbp_server_submit_qasm": [_vp, C.c_char_p, C.c_char_p, C.c_int32, C.c_double, C.c_int32, C.c_double,
                                C.c_int32, C.c_double, _i64p],
    "tnbp_server_tpo_cache_stats": [_vp, _i64p, _i64p, _i64p],
    "tnbp_server_cancel": [_vp, C.c_int64],
    "tnbp_server_step": [_vp, _i32p, _i32p, _i32p],
    "tnbp_server_result": [_vp, C.c_int64, _f64p, _i32p],
    "tnbp_server_set_escalation": [_vp, C.c_int32],
    "tnbp_server_request_info": [_vp, C.c_int64, _i32p, _i32p, _i32p],
    "tnbp_server_set_escalation_threshold": [_vp, C.c_double],
    "tnbp_server_request_bp_stats": [_vp, C.c_int64, _i32p, _f64p, _f64p],
}
for _n, _a in _SIGS.items():
    _f = getattr(lib, _n)
    _f.argtypes = _a
    _f.restype = C.c_int
lib.tnbp_kernel_launches.argtypes = []
lib.tnbp_kernel_launches.restype = C.c_ulonglong


def kernel_launches():
    """Kernels launched by this process through the library so far."""
    return int(lib.tnbp_kernel_launches())


def _chk(rc):
    if rc != OK:
        raise TnbpError(rc, lib.tnbp_last_error().decode(errors="replace"))


def _p(a, t):
    return a.ctypes.data_as(t)


def _edges_arr(edges):
    return np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))


def _c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def device_available():
    return bool(lib.tnbp_device_available())


def version():
    return lib.tnbp_version().decode()


# ----------------------------------------------------------- host builders
def bond_square_lattice(Lx, Ly):
    """bond_square_lattice (include/tnbp/lattice/square.h:14-34)."""
    n = C.c_int64()
    _chk(lib.tnbp_square_lattice(Lx, Ly, None, 0, C.byref(n)))
    out = np.zeros((n.value, 2), np.int32)
    _chk(lib.tnbp_square_lattice(Lx, Ly, _p(out, _i32p), n.value, C.byref(n)))
    return [tuple(map(int, e)) for e in out]


def GreedyEdgeLayering(edges):
    """GreedyEdgeLayering (graph.h:138-170): list of layers of edges."""
    e = _edges_arr(edges)
    lay = np.zeros(len(e), np.int32)
    nl = C.c_int32()
    _chk(lib.tnbp_greedy_layering(_p(e, _i32p), len(e), _p(lay, _i32p), C.byref(nl)))
    return [[tuple(map(int, e[i])) for i in range(len(e)) if lay[i] == l] for l in range(nl.value)]


def GetSurroundingBondIndex(site, edges):
    e = _edges_arr(edges)
    out = np.zeros(max(1, len(e) * 2), np.int32)
    n = C.c_int32()
    _chk(lib.tnbp_surrounding_bonds(_p(e, _i32p), len(e), site, _p(out, _i32p), len(out), C.byref(n)))
    return [int(x) for x in out[: n.value]]


def GetSiteIndexFromBond(edges):
    return sorted({int(v) for e in edges for v in e})


def FindShortestPath(edges, src, dst):
    e = _edges_arr(edges)
    out = np.zeros(max(1, len(e) + 2), np.int32)
    n = C.c_int32()
    _chk(lib.tnbp_shortest_path(_p(e, _i32p), len(e), src, dst, _p(out, _i32p), len(out), C.byref(n)))
    return [int(x) for x in out[: n.value]]


def EdgesFromQasm(src):
    s = src.encode()
    n = C.c_int64()
    _chk(lib.tnbp_qasm_edges(s, None, 0, C.byref(n)))
    out = np.zeros((max(n.value, 1), 2), np.int32)
    _chk(lib.tnbp_qasm_edges(s, _p(out, _i32p), n.value, C.byref(n)))
    return [tuple(map(int, e)) for e in out[: n.value]]


def qasm_instructions(src):
    """qasm::parse_any: list of (op enumerator, qubits, params)."""
    s = src.encode()
    n = C.c_int64()
    _chk(lib.tnbp_qasm_instructions(s, None, None, None, None, None, 0, C.byref(n)))
    k = n.value
    op = np.zeros(k, np.int32)
    nq = np.zeros(k, np.int32)
    qs = np.zeros(4 * k, np.int32)
    npar = np.zeros(k, np.int32)
    par = np.zeros(3 * k, np.float64)
    if k:
        _chk(lib.tnbp_qasm_instructions(s, _p(op, _i32p), _p(nq, _i32p), _p(qs, _i32p), _p(npar, _i32p),
                                        _p(par, _f64p), k, C.byref(n)))
    out = []
    for i in range(k):
        out.append((int(op[i]), [int(q) for q in qs[4 * i: 4 * i + min(4, nq[i])]],
                    [float(x) for x in par[3 * i: 3 * i + npar[i]]], int(nq[i])))
    return out


class PauliTerms:
    """Kept terms of a sparse Pauli observable (load_sparse_pauli_op +
    ClassifyOps): arrays kind, q0, q1, letters (2 chars each), coeff
    (complex), row (line order)."""

    def __init__(self, kind, q0, q1, letters, coeff, row, dropped):
        self.kind, self.q0, self.q1, self.letters = kind, q0, q1, letters
        self.coeff, self.row, self.dropped = coeff, row, dropped

    def __len__(self):
        return len(self.kind)


def load_sparse_pauli(text, edges):
    e = _edges_arr(edges)
    s = text.encode()
    nk, nd = C.c_int64(), C.c_int64()
    _chk(lib.tnbp_pauli_terms(s, _p(e, _i32p), len(e), None, None, None, None, None, None, 0, C.byref(nk),
                              C.byref(nd)))
    k = nk.value
    kind = np.zeros(max(k, 1), np.int32)
    q0 = np.zeros(max(k, 1), np.int32)
    q1 = np.zeros(max(k, 1), np.int32)
    let = C.create_string_buffer(2 * max(k, 1))
    co = np.zeros(2 * max(k, 1), np.float64)
    row = np.zeros(max(k, 1), np.int32)
    if k:
        _chk(lib.tnbp_pauli_terms(s, _p(e, _i32p), len(e), _p(kind, _i32p), _p(q0, _i32p), _p(q1, _i32p), let,
                                  _p(co, _f64p), _p(row, _i32p), k, C.byref(nk), C.byref(nd)))
    return PauliTerms(kind[:k], q0[:k], q1[:k], let.raw[: 2 * k], co[: 2 * k].view(np.complex128), row[:k],
                      nd.value)


class TPOLayer:
    """One TPO layer: edge_rank[ne], op_offset[ns] (complex elements) and the
    packed complex128 op data, each site op of shape (r_legs..., 2, 2)."""

    def __init__(self, edge_rank, op_offset, op_data):
        self.edge_rank = np.ascontiguousarray(edge_rank, np.int32)
        self.op_offset = np.ascontiguousarray(op_offset, np.int64)
        self.op_data = _c128(op_data)

    @staticmethod
    def from_ops(edges, ops):
        """Pack per-site op tensors O[s] (numpy, shape (r_0..r_{g-1}, 2, 2))."""
        sites = GetSiteIndexFromBond(edges)
        rank = np.ones(len(edges), np.int32)
        off, data, o = [], [], 0
        for si, s in enumerate(sites):
            for k, m in enumerate(GetSurroundingBondIndex(s, edges)):
                rank[m] = ops[si].shape[k]
            off.append(o)
            flat = np.asarray(ops[si], np.complex128).reshape(-1, order="F")
            data.append(flat)
            o += flat.size
        return TPOLayer(rank, off, np.concatenate(data))

    def site_op(self, edges, si):
        sites = GetSiteIndexFromBond(edges)
        bonds = GetSurroundingBondIndex(sites[si], edges)
        shape = [int(self.edge_rank[m]) for m in bonds] + [2, 2]
        n = int(np.prod(shape))
        return self.op_data[self.op_offset[si]: self.op_offset[si] + n].reshape(shape, order="F")


def _layers(ne, ns, nl, rank, off, data):
    return [TPOLayer(rank[l * ne:(l + 1) * ne], off[l * ns:(l + 1) * ns], data) for l in range(nl)]


def QasmToTPO(src, edges):
    """QasmToTPO, barrier layering (qasmtotpo.h:743-767)."""
    e = _edges_arr(edges)
    ns = len(GetSiteIndexFromBond(edges))
    s = src.encode()
    nl, nel = C.c_int32(), C.c_int64()
    _chk(lib.tnbp_qasm_tpo(s, _p(e, _i32p), len(e), None, None, None, 0, C.byref(nl), C.byref(nel)))
    rank = np.zeros(max(1, nl.value * len(e)), np.int32)
    off = np.zeros(max(1, nl.value * ns), np.int64)
    data = np.zeros(2 * max(1, nel.value), np.float64)
    _chk(lib.tnbp_qasm_tpo(s, _p(e, _i32p), len(e), _p(rank, _i32p), _p(off, _i64p), _p(data, _f64p),
                           max(1, nel.value), C.byref(nl), C.byref(nel)))
    return _layers(len(e), ns, nl.value, rank, off, data.view(np.complex128))


def QasmToTPOByCount(src, edges, num_gates):
    """QasmToTPO with manual gate-number layering (qasmtotpo.h:709-738)."""
    e = _edges_arr(edges)
    ns = len(GetSiteIndexFromBond(edges))
    s = src.encode()
    ng = np.ascontiguousarray(num_gates, np.int32)
    nl, nel = C.c_int32(), C.c_int64()
    _chk(lib.tnbp_qasm_tpo_counts(s, _p(e, _i32p), len(e), _p(ng, _i32p), len(ng), None, None, None, 0,
                                  C.byref(nl), C.byref(nel)))
    rank = np.zeros(max(1, nl.value * len(e)), np.int32)
    off = np.zeros(max(1, nl.value * ns), np.int64)
    data = np.zeros(2 * max(1, nel.value), np.float64)
    _chk(lib.tnbp_qasm_tpo_counts(s, _p(e, _i32p), len(e), _p(ng, _i32p), len(ng), _p(rank, _i32p), _p(off, _i64p),
                                  _p(data, _f64p), max(1, nel.value), C.byref(nl), C.byref(nel)))
    return _layers(len(e), ns, nl.value, rank, off, data.view(np.complex128))


def KickedIsingTPO(edges, Jz, hz, hx, dt):
    """One Floquet step (apps/kicked_ising_lattice/circuit.h:14-229)."""
    e = _edges_arr(edges)
    ns = len(GetSiteIndexFromBond(edges))
    nel = C.c_int64()
    _chk(lib.tnbp_kicked_ising_tpo(_p(e, _i32p), len(e), Jz, hz, hx, dt, None, None, None, 0, C.byref(nel)))
    rank = np.zeros(len(e), np.int32)
    off = np.zeros(ns, np.int64)
    data = np.zeros(2 * nel.value, np.float64)
    _chk(lib.tnbp_kicked_ising_tpo(_p(e, _i32p), len(e), Jz, hz, hx, dt, _p(rank, _i32p), _p(off, _i64p),
                                   _p(data, _f64p), nel.value, C.byref(nel)))
    return TPOLayer(rank, off, data.view(np.complex128))


def OptTPObySVD(edges, layer, eps=1.0e-8):
    """OptTPObySVD (optsvdtpo.h:86-214): compress every operator bond of one
    TPO layer by a truncated SVD (singular values > eps kept), in place as
    the reference updates its container; returns the layer."""
    e = _edges_arr(edges)
    rank = layer.edge_rank.copy()
    off = layer.op_offset - layer.op_offset.min() if len(layer.op_offset) else layer.op_offset.copy()
    lo = int(layer.op_offset.min()) if len(layer.op_offset) else 0
    data = np.ascontiguousarray(layer.op_data[lo:]).view(np.float64).copy()
    nel = C.c_int64()
    _chk(lib.tnbp_opt_tpo_svd(_p(e, _i32p), len(e), float(eps), _p(rank, _i32p), _p(off, _i64p),
                              _p(data, _f64p), C.byref(nel)))
    layer.edge_rank = rank
    layer.op_offset = off
    layer.op_data = data.view(np.complex128)[: nel.value].copy()
    return layer


def SaveTPS(path, edges, V, E):
    """SaveTPS (iotps.h:37-67) of a whole single-rank state held on the host:
    V[s] site tensors in sorted-site order, E[m] the 2|E| messages."""
    e = _edges_arr(edges)
    sites = GetSiteIndexFromBond(edges)
    bond = np.array([np.asarray(E[m]).shape[0] for m in range(len(e))], np.int32)
    phys = np.array([np.asarray(v).shape[-1] for v in V], np.int32)
    vdata = np.concatenate([_c128(v).reshape(-1, order="F") for v in V]) if len(sites) else np.zeros(1, np.complex128)
    mdata = np.concatenate([_c128(x).reshape(-1, order="F") for x in E]) if len(e) else np.zeros(1, np.complex128)
    _chk(lib.tnbp_tps_write(os.fsencode(path), _p(e, _i32p), len(e), _p(bond, _i32p), _p(phys, _i32p),
                            _p(vdata.view(np.float64), _f64p), _p(mdata.view(np.float64), _f64p)))


def LoadTPS(path, edges):
    """LoadTPS (iotps.h:69-105) of a whole single-rank checkpoint of `edges`:
    returns (V, E) as lists of complex128 arrays."""
    e = _edges_arr(edges)
    sites = GetSiteIndexFromBond(edges)
    bond = np.zeros(max(1, len(e)), np.int32)
    phys = np.zeros(max(1, len(sites)), np.int32)
    nv, nm = C.c_int64(), C.c_int64()
    s = os.fsencode(path)
    _chk(lib.tnbp_tps_read(s, _p(e, _i32p), len(e), None, None, None, 0, None, 0, C.byref(nv), C.byref(nm)))
    vdata = np.zeros(max(1, nv.value), np.complex128)
    mdata = np.zeros(max(1, nm.value), np.complex128)
    _chk(lib.tnbp_tps_read(s, _p(e, _i32p), len(e), _p(bond, _i32p), _p(phys, _i32p),
                           _p(vdata.view(np.float64), _f64p), nv.value, _p(mdata.view(np.float64), _f64p), nm.value,
                           C.byref(nv), C.byref(nm)))
    V, o = [], 0
    for si, site in enumerate(sites):
        shape = [int(bond[m]) for m in GetSurroundingBondIndex(site, edges)] + [int(phys[si])]
        n = int(np.prod(shape))
        V.append(vdata[o:o + n].reshape(shape, order="F").copy())
        o += n
    E, o = [], 0
    for m in range(2 * len(e)):
        D = int(bond[m % len(e)])
        E.append(mdata[o:o + D * D].reshape((D, D), order="F").copy())
        o += D * D
    return V, E


def footprint_estimate(edges, bond_dims, precision=C128):
    """Estimated peak device bytes of a job on `edges` with BP at the given
    bond dimension per edge (tnbp_footprint_estimate; host only)."""
    e = _edges_arr(edges)
    d = np.ascontiguousarray(bond_dims, np.int32)
    out = C.c_uint64()
    _chk(lib.tnbp_footprint_estimate(_p(e, _i32p), len(e), _p(d, _i32p), precision, C.byref(out)))
    return out.value


# ------------------------------------------------------------------ state
class State:
    """Device-resident PEPS of one job (site tensors and both message
    arenas).  Created in the product state |0...0>
    (InitTensorProductState, include/tnbp/ptns/function/init.h:18-95)."""

    def __init__(self, edges, precision=C128, pdims=None, hbm_budget=0):
        self.edges = [tuple(map(int, e)) for e in edges]
        e = _edges_arr(edges)
        self.sites = GetSiteIndexFromBond(self.edges)
        pd = None if pdims is None else _p(np.ascontiguousarray(pdims, np.int32), _i32p)
        h = _vp()
        _chk(lib.tnbp_job_create(_p(e, _i32p), len(e), pd, precision, None, int(hbm_budget), C.byref(h)))
        self.h = h
        self.precision = precision
        self._tpos = []

    def close(self):
        if getattr(self, "h", None):
            for t in self._tpos:
                lib.tnbp_tpo_destroy(t)
            self._tpos = []
            lib.tnbp_job_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def ne(self):
        return len(self.edges)

    def bond_dims(self):
        out = np.zeros(self.ne, np.int32)
        _chk(lib.tnbp_bond_dims(self.h, _p(out, _i32p)))
        return out

    def device_bytes(self):
        b = C.c_uint64()
        _chk(lib.tnbp_job_device_bytes(self.h, C.byref(b)))
        return b.value

    def site_shape(self, si):
        sh = np.zeros(16, np.int32)
        r = C.c_int32()
        _chk(lib.tnbp_site_shape(self.h, si, _p(sh, _i32p), 16, C.byref(r)))
        return tuple(int(x) for x in sh[: r.value])

    def get_site(self, si):
        sh = self.site_shape(si)
        n = int(np.prod(sh))
        out = np.zeros(n, np.complex128)
        _chk(lib.tnbp_download_site(self.h, si, _p(out.view(np.float64), _f64p), n))
        return out.reshape(sh, order="F")

    def set_site(self, si, a):
        a = _c128(a)
        sh = np.ascontiguousarray(a.shape, np.int32)
        flat = np.ascontiguousarray(a.reshape(-1, order="F"))
        _chk(lib.tnbp_upload_site(self.h, si, _p(sh, _i32p), a.ndim, _p(flat.view(np.float64), _f64p)))

    def get_message(self, m):
        d = C.c_int32()
        _chk(lib.tnbp_download_message(self.h, m, None, 0, C.byref(d)))
        out = np.zeros(d.value * d.value, np.complex128)
        _chk(lib.tnbp_download_message(self.h, m, _p(out.view(np.float64), _f64p), out.size, C.byref(d)))
        return out.reshape((d.value, d.value), order="F")

    def set_message(self, m, a):
        a = _c128(a)
        flat = np.ascontiguousarray(a.reshape(-1, order="F"))
        _chk(lib.tnbp_upload_message(self.h, m, a.shape[0], _p(flat.view(np.float64), _f64p)))

    def get_V(self):
        return [self.get_site(i) for i in range(len(self.sites))]

    def get_E(self):
        return [self.get_message(m) for m in range(2 * self.ne)]

    def set_state(self, V, E):
        """Upload a full state (messages first: they fix the bond dims)."""
        for m, a in enumerate(E):
            self.set_message(m, a)
        for i, v in enumerate(V):
            self.set_site(i, v)

    def tpo(self, layer):
        t = _vp()
        _chk(lib.tnbp_tpo_create(self.h, _p(layer.edge_rank, _i32p), _p(layer.op_offset, _i64p),
                                 _p(layer.op_data.view(np.float64), _f64p), C.byref(t)))
        self._tpos.append(t)
        return t

    def save(self, path):
        """SaveTPS of the device state (tnbp_save_state)."""
        _chk(lib.tnbp_save_state(self.h, os.fsencode(path)))

    def load(self, path):
        """LoadTPS into this job (tnbp_load_state)."""
        _chk(lib.tnbp_load_state(self.h, os.fsencode(path)))

    def sweep_stats(self):
        ms, fl, by = C.c_double(), C.c_double(), C.c_double()
        _chk(lib.tnbp_sweep_stats(self.h, C.byref(ms), C.byref(fl), C.byref(by)))
        return ms.value, fl.value, by.value

    def sweep_totals(self):
        """(total ms, total algorithmic flops, total algorithmic bytes, sweeps)
        over every sweep whose condition was read (CUDA events on the job's
        stream)."""
        ms, fl, by, n = C.c_double(), C.c_double(), C.c_double(), C.c_int64()
        _chk(lib.tnbp_sweep_totals(self.h, C.byref(ms), C.byref(fl), C.byref(by), C.byref(n)))
        return ms.value, fl.value, by.value, n.value


def InitTensorProductState(edges, precision=C128, pdims=None, hbm_budget=0):
    """InitTensorProductState (init.h:18-95): returns the device State."""
    return State(edges, precision, pdims, hbm_budget)


def AbsorbTPO(state, layer):
    """AbsorbTPO (include/tnbp/ptns/function/apply.h:15-177)."""
    t = layer if isinstance(layer, _vp) else state.tpo(layer)
    _chk(lib.tnbp_absorb_tpo(state.h, t))


def BeliefPropagation(state):
    """BeliefPropagation over all layers + F -> E (bp.h:66-261)."""
    _chk(lib.tnbp_bp_sweep(state.h))


def BeliefPropagationCondition(state):
    """BeliefPropagationCondition (bp.h:266-355)."""
    r = C.c_double()
    _chk(lib.tnbp_bp_condition(state.h, C.byref(r)))
    return r.value


def BeliefPropagationLoop(state, tol, max_iter):
    """The apps' BP loop (apps/estimator/main.cc:131-157): (sweeps, last condition)."""
    it, c = C.c_int32(), C.c_double()
    _chk(lib.tnbp_bp_run(state.h, tol, max_iter, C.byref(it), C.byref(c)))
    return it.value, c.value


def Truncation(state, max_dim, sv_min):
    """Truncation (include/tnbp/ptns/function/truncation.h:18-222):
    returns (res_bond_dim, res_trunc_err) per edge."""
    d = np.zeros(state.ne, np.int32)
    e = np.zeros(state.ne, np.float64)
    _chk(lib.tnbp_truncate(state.h, max_dim, sv_min, _p(d, _i32p), _p(e, _f64p)))
    return d, e


def Measure(state, where, ops):
    """Measure (include/tnbp/ptns/function/measure.h): `where` is a list of
    site labels (one-site ops O[p, p']) or of label pairs (two-site ops
    O[p_a, p_b, p_a', p_b'])."""
    if len(where) == 0:
        return np.zeros(0, np.complex128)
    out = np.zeros(len(where), np.complex128)
    if np.ndim(where[0]) == 0:
        pos = {s: i for i, s in enumerate(state.sites)}
        sites = np.ascontiguousarray([pos[int(s)] for s in where], np.int64)
        o = np.ascontiguousarray(np.stack([_c128(x).reshape(-1, order="F") for x in ops]))
        _chk(lib.tnbp_measure_1site(state.h, len(where), _p(sites, _i64p), _p(o.view(np.float64), _f64p),
                                    _p(out.view(np.float64), _f64p)))
    else:
        pr = np.ascontiguousarray(np.asarray(where, np.int32).reshape(-1, 2))
        o = np.ascontiguousarray(np.stack([_c128(x).reshape(-1, order="F") for x in ops]))
        _chk(lib.tnbp_measure_2site(state.h, len(where), _p(pr, _i32p), _p(o.view(np.float64), _f64p),
                                    _p(out.view(np.float64), _f64p)))
    return out


def MeasureCluster(state, terms, coeffs=None):
    """Pauli products on any distinct qubits, each measured on its tree
    cluster (tnbp_measure_cluster).  terms: list of (qubits, letters);
    returns (values per term, sum_k c_k <P_k>)."""
    n = len(terms)
    if n == 0:
        return np.zeros(0, np.complex128), 0j
    nq = np.array([len(q) for q, _ in terms], np.int32)
    qs = np.ascontiguousarray(np.concatenate([np.asarray(q, np.int32) for q, _ in terms]))
    letters = "".join(l for _, l in terms).encode()
    co = np.ones(n, np.complex128) if coeffs is None else np.ascontiguousarray(coeffs, np.complex128)
    vals = np.zeros(n, np.complex128)
    tot = np.zeros(1, np.complex128)
    _chk(lib.tnbp_measure_cluster(state.h, n, _p(nq, _i32p), _p(qs, _i32p), letters, _p(co.view(np.float64), _f64p),
                                  _p(vals.view(np.float64), _f64p), _p(tot.view(np.float64), _f64p)))
    return vals, complex(tot[0])


def MeasurePauliText(state, text, clusters=True):
    """Every row of a sparse-Pauli text (tnbp_measure_pauli_text): returns
    (sum, values per row, kinds per row)."""
    n = C.c_int64()
    s = text.encode()
    _chk(lib.tnbp_measure_pauli_text(state.h, s, 1 if clusters else 0, None, None, 0, C.byref(n), None))
    vals = np.zeros(max(1, n.value), np.complex128)
    kinds = np.zeros(max(1, n.value), np.int32)
    tot = np.zeros(1, np.complex128)
    _chk(lib.tnbp_measure_pauli_text(state.h, s, 1 if clusters else 0, _p(vals.view(np.float64), _f64p),
                                     _p(kinds, _i32p), n.value, C.byref(n), _p(tot.view(np.float64), _f64p)))
    return complex(tot[0]), vals[: n.value], kinds[: n.value]


class Server:
    """Continuous-batching request loop (tnbp_server_*)."""

    def __init__(self, precision=C64, hbm_budget=0, max_active=64):
        h = _vp()
        _chk(lib.tnbp_server_create(precision, int(hbm_budget), max_active, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.tnbp_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_kicked_ising(self, L, chi, steps, theta_j, theta_h, terms, bp_tol=1e-8, bp_max_iter=50,
                            sv_min=1e-8):
        rid = C.c_int64()
        n = len(terms)
        co = np.ascontiguousarray(terms.coeff, np.complex128) if n else np.zeros(1, np.complex128)
        kind = np.ascontiguousarray(terms.kind, np.int32) if n else np.zeros(1, np.int32)
        q0 = np.ascontiguousarray(terms.q0, np.int32) if n else np.zeros(1, np.int32)
        q1 = np.ascontiguousarray(terms.q1, np.int32) if n else np.zeros(1, np.int32)
        _chk(lib.tnbp_server_submit_kicked_ising(self.h, L, chi, steps, theta_j, theta_h, bp_tol, bp_max_iter, sv_min,
                                                 n, _p(kind, _i32p), _p(q0, _i32p), _p(q1, _i32p),
                                                 terms.letters if n else b"II", _p(co.view(np.float64), _f64p),
                                                 C.byref(rid)))
        return rid.value

    def submit_qasm(self, qasm_src, pauli_text, chi, bp_tol=1e-8, bp_max_iter=50, sv_min=1e-8, do_opt_tpo=False,
                    eps_opt_tpo=1e-8):
        """The estimator app's workload as a served request: returns its id."""
        rid = C.c_int64()
        _chk(lib.tnbp_server_submit_qasm(self.h, qasm_src.encode(), pauli_text.encode(), chi, bp_tol, bp_max_iter,
                                         sv_min, 1 if do_opt_tpo else 0, eps_opt_tpo, C.byref(rid)))
        return rid.value

    def tpo_cache_stats(self):
        """(hits, misses, entries) of the server's TPO cache."""
        h, m, e = C.c_int64(), C.c_int64(), C.c_int64()
        _chk(lib.tnbp_server_tpo_cache_stats(self.h, C.byref(h), C.byref(m), C.byref(e)))
        return h.value, m.value, e.value

    def cancel(self, rid):
        """Cancel a request that has not finished (tnbp_server_cancel)."""
        _chk(lib.tnbp_server_cancel(self.h, rid))

    def step(self):
        a, q, d = C.c_int32(), C.c_int32(), C.c_int32()
        _chk(lib.tnbp_server_step(self.h, C.byref(a), C.byref(q), C.byref(d)))
        return a.value, q.value, d.value

    def set_escalation(self, on=True):
        """Restart, in complex128, requests whose BP loop does not converge
        (tnbp_server_set_escalation; reduced-precision servers only)."""
        _chk(lib.tnbp_server_set_escalation(self.h, 1 if on else 0))

    def set_escalation_threshold(self, min_cond):
        """Escalate only loops whose condition never fell below min_cond
        (tnbp_server_set_escalation_threshold; 0 = every non-converging loop)."""
        _chk(lib.tnbp_server_set_escalation_threshold(self.h, float(min_cond)))

    def info(self, rid):
        """{'precision', 'escalated', 'bp_converged', 'unconverged_loops',
        'worst_final_cond', 'worst_min_cond'} of a request
        (tnbp_server_request_info, tnbp_server_request_bp_stats)."""
        p, e, c = C.c_int32(), C.c_int32(), C.c_int32()
        _chk(lib.tnbp_server_request_info(self.h, rid, C.byref(p), C.byref(e), C.byref(c)))
        n, wf, wm = C.c_int32(), C.c_double(), C.c_double()
        _chk(lib.tnbp_server_request_bp_stats(self.h, rid, C.byref(n), C.byref(wf), C.byref(wm)))
        return {"precision": p.value, "escalated": bool(e.value), "bp_converged": bool(c.value),
                "unconverged_loops": n.value, "worst_final_cond": wf.value, "worst_min_cond": wm.value}

    def result(self, rid):
        out = np.zeros(2, np.float64)
        pend = C.c_int32()
        _chk(lib.tnbp_server_result(self.h, rid, _p(out, _f64p), C.byref(pend)))
        return None if pend.value else complex(out[0], out[1])


def MeasurePauliSum(state, terms):
    """Sum_k c_k <P_k> (FP64 on the device) and the per-term values."""
    n = len(terms)
    per = np.zeros(max(n, 1), np.complex128)
    tot = np.zeros(1, np.complex128)
    if n == 0:
        return 0j, per[:0]
    co = np.ascontiguousarray(terms.coeff, np.complex128)
    _chk(lib.tnbp_measure_pauli_sum(state.h, n, _p(np.ascontiguousarray(terms.kind, np.int32), _i32p),
                                    _p(np.ascontiguousarray(terms.q0, np.int32), _i32p),
                                    _p(np.ascontiguousarray(terms.q1, np.int32), _i32p), terms.letters,
                                    _p(co.view(np.float64), _f64p), _p(per.view(np.float64), _f64p),
                                    _p(tot.view(np.float64), _f64p)))
    return complex(tot[0]), per[:n]
