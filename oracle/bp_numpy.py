"""CPU restatement (numpy, FP64) of tnbp's loopy-BP PEPS estimator path.

TEST INFRASTRUCTURE ONLY.  This module is the oracle the B200 engine is
checked against; only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may import it.  It is pinned to the reference itself through the
golden fixtures of tests/golden/ (made by tests/golden/make_golden.py from the
reference's own headers compiled in oracle/_ref/).

Conventions (restated from the reference, r-ccs-cms/tnbp):
  * sites = sorted distinct labels of the edge list
    (include/tnbp/framework/graph.h:23-35);
  * leg k of a site = k-th edge in edge order containing it
    (graph.h:40-55); the physical leg is last;
  * a site tensor is an ndarray of shape (D_0, ..., D_{g-1}, d); merged
    indices use the column-major rule (a, b) -> a + dim(a) * b;
  * E[m] (m < ne) is the message computed at edges[m][0], E[m + ne] the one
    computed at edges[m][1] (include/tnbp/ptns/function/bp.h:170-174).
"""
import numpy as np


# ------------------------------------------------------------------ graph
def sites_of(edges):
    """GetSiteIndexFromBond (graph.h:23-35)."""
    return sorted({v for e in edges for v in e})


def bonds_of(edges, site):
    """GetSurroundingBondIndex (graph.h:40-55)."""
    out = []
    for m, (i, j) in enumerate(edges):
        if i == site:
            out.append(m)
        if j == site:
            out.append(m)
    return out


def in_msg(edges, site, m):
    """Message absorbed by `site` along edge m (bp.h:147-151)."""
    return m + len(edges) if edges[m][0] == site else m


def out_msg(edges, site, m):
    """Message computed at `site` along edge m (bp.h:170-174)."""
    return m if edges[m][0] == site else m + len(edges)


def normalize(t):
    n = np.linalg.norm(t)
    return (t / n if n > 0 else t), n


# ---------------------------------------------------------------- init
def init_state(edges, pdim=2):
    """InitTensorProductState (include/tnbp/ptns/function/init.h:18-95)."""
    sites = sites_of(edges)
    V = []
    for s in sites:
        g = len(bonds_of(edges, s))
        v = np.zeros((1,) * g + (pdim,), dtype=np.complex128)
        v[(0,) * (g + 1)] = 1.0
        V.append(v)
    E = [np.ones((1, 1), dtype=np.complex128) for _ in range(2 * len(edges))]
    return V, E


# --------------------------------------------------------------- absorb
def absorb_tpo(edges, V, E, O):
    """AbsorbTPO (include/tnbp/ptns/function/apply.h:15-177).
    O[s] has shape (r_0, ..., r_{g-1}, d_in, d_out).
    V'[(v_k, o_k)..., p'] = sum_p O[o..., p, p'] V[v..., p], merged v + D o;
    E' = E (x) I_r with merged (e, i) -> e + D i."""
    sites = sites_of(edges)
    nV = []
    for si, s in enumerate(sites):
        v, o = V[si], O[si]
        g = v.ndim - 1
        # w[v0..v_{g-1}, o0..o_{g-1}, p'] = sum_p v[v.., p] o[o.., p, p']
        w = np.tensordot(v, o, axes=([g], [g]))
        perm = []
        for k in range(g):
            perm += [k, g + k]
        perm.append(2 * g)
        w = np.transpose(w, perm)
        shape = [v.shape[k] * o.shape[k] for k in range(g)] + [o.shape[g + 1]]
        nV.append(np.reshape(w, shape, order="F"))
    ne = len(edges)
    nE = []
    rank = [None] * ne
    for si, s in enumerate(sites):
        for k, m in enumerate(bonds_of(edges, s)):
            rank[m] = O[si].shape[k]
    for m in range(2 * ne):
        r = rank[m % ne]
        e = E[m]
        t = np.einsum("ab,ij->aibj", e, np.eye(r))
        D = e.shape[0]
        nE.append(np.reshape(t, (D * r, D * r), order="F"))
    return nV, nE


def opt_tpo_svd(edges, O, eps):
    """OptTPObySVD (include/tnbp/ptns/function/optsvdtpo.h:86-214), step by
    step: for each edge m = (a, b) in edge order, C = O_a contracted with
    O_b over the bond (remaining legs of O_a, then of O_b, 162-164), an SVD
    of C with O_a's legs as rows (173-174; kept: s > eps, at most the bond
    dimension, at least one -- the TruncSVD rule), sqrt(s) to both sides
    (175-181), O_a = U sqrt(s) with the new bond at its old leg position
    (182-197), O_b = sqrt(s) V with the same (198-212).  O is a list of site
    operators (r_0, ..., r_{g-1}, d_in, d_out); a new list is returned."""
    sites = sites_of(edges)
    pos = {s: i for i, s in enumerate(sites)}
    O = [np.array(o, dtype=np.complex128) for o in O]
    for m, (a, b) in enumerate(edges):
        ia, ib = pos[a], pos[b]
        pa = bonds_of(edges, a).index(m)
        pb = bonds_of(edges, b).index(m)
        A, B = O[ia], O[ib]
        r = A.shape[pa]
        C = np.tensordot(A, B, axes=([pa], [pb]))
        rows = [A.shape[k] for k in range(A.ndim) if k != pa]
        cols = [B.shape[k] for k in range(B.ndim) if k != pb]
        M = C.reshape(int(np.prod(rows)), int(np.prod(cols)), order="F")
        U, s, Vh = np.linalg.svd(M, full_matrices=False)
        keep = 0
        while keep < len(s) and keep < r and s[keep] > eps:
            keep += 1
        keep = max(keep, 1)
        sq = np.sqrt(s[:keep])
        Ua = (U[:, :keep] * sq[None, :]).reshape(rows + [keep], order="F")
        Vb = (sq[:, None] * Vh[:keep, :]).reshape([keep] + cols, order="F")
        O[ia] = np.moveaxis(Ua, -1, pa)
        O[ib] = np.moveaxis(Vb, 0, pb)
    return O


# ------------------------------------------------------------------- BP
def _absorb_leg(t, leg, M):
    """T_new[..., k', ...] = sum_j T[..., j, ...] M[j, k'] (bp.h:137-152)."""
    r = np.tensordot(t, M, axes=([leg], [0]))
    return np.moveaxis(r, -1, leg)


def message(edges, V, E, si, site, t):
    """Message computed at `site` along its leg t (bp.h:128-175): absorb the
    incoming messages on every other leg (normalizing after each leg, as the
    reference does), then contract with conj(V) over all legs but t."""
    bonds = bonds_of(edges, site)
    T = V[si].copy()
    for k, m in enumerate(bonds):
        if k != t:
            T = _absorb_leg(T, k, E[in_msg(edges, site, m)])
        T, _ = normalize(T)
    axes = [a for a in range(T.ndim) if a != t]
    N = np.tensordot(T, V[si].conj(), axes=(axes, axes))
    N, _ = normalize(N)
    return N


def bp_sweep(edges, V, E):
    """BeliefPropagation over all layers (bp.h:66-261) plus the app's F -> E
    copy: every directed message recomputed from the old E (Jacobi)."""
    sites = sites_of(edges)
    F = [None] * (2 * len(edges))
    for si, s in enumerate(sites):
        for t, m in enumerate(bonds_of(edges, s)):
            F[out_msg(edges, s, m)] = message(edges, V, E, si, s, t)
    return F


def bp_condition(edges, V, E):
    """BeliefPropagationCondition (bp.h:266-355)."""
    sites = sites_of(edges)
    acc = 0.0
    for si, s in enumerate(sites):
        for t, m in enumerate(bonds_of(edges, s)):
            N = message(edges, V, E, si, s, t)
            St, _ = normalize(E[out_msg(edges, s, m)])
            acc += np.linalg.norm(N - St)
    return acc / (2.0 * len(edges))


def bp_run(edges, V, E, tol, max_iter):
    """The apps' BP loop (apps/estimator/main.cc:131-157)."""
    conds = []
    for _ in range(max_iter):
        E = bp_sweep(edges, V, E)
        c = bp_condition(edges, V, E)
        conds.append(c)
        if c < tol:
            break
    return E, conds


# ------------------------------------------------------------ truncation
def sqrt_and_inverse(M, sv_min):
    """SquareRootAndInverse (include/tnbp/framework/root.h:66-148):
    M = U s Vh; R = U sqrt(s) Vh (sqrt(s) := 0 where s <= sv_min);
    S = Vh^H (1/sqrt(s)) U^H (1/sqrt(s) := 0 where sqrt(s) <= sqrt(sv_min))."""
    U, s, Vh = np.linalg.svd(M)
    sq = np.where(np.abs(s) > sv_min, np.sqrt(np.abs(s)), 0.0)
    inv = np.where(np.abs(sq) > np.sqrt(sv_min), 1.0 / np.where(sq > 0, sq, 1.0), 0.0)
    R = (U * sq) @ Vh
    S = (Vh.conj().T * inv) @ U.conj().T
    return R, S


def trunc_svd(T, chi_max, s_min):
    """Truncated SVD with the rule documented for the engine: keep
    s_i > s_min, at most chi_max, at least one; err = cut s^2 / all s^2."""
    X, s, Y = np.linalg.svd(T)
    keep = 0
    while keep < len(s) and keep < chi_max and s[keep] > s_min:
        keep += 1
    keep = max(keep, 1)
    tot = float(np.sum(s ** 2))
    err = float(np.sum(s[keep:] ** 2)) / tot if tot > 0 else 0.0
    return X[:, :keep], s[:keep], Y[:keep, :], err


def truncate(edges, V, E, chi_max, sv_min):
    """Truncation (include/tnbp/ptns/function/truncation.h:18-222)."""
    sites = sites_of(edges)
    pos = {s: i for i, s in enumerate(sites)}
    ne = len(edges)
    V = [v.copy() for v in V]
    E = list(E)
    dims, errs = [0] * ne, [0.0] * ne
    for m, (a, b) in enumerate(edges):
        Ra, Sa = sqrt_and_inverse(E[m], sv_min)
        Rb, Sb = sqrt_and_inverse(E[m + ne], sv_min)
        T = Ra.T @ Rb
        T, _ = normalize(T)
        X, s, Y, err = trunc_svd(T, chi_max, sv_min)
        dims[m], errs[m] = len(s), err
        Z = np.diag(s).astype(np.complex128)
        E[m] = Z.copy()
        E[m + ne] = Z.copy()
        P = np.sqrt(s)
        Ta = (Sa.T @ X) * P
        Tb = (P[:, None] * Y) @ Sb
        ka = bonds_of(edges, a).index(m)
        kb = bonds_of(edges, b).index(m)
        va = _absorb_leg(V[pos[a]], ka, Ta)
        V[pos[a]], _ = normalize(va)
        vb = _absorb_leg(V[pos[b]], kb, Tb.T)
        V[pos[b]], _ = normalize(vb)
    return V, E, dims, errs


# ------------------------------------------------------------ measurement
def measure_1site(edges, V, E, site, O):
    """Measure, one site (include/tnbp/ptns/function/measure.h:15-94).
    O[p, p'] in the reference layout (operator applied as sum_p W[..p] O[p, p'])."""
    sites = sites_of(edges)
    si = sites.index(site)
    W = V[si].copy()
    for k, m in enumerate(bonds_of(edges, site)):
        W = _absorb_leg(W, k, E[in_msg(edges, site, m)])
    g = W.ndim - 1
    R = np.tensordot(W, O, axes=([g], [0]))
    return np.vdot(V[si], R) / np.vdot(V[si], W)


def _env(edges, V, E, site, target):
    """AdagA[p, p', t, t'] of measure.h:168-205."""
    sites = sites_of(edges)
    si = sites.index(site)
    A = V[si].copy()
    for k, m in enumerate(bonds_of(edges, site)):
        if k != target:
            A = _absorb_leg(A, k, E[in_msg(edges, site, m)])
            A, _ = normalize(A)
    g = A.ndim - 1
    axes = [a for a in range(g) if a != target]
    env = np.tensordot(A, V[si].conj(), axes=(axes, axes))  # (t, p, t', p')
    return np.transpose(env, (1, 3, 0, 2))


def measure_2site(edges, V, E, pair, O):
    """Measure, nearest-neighbour pair (measure.h:100-300).
    O[p_a, p_b, p_a', p_b'] (reference layout, contracted as in 256-289)."""
    a, b = pair
    m = [i for i, e in enumerate(edges) if e == (a, b) or e == (b, a)][0]
    ta = bonds_of(edges, a).index(m)
    tb = bonds_of(edges, b).index(m)
    AA = _env(edges, V, E, a, ta)
    BB = _env(edges, V, E, b, tb)
    num = np.einsum("xytu,xcyd,cdtu->", AA, O, BB)
    den = np.einsum("xxtu,cctu->", AA, BB)
    return num / den


def shortest_path(edges, src, dst):
    """FindShortestPath (include/tnbp/framework/graph.h:57-108): BFS from src,
    neighbours in edge-list order, stopping when dst is dequeued."""
    adj = {s: [] for s in sites_of(edges)}
    for a, b in edges:
        adj[a].append(b)
        adj[b].append(a)
    if src not in adj or dst not in adj:
        return []
    prev = {src: None}
    queue = [src]
    head = 0
    while head < len(queue):
        u = queue[head]
        head += 1
        if u == dst:
            break
        for v in adj[u]:
            if v not in prev:
                prev[v] = u
                queue.append(v)
    if dst not in prev:
        return []
    path = [dst]
    while prev[path[-1]] is not None:
        path.append(prev[path[-1]])
    return path[::-1]


def cluster_tree(edges, qubits):
    """The tree cluster of a Pauli product on `qubits`: the union of the
    shortest paths from the lowest-numbered qubit to each other qubit, as
    {site: parent} (the root's parent is None)."""
    qubits = sorted(qubits)
    parent = {qubits[0]: None}
    for q in qubits[1:]:
        path = shortest_path(edges, qubits[0], q)
        for u, v in zip(path, path[1:]):
            assert parent.get(v, u) == u, "paths from the first qubit do not form a tree"
            parent[v] = u
    return parent


def measure_cluster(edges, V, E, qubits, letters):
    """A Pauli product on distinct qubits measured on its tree cluster (the
    terms ClassifyOps drops; not in the reference).  The ket and bra layers of
    the tree's sites, the Pauli letters on the qubit sites (identity
    elsewhere) and the BP messages on every leg leaving the tree are
    contracted exactly: Z(P) / Z(identity).  Each site is first reduced to a
    tensor over its tree legs (ket legs, then bra legs), then the tree is one
    einsum."""
    sites = sites_of(edges)
    parent = cluster_tree(edges, list(qubits))
    tree_edges = set()
    for v, u in parent.items():
        if u is not None:
            tree_edges.add([m for m, e in enumerate(edges) if e in ((u, v), (v, u))][0])
    opmap = dict(zip(qubits, letters))
    te = sorted(tree_edges)
    letter_of = {m: (2 * i, 2 * i + 1) for i, m in enumerate(te)}  # (ket, bra) einsum ids

    def z(with_ops):
        args = []
        for s in parent:
            v = V[sites.index(s)]
            g = v.ndim - 1
            bonds = bonds_of(edges, s)
            W = v.copy()
            for k, m in enumerate(bonds):
                if m not in tree_edges:
                    W = _absorb_leg(W, k, E[in_msg(edges, s, m)])
            O = pauli_op(opmap[s]) if (with_ops and s in opmap) else np.eye(2, dtype=np.complex128)
            W = np.tensordot(W, O, axes=([g], [0]))
            closed = [k for k, m in enumerate(bonds) if m not in tree_edges] + [g]
            T = np.tensordot(W, v.conj(), axes=(closed, closed))
            open_m = [m for m in bonds if m in tree_edges]
            args += [T, [letter_of[m][0] for m in open_m] + [letter_of[m][1] for m in open_m]]
        return np.einsum(*args, [])

    return z(True) / z(False)


# --------------------------------------------------------------- Pauli
PAULI = {
    "I": [1, 0, 0, 1],
    "X": [0, 1, 1, 0],
    "Y": [0, -1j, 1j, 0],
    "Z": [1, 0, 0, -1],
}


def pauli_op(letter):
    """PauliOpMatrix (include/tnbp/parser/paulitotpo.h:21-35) in the
    reference's tensor layout O[c0, c1] = list[c0 + 2 c1]."""
    return np.reshape(np.array(PAULI[letter], dtype=np.complex128), (2, 2), order="F")


def pauli_two(la, lb):
    """SparsePauliToTensorOp for two letters: O[i0, i1, i2, i3] = Pa[i0, i2] Pb[i1, i3]."""
    return np.einsum("ac,bd->abcd", pauli_op(la), pauli_op(lb))


def parse_pauli_text(text, edges):
    """load_sparse_pauli_op (include/pauli/sparse_pauli.h:52-97) followed by
    ClassifyOps (paulitotpo.h:99-153): kept terms as
    (kind, qubits, letters, coeff); dropped count."""
    kept, dropped = [], 0
    eset = {tuple(e) for e in edges} | {(b, a) for a, b in edges}
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("#") or line.startswith("//"):
            continue
        tok = line.split()
        try:
            re_, im_ = float(tok[0]), float(tok[1])
            ps = tok[2]
        except (ValueError, IndexError):
            re_, im_, ps = float(tok[0]), 0.0, tok[1]
        ps = ps.strip().upper()
        if any(c not in "IXYZ" for c in ps):
            raise ValueError("Invalid Pauli label: only I/X/Y/Z are allowed.")
        n = len(ps)
        ops = [(i, ps[n - 1 - i]) for i in range(n) if ps[n - 1 - i] != "I"]
        if len(ops) == 1:
            kept.append((1, (ops[0][0],), (ops[0][1],), complex(re_, im_)))
        elif len(ops) == 2 and (ops[0][0], ops[1][0]) in eset:
            kept.append((2, (ops[0][0], ops[1][0]), (ops[0][1], ops[1][1]), complex(re_, im_)))
        else:
            dropped += 1
    return kept, dropped


def pauli_sum(edges, V, E, terms):
    """Sum_k c_k <P_k> in FP64 over kept terms; also the per-term values."""
    vals = []
    for kind, qs, ls, c in terms:
        if kind == 1:
            vals.append(measure_1site(edges, V, E, qs[0], pauli_op(ls[0])))
        else:
            vals.append(measure_2site(edges, V, E, qs, pauli_two(ls[0], ls[1])))
    total = sum(t[3] * v for t, v in zip(terms, vals))
    return total, vals


# ------------------------------------------------------------ estimator
def run_estimator(edges, tpo_layers, chi, sv_min, tol, max_iter, V=None, E=None):
    """apps/estimator/main.cc:105-178 on given TPO layers."""
    if V is None:
        V, E = init_state(edges)
    log = []
    for O in tpo_layers:
        V, E = absorb_tpo(edges, V, E, O)
        E, conds = bp_run(edges, V, E, tol, max_iter)
        V, E, dims, errs = truncate(edges, V, E, chi, sv_min)
        log.append(dict(conds=conds, dims=dims, errs=errs))
    return V, E, log


# ------------------------------------------------------------- statevector
def statevector_expect(n, layers_ops, terms):
    """Exact <P> after applying gate lists (KAT for trees/small systems).
    layers_ops: list of (matrix U[out, in] in little-endian qubit order, qubits)."""
    psi = np.zeros(2 ** n, dtype=np.complex128)
    psi[0] = 1.0
    for U, qs in layers_ops:
        k = len(qs)
        t = psi.reshape([2] * n, order="F")
        Ut = U.reshape([2] * (2 * k), order="F")  # U[(out bits), (in bits)] little-endian
        t = np.tensordot(Ut, t, axes=(list(range(k, 2 * k)), list(qs)))
        t = np.moveaxis(t, list(range(k)), list(qs))
        psi = t.reshape(-1, order="F")
    out = []
    for kind, qs, ls, c in terms:
        phi = psi.reshape([2] * n, order="F")
        for q, l in zip(qs, ls):
            P = np.array(PAULI[l], dtype=np.complex128).reshape(2, 2)  # row-major P[out][in]
            phi = np.moveaxis(np.tensordot(P, phi, axes=([1], [q])), 0, q)
        out.append(np.vdot(psi, phi.reshape(-1, order="F")))
    return out
