// Host-side problem builders of the estimator path, written for this
// engine: lattice and edge bookkeeping, OpenQASM 2 / 3-subset parsing,
// sparse-Pauli parsing and classification, and TPO (tensor-product
// operator) construction.  Their outputs (edge order, leg order, layer
// split, gate order, Pauli qubit order, kept terms) are required to be
// identical to the reference's; numeric TPO factors may differ by a gauge
// on the operator bonds (a different but equally valid SVD), which leaves
// every observable unchanged.
#include "host_setup.h"

#include <algorithm>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdint>
#include <complex>
#include <cstdlib>
#include <map>
#include <numeric>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace tnbp_host {

using cd = std::complex<double>;

// ------------------------------------------------------------- lattice
// bond_square_lattice (include/tnbp/lattice/square.h:14-34): row-major sites
// ix + Lx*iy, per site the right neighbour then the one below.
Edges square_lattice(int Lx, int Ly) {
  if (Lx < 1 || Ly < 1) throw HostError(-1, "lattice sides must be >= 1");
  Edges out;
  for (int iy = 0; iy < Ly; ++iy)
    for (int ix = 0; ix < Lx; ++ix) {
      const int s = ix + Lx * iy;
      if (ix + 1 < Lx) out.push_back({s, s + 1});
      if (iy + 1 < Ly) out.push_back({s, s + Lx});
    }
  return out;
}

// GreedyEdgeLayering (graph.h:138-170): repeated first-fit matchings in edge order.
std::vector<int> greedy_layering(const Edges& e, int* nlayers) {
  std::vector<int> layer(e.size(), -1);
  int l = 0;
  size_t left = e.size();
  while (left > 0) {
    std::unordered_set<int> used;
    for (size_t i = 0; i < e.size(); ++i) {
      if (layer[i] >= 0) continue;
      if (used.count(e[i].first) || used.count(e[i].second)) continue;
      layer[i] = l;
      used.insert(e[i].first);
      used.insert(e[i].second);
      --left;
    }
    ++l;
  }
  *nlayers = l;
  return layer;
}

std::vector<int> surrounding_bonds(const Edges& e, int site) {
  std::vector<int> r;
  for (size_t m = 0; m < e.size(); ++m) {
    if (e[m].first == site) r.push_back((int)m);
    if (e[m].second == site) r.push_back((int)m);
  }
  return r;
}

std::vector<int> site_labels(const Edges& e) {
  std::vector<int> s;
  for (auto& p : e) { s.push_back(p.first); s.push_back(p.second); }
  std::sort(s.begin(), s.end());
  s.erase(std::unique(s.begin(), s.end()), s.end());
  return s;
}

// FindShortestPath (graph.h:57-108): BFS over compressed labels, neighbours
// visited in edge-list insertion order; empty if unreachable.
std::vector<int> shortest_path(const Edges& e, int src, int dst) {
  const auto sites = site_labels(e);
  std::unordered_map<int, size_t> idx;
  for (size_t i = 0; i < sites.size(); ++i) idx[sites[i]] = i;
  if (!idx.count(src) || !idx.count(dst)) return {};
  std::vector<std::vector<size_t>> adj(sites.size());
  for (auto& p : e) { adj[idx[p.first]].push_back(idx[p.second]); adj[idx[p.second]].push_back(idx[p.first]); }
  const size_t s = idx[src], t = idx[dst];
  std::vector<char> seen(sites.size(), 0);
  std::vector<size_t> prev(sites.size(), (size_t)-1);
  std::queue<size_t> q;
  q.push(s);
  seen[s] = 1;
  while (!q.empty()) {
    const size_t u = q.front();
    q.pop();
    if (u == t) break;
    for (size_t v : adj[u])
      if (!seen[v]) { seen[v] = 1; prev[v] = u; q.push(v); }
  }
  if (!seen[t]) return {};
  std::vector<int> path;
  for (size_t c = t; c != (size_t)-1; c = prev[c]) path.push_back(sites[c]);
  std::reverse(path.begin(), path.end());
  return path;
}

// QASM text: qasm_text.cpp (tokenizer and statement reader).

int qubit_count(const Instruction& in) {
  switch (in.op) {
    case Op::MEASURE: case Op::RESET: return 1;
    case Op::BARRIER: case Op::CUSTOM: return (int)in.qubits.size();
    default: return op_arity(in.op);
  }
}

// EdgesFromQasm (qasmtoedge.h:38-56)
Edges qasm_edges(const Program& p) {
  Edges e;
  for (auto& in : p.instructions) {
    if (qubit_count(in) != 2) continue;
    int a = (int)in.qubits[0].index, b = (int)in.qubits[1].index;
    e.push_back(a < b ? std::make_pair(a, b) : std::make_pair(b, a));
  }
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  return e;
}

// ------------------------------------------------------------ gate matrices
// U[out][in] in the qubit order of the instruction, state index
// q0 + 2 q1 (+ 4 q2) (little-endian, as qasmtotpo.h:19-144 encodes them).
static std::vector<cd> gate_matrix(const Instruction& in) {
  const double pi = 3.14159265358979323846;
  auto P = [&](size_t k) { return in.params.size() > k ? in.params[k] : 0.0; };
  const cd I(0, 1);
  switch (in.op) {
    case Op::U3: {
      const double th = P(0), ph = P(1), la = P(2);
      return {std::cos(th / 2), -std::exp(I * la) * std::sin(th / 2), std::exp(I * ph) * std::sin(th / 2),
              std::exp(I * (ph + la)) * std::cos(th / 2)};
    }
    case Op::U2: {
      const double ph = P(0), la = P(1), s = 1 / std::sqrt(2.0);
      return {s, -std::exp(I * la) * s, std::exp(I * ph) * s, std::exp(I * (ph + la)) * s};
    }
    case Op::U1: return {1, 0, 0, std::exp(I * P(0))};
    case Op::RX: { const double t = P(0); return {std::cos(t / 2), -I * std::sin(t / 2), -I * std::sin(t / 2), std::cos(t / 2)}; }
    case Op::RY: { const double t = P(0); return {std::cos(t / 2), -std::sin(t / 2), std::sin(t / 2), std::cos(t / 2)}; }
    case Op::RZ: { const double t = P(0); return {std::exp(-I * (t / 2)), 0, 0, std::exp(I * (t / 2))}; }
    case Op::H: { const double s = 1 / std::sqrt(2.0); return {s, s, s, -s}; }
    case Op::X: return {0, 1, 1, 0};
    case Op::Y: return {0, -I, I, 0};
    case Op::Z: return {1, 0, 0, -1};
    case Op::S: return {1, 0, 0, I};
    case Op::SDG: return {1, 0, 0, -I};
    case Op::T: return {1, 0, 0, std::exp(I * (pi / 4))};
    case Op::TDG: return {1, 0, 0, std::exp(-I * (pi / 4))};
    case Op::ID: return {1, 0, 0, 1};
    case Op::CX: { std::vector<cd> m(16, 0.0); m[0] = 1; m[2 * 4 + 2] = 1; m[1 * 4 + 3] = 1; m[3 * 4 + 1] = 1; return m; }
    case Op::CZ: { std::vector<cd> m(16, 0.0); m[0] = 1; m[5] = 1; m[10] = 1; m[15] = -1; return m; }
    case Op::SWAP: { std::vector<cd> m(16, 0.0); m[0] = 1; m[1 * 4 + 2] = 1; m[2 * 4 + 1] = 1; m[15] = 1; return m; }
    case Op::RZZ: {
      const double t = P(0);
      std::vector<cd> m(16, 0.0);
      m[0] = std::exp(-I * (t / 2)); m[5] = std::exp(I * (t / 2)); m[10] = std::exp(I * (t / 2)); m[15] = std::exp(-I * (t / 2));
      return m;
    }
    case Op::CCX: {
      std::vector<cd> m(64, 0.0);
      for (int i = 0; i < 8; ++i) m[i * 8 + i] = 1;
      m[3 * 8 + 3] = 0; m[3 * 8 + 7] = 1; m[7 * 8 + 3] = 1; m[7 * 8 + 7] = 0;
      return m;
    }
    case Op::CSWAP: {
      // Fredkin, control q0: swaps q1 and q2 (|011> <-> |101>, indices 3 and
      // 5); the other six basis states stay.  The reference's table
      // (qasmtotpo.h:127-137) places the diagonal entry of index 4 at index
      // 5, which is not unitary; its three-qubit branch cannot run anyway
      // (it indexes past its path vector), so the correct gate is used here.
      std::vector<cd> m(64, 0.0);
      for (int i : {0, 1, 2, 4, 6, 7}) m[i * 8 + i] = 1;
      m[3 * 8 + 5] = 1;
      m[5 * 8 + 3] = 1;
      return m;
    }
    default:
      throw HostError(-6, "matrix for this op not implemented");
  }
}

// ------------------------------------------------------- small dense SVD
// One-sided Jacobi SVD of an m x n complex matrix (column-major), m >= n
// handled directly, m < n through the adjoint.  s descending.
static void small_svd(int m, int n, const std::vector<cd>& A, std::vector<cd>& U, std::vector<double>& s,
                      std::vector<cd>& Vh) {
  const bool tall = m >= n;
  const int M = tall ? m : n, N = tall ? n : m;
  std::vector<cd> W(M * N);
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < n; ++c) {
      if (tall) W[r + M * c] = A[r + m * c];
      else W[c + M * r] = std::conj(A[r + m * c]);
    }
  std::vector<cd> V(N * N, 0.0);
  for (int i = 0; i < N; ++i) V[i + N * i] = 1.0;
  double fro = 0;
  for (auto& x : W) fro += std::norm(x);
  const double eps = 2.220446049250313e-16, tol = eps * std::max(M, 8);
  for (int sweep = 0; sweep < 80; ++sweep) {
    bool rot = false;
    for (int i = 0; i < N - 1; ++i)
      for (int j = i + 1; j < N; ++j) {
        double al = 0, be = 0;
        cd ga = 0;
        for (int r = 0; r < M; ++r) {
          al += std::norm(W[r + M * i]);
          be += std::norm(W[r + M * j]);
          ga += std::conj(W[r + M * i]) * W[r + M * j];
        }
        const double g = std::abs(ga);
        // numerically-zero columns (rank-deficient gates) are not rotated
        if (!(g > 0) || g <= tol * std::sqrt(al * be) || std::min(al, be) <= tol * tol * fro) continue;
        const cd ph = ga / g;
        const double z = (be - al) / (2 * g);
        const double t = (z >= 0 ? 1.0 : -1.0) / (std::abs(z) + std::sqrt(1 + z * z));
        if (std::abs(t) < eps) continue;
        rot = true;
        const double c = 1 / std::sqrt(1 + t * t), sn = c * t;
        for (int r = 0; r < M; ++r) {
          const cd x = W[r + M * i], y = W[r + M * j];
          W[r + M * i] = c * x - sn * std::conj(ph) * y;
          W[r + M * j] = sn * ph * x + c * y;
        }
        for (int r = 0; r < N; ++r) {
          const cd x = V[r + N * i], y = V[r + N * j];
          V[r + N * i] = c * x - sn * std::conj(ph) * y;
          V[r + N * j] = sn * ph * x + c * y;
        }
      }
    if (!rot) break;
  }
  std::vector<double> sv(N);
  for (int j = 0; j < N; ++j) {
    double a = 0;
    for (int r = 0; r < M; ++r) a += std::norm(W[r + M * j]);
    sv[j] = std::sqrt(a);
  }
  std::vector<int> ord(N);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return sv[a] > sv[b]; });
  // worked matrix = L diag(s) R^H with L (M x N), R (N x N)
  std::vector<cd> L(M * N, 0.0), Rm(N * N);
  s.assign(N, 0.0);
  for (int k = 0; k < N; ++k) {
    const int j = ord[k];
    s[k] = sv[j];
    for (int r = 0; r < N; ++r) Rm[r + N * k] = V[r + N * j];
    if (sv[j] > 0)
      for (int r = 0; r < M; ++r) L[r + M * k] = W[r + M * j] / sv[j];
  }
  if (tall) {
    U = L;
    Vh.assign(N * n, 0.0);
    for (int k = 0; k < N; ++k)
      for (int c = 0; c < n; ++c) Vh[k + N * c] = std::conj(Rm[c + N * k]);
  } else {  // A = R diag(s) L^H
    U = Rm;
    Vh.assign(N * n, 0.0);
    for (int k = 0; k < N; ++k)
      for (int c = 0; c < n; ++c) Vh[k + N * c] = std::conj(L[c + M * k]);
  }
}

// ---------------------------------------------------------- TPO building
// Operator tensor of one site: legs (bond_0..bond_{g-1}, in, out),
// column-major, entry O[..., in, out] = <out| op |in>.
struct SiteOp {
  std::vector<int> shape;  // g bond dims then 2, 2
  std::vector<cd> data;
};

static SiteOp identity_op(int g) {
  SiteOp o;
  o.shape.assign(g, 1);
  o.shape.push_back(2);
  o.shape.push_back(2);
  o.data = {1.0, 0.0, 0.0, 1.0};
  return o;
}

// Apply X after the current operator along bond legs `legs` (X's leading
// legs, in the given order), merging each (old bond, X leg) pair as
// old + D_old * x:  new[..., (b, x)..., in, o'] = sum_o T[..., b..., in, o] X[x..., o, o'].
// X layout: (x_0, ..., x_{k-1}, o_in, o_out) column-major.
static void attach(SiteOp& T, const std::vector<int>& legs, const std::vector<int>& xdims, const std::vector<cd>& X) {
  const int g = (int)T.shape.size() - 2;
  std::vector<int> nshape = T.shape;
  for (size_t i = 0; i < legs.size(); ++i) nshape[legs[i]] = T.shape[legs[i]] * xdims[i];
  size_t nx = 1;
  for (int d : xdims) nx *= d;
  size_t nb = 1;
  for (int k = 0; k < g; ++k) nb *= T.shape[k];
  size_t nnew = 1;
  for (int d : nshape) nnew *= d;
  std::vector<cd> out(nnew, 0.0);
  std::vector<int> bc(g), xc(legs.size());
  for (size_t b = 0; b < nb; ++b) {
    size_t t = b;
    for (int k = 0; k < g; ++k) { bc[k] = (int)(t % T.shape[k]); t /= T.shape[k]; }
    for (size_t x = 0; x < nx; ++x) {
      size_t u = x;
      for (size_t i = 0; i < legs.size(); ++i) { xc[i] = (int)(u % xdims[i]); u /= xdims[i]; }
      size_t nidx = 0, st = 1;
      for (int k = 0; k < g; ++k) {
        int v = bc[k];
        for (size_t i = 0; i < legs.size(); ++i)
          if (legs[i] == k) v = bc[k] + T.shape[k] * xc[i];
        nidx += v * st;
        st *= nshape[k];
      }
      for (int in = 0; in < 2; ++in)
        for (int o2 = 0; o2 < 2; ++o2) {
          cd acc = 0;
          for (int o = 0; o < 2; ++o)
            acc += T.data[b + nb * (in + 2 * o)] * X[x + nx * (o + 2 * o2)];
          out[nidx + st * (in + 2 * o2)] += acc;
        }
    }
  }
  T.shape = nshape;
  T.data = std::move(out);
}

// X for a 1-qubit matrix given row-major, list[2 out + in] = U[out][in]:
// X[o_in + 2 o_out] = U[o_out][o_in] is the same list (the reference's
// InstructionTensor reads it with address c0 + 2 c1, qasmtotpo.h:177-192).
static std::vector<cd> one_qubit_x(const std::vector<cd>& U) { return U; }

struct LayerBuilder {
  const Edges& edges;
  std::vector<int> sites;
  std::map<int, int> pos;
  std::vector<std::vector<int>> bonds;  // per site index: incident edge ids
  std::vector<SiteOp> ops;
  // shortest paths by (from, to) label: FindShortestPath's BFS is the same
  // for every gate on the pair, so each pair is searched once per builder
  std::map<std::pair<int, int>, std::vector<int>> paths;
  const std::vector<int>& path(int a, int b) {
    auto it = paths.find({a, b});
    if (it == paths.end()) it = paths.emplace(std::make_pair(a, b), shortest_path(edges, a, b)).first;
    return it->second;
  }
  LayerBuilder(const Edges& e) : edges(e) {
    sites = site_labels(e);
    for (size_t i = 0; i < sites.size(); ++i) pos[sites[i]] = (int)i;
    bonds.resize(sites.size());
    for (size_t i = 0; i < sites.size(); ++i) bonds[i] = surrounding_bonds(e, sites[i]);
    reset();
  }
  void reset() {
    ops.clear();
    for (size_t i = 0; i < sites.size(); ++i) ops.push_back(identity_op((int)bonds[i].size()));
  }
  int site_index(int label) const {
    auto it = pos.find(label);
    if (it == pos.end()) throw HostError(-1, "gate on qubit " + std::to_string(label) + " that no 2-qubit gate touches");
    return it->second;
  }
  int leg_toward(int si, int other_label) const {
    const int me = sites[si];
    for (size_t k = 0; k < bonds[si].size(); ++k) {
      const auto& e = edges[bonds[si][k]];
      if ((e.first == me && e.second == other_label) || (e.second == me && e.first == other_label)) return (int)k;
    }
    throw HostError(-1, "no edge between path neighbours");
  }
  void one_qubit(int label, const std::vector<cd>& U) {
    const int si = site_index(label);
    attach(ops[si], {}, {}, one_qubit_x(U));
  }
  // Two-qubit gate on (a, b): operator-Schmidt split with trunc SVD
  // (chi_max 4, s_min 1e-12, sqrt(s) to both factors), identity
  // pass-through tensors on intermediate path sites (qasmtotpo.h:287-437).
  void two_qubit(int qa, int qb, const std::vector<cd>& U) {
    // G(a_in, a_out ; b_in, b_out) as a 4 x 4 matrix, row a_in + 2 a_out
    std::vector<cd> G(16);
    for (int ai = 0; ai < 2; ++ai)
      for (int ao = 0; ao < 2; ++ao)
        for (int bi = 0; bi < 2; ++bi)
          for (int bo = 0; bo < 2; ++bo)
            G[(ai + 2 * ao) + 4 * (bi + 2 * bo)] = U[(ao + 2 * bo) * 4 + (ai + 2 * bi)];
    std::vector<cd> Uf, Vh;
    std::vector<double> s;
    small_svd(4, 4, G, Uf, s, Vh);
    int k = 0;
    while (k < 4 && s[k] > 1e-12) ++k;
    if (k == 0) k = 1;
    // A[k, a_in, a_out] = U[(a_in,a_out), k] sqrt(s_k); B[k, b_in, b_out] = sqrt(s_k) Vh[k, (b_in,b_out)]
    std::vector<cd> A(k * 4), B(k * 4);
    for (int c = 0; c < k; ++c) {
      const double sq = std::sqrt(std::abs(s[c]));
      for (int rw = 0; rw < 4; ++rw) {
        A[c + k * rw] = Uf[rw + 4 * c] * sq;
        B[c + k * rw] = sq * Vh[c + 4 * rw];
      }
    }
    const auto& path = this->path(qa, qb);
    if (path.size() < 2) throw HostError(-1, "two-qubit gate between disconnected or equal qubits");
    for (size_t i = 0; i < path.size(); ++i) {
      const int si = site_index(path[i]);
      if (i == 0) {
        attach(ops[si], {leg_toward(si, path[1])}, {k}, A);
      } else if (i + 1 == path.size()) {
        attach(ops[si], {leg_toward(si, path[i - 1])}, {k}, B);
      } else {
        int lm = leg_toward(si, path[i - 1]), lp = leg_toward(si, path[i + 1]);
        std::vector<cd> X(k * k * 4, 0.0);
        for (int x = 0; x < k; ++x)
          for (int o = 0; o < 2; ++o) X[x + k * x + k * k * (o + 2 * o)] = 1.0;
        std::vector<int> legs = {std::min(lm, lp), std::max(lm, lp)};
        attach(ops[si], legs, {k, k}, X);
      }
    }
  }
  // Identity on the physical leg, passing a bond of dimension k from the
  // site's leg toward `prev` to its leg toward `next` (a path's inner site).
  void pass_through(int si, int prev, int next, int k) {
    std::vector<cd> X(k * k * 4, 0.0);
    for (int x = 0; x < k; ++x)
      for (int o = 0; o < 2; ++o) X[x + k * x + k * k * (o + 2 * o)] = 1.0;
    const int lm = leg_toward(si, prev), lp = leg_toward(si, next);
    attach(ops[si], {std::min(lm, lp), std::max(lm, lp)}, {k, k}, X);
  }
  // Three-qubit gate (ccx, cswap; the reference's branch is
  // qasmtotpo.h:439-698): two operator-Schmidt splits of the 8 x 8 gate,
  // each a truncated SVD (chi_max 4, s_min 1e-12, sqrt(s) to both sides):
  //   G[(a), (b), (c)] = sum_{k1,k2} A[k1, a] Bm[k1, k2, b] C[k2, c]
  // with a = (in, out) of the first qubit of the chosen order, etc.  The
  // middle qubit is the one with the shortest total distance to the other
  // two (the instruction's second qubit on ties); bond k1 runs along the
  // shortest path from the first qubit to the middle one and k2 from the
  // middle one to the last, through identity pass-through tensors.  Where
  // the two paths share an edge, that edge carries both bonds (merged in
  // the same order at both ends), so any three connected qubits work.
  void three_qubit(const std::vector<int>& q, const std::vector<cd>& U) {
    int mid = 1;
    size_t best = SIZE_MAX;
    for (int m : {1, 0, 2}) {
      size_t len = 0;
      for (int o = 0; o < 3; ++o)
        if (o != m) {
          const auto& p = path(q[o], q[m]);
          if (p.size() < 2) throw HostError(-1, "three-qubit gate between disconnected or equal qubits");
          len += p.size();
        }
      if (len < best) { best = len; mid = m; }
    }
    int order[3] = {0, mid, 0};
    {
      int j = 0;
      int rest[2];
      for (int o = 0; o < 3; ++o) if (o != mid) rest[j++] = o;
      order[0] = rest[0];
      order[2] = rest[1];
    }
    // G[(a_in, a_out), (b_in, b_out), (c_in, c_out)], qubit x = q[order[x]]
    std::vector<cd> G(64);
    int bit[3];
    for (int x = 0; x < 3; ++x) bit[x] = order[x];  // bit position of x in U's index
    for (int ai = 0; ai < 2; ++ai) for (int ao = 0; ao < 2; ++ao)
      for (int bi = 0; bi < 2; ++bi) for (int bo = 0; bo < 2; ++bo)
        for (int ci = 0; ci < 2; ++ci) for (int co = 0; co < 2; ++co) {
          const int in = (ai << bit[0]) | (bi << bit[1]) | (ci << bit[2]);
          const int out = (ao << bit[0]) | (bo << bit[1]) | (co << bit[2]);
          G[(ai + 2 * ao) + 4 * (bi + 2 * bo) + 16 * (ci + 2 * co)] = U[out * 8 + in];
        }
    auto keep_of = [](const std::vector<double>& s) {
      int k = 0;
      while (k < (int)s.size() && k < 4 && s[k] > 1e-12) ++k;
      return k == 0 ? 1 : k;
    };
    // split 1: (a) x (b, c)
    std::vector<cd> U1, V1;
    std::vector<double> s1;
    small_svd(4, 16, G, U1, s1, V1);
    const int k1 = keep_of(s1);
    std::vector<cd> A(k1 * 4), R1(k1 * 16);  // A[k1 + k1 a]; R1[(k1, b), c] as (4 k1) x 4
    for (int c = 0; c < k1; ++c) {
      const double sq = std::sqrt(std::abs(s1[c]));
      for (int a = 0; a < 4; ++a) A[c + k1 * a] = U1[a + 4 * c] * sq;
      for (int bc = 0; bc < 16; ++bc) {
        const int b = bc % 4, cc = bc / 4;
        R1[(c + k1 * b) + 4 * k1 * cc] = sq * V1[c + std::min(4, 16) * bc];
      }
    }
    // split 2: (k1, b) x (c)
    std::vector<cd> U2, V2;
    std::vector<double> s2;
    small_svd(4 * k1, 4, R1, U2, s2, V2);
    const int k2 = keep_of(s2);
    const int r2 = std::min(4 * k1, 4);  // rank count of the second SVD
    std::vector<cd> Bm(k1 * k2 * 4), C(k2 * 4);  // Bm[x1 + k1 x2 + k1 k2 b]; C[x2 + k2 c]
    for (int c = 0; c < k2; ++c) {
      const double sq = std::sqrt(std::abs(s2[c]));
      for (int x1 = 0; x1 < k1; ++x1)
        for (int b = 0; b < 4; ++b) Bm[x1 + k1 * c + k1 * k2 * b] = U2[(x1 + k1 * b) + 4 * k1 * c] * sq;
      for (int cc = 0; cc < 4; ++cc) C[c + k2 * cc] = sq * V2[c + r2 * cc];
    }
    const int qa = q[order[0]], qb = q[order[1]], qc = q[order[2]];
    const auto& p1 = path(qa, qb);
    const auto& p2 = path(qb, qc);
    // bond k1 from qa to qb
    attach(ops[site_index(qa)], {leg_toward(site_index(qa), p1[1])}, {k1}, A);
    for (size_t i = 1; i + 1 < p1.size(); ++i) pass_through(site_index(p1[i]), p1[i - 1], p1[i + 1], k1);
    // the middle factor joins both bonds
    {
      const int si = site_index(qb);
      const int la = leg_toward(si, p1[p1.size() - 2]), lc = leg_toward(si, p2[1]);
      // both bonds leave through the same edge: one merged index x1 + k1 x2
      // (Bm's layout already), the order of the merges at the other end
      if (la == lc) attach(ops[si], {la}, {k1 * k2}, Bm);
      else attach(ops[si], {la, lc}, {k1, k2}, Bm);
    }
    for (size_t i = 1; i + 1 < p2.size(); ++i) pass_through(site_index(p2[i]), p2[i - 1], p2[i + 1], k2);
    attach(ops[site_index(qc)], {leg_toward(site_index(qc), p2[p2.size() - 2])}, {k2}, C);
  }
  void append(const Instruction& in) {
    // the reference builds NaN operators from an infinite angle (strtod of
    // "1e400") without complaint; here the layer is refused before it can
    // reach the device
    for (double p : in.params)
      if (!std::isfinite(p)) throw HostError(-1, "non-finite gate parameter");
    const auto U = gate_matrix(in);
    const int nq = qubit_count(in);
    if (nq == 1) one_qubit((int)in.qubits[0].index, U);
    else if (nq == 2) two_qubit((int)in.qubits[0].index, (int)in.qubits[1].index, U);
    else if (nq == 3) three_qubit({(int)in.qubits[0].index, (int)in.qubits[1].index, (int)in.qubits[2].index}, U);
    else throw HostError(-6, "gates on more than three qubits are not supported on the estimator path");
  }
};

static Layer pack_layer(const LayerBuilder& lb) {
  Layer L;
  const size_t ne = lb.edges.size();
  L.edge_rank.assign(ne, 1);
  for (size_t si = 0; si < lb.sites.size(); ++si)
    for (size_t k = 0; k < lb.bonds[si].size(); ++k) L.edge_rank[lb.bonds[si][k]] = lb.ops[si].shape[k];
  int64_t off = 0;
  for (size_t si = 0; si < lb.sites.size(); ++si) {
    L.op_offset.push_back(off);
    for (auto& v : lb.ops[si].data) { L.op_data.push_back(v.real()); L.op_data.push_back(v.imag()); }
    off += (int64_t)lb.ops[si].data.size();
  }
  return L;
}

// QasmToTPO, barrier layering (qasmtotpo.h:743-767): a new layer at every
// barrier except a final one.
std::vector<Layer> qasm_tpo(const Program& p, const Edges& edges) {
  LayerBuilder lb(edges);
  std::vector<Layer> out;
  for (size_t i = 0; i < p.instructions.size(); ++i) {
    const auto& in = p.instructions[i];
    if (in.op == Op::BARRIER) {
      if (i + 1 == p.instructions.size()) break;
      out.push_back(pack_layer(lb));
      lb.reset();
      continue;
    }
    lb.append(in);
  }
  out.push_back(pack_layer(lb));
  return out;
}

// QasmToTPO with manual gate-number layering (qasmtotpo.h:709-738): layer m
// takes the next num_gates[m] instructions.  Every instruction is appended as
// a gate, so a barrier (like measure / reset / custom) is an unsupported
// operation there.  The reference writes past its layer vector when the
// program has more instructions than the counts cover and leaves a layer
// that receives no instruction uninitialized; both are refused here.
std::vector<Layer> qasm_tpo_counts(const Program& p, const Edges& edges, const std::vector<int>& num_gates) {
  if (num_gates.empty()) throw HostError(-1, "num_gates is empty");
  for (int n : num_gates)
    if (n < 1) throw HostError(-1, "num_gates entries must be >= 1");
  long long total = 0;
  for (int n : num_gates) total += n;
  if ((long long)p.instructions.size() > total)
    throw HostError(-1, "the program has more instructions than num_gates covers");
  LayerBuilder lb(edges);
  std::vector<Layer> out;
  int count = 0;
  size_t m = 0;
  for (const auto& in : p.instructions) {
    if (in.op == Op::BARRIER || in.op == Op::MEASURE || in.op == Op::RESET || in.op == Op::CUSTOM)
      throw HostError(-6, "matrix for this op not implemented");
    lb.append(in);
    if (++count == num_gates[m]) {
      out.push_back(pack_layer(lb));
      lb.reset();
      count = 0;
      ++m;
    }
  }
  if (count > 0) { out.push_back(pack_layer(lb)); ++m; }
  if (m != num_gates.size()) throw HostError(-1, "a layer of num_gates receives no instruction");
  return out;
}

// One Floquet step of apps/kicked_ising_lattice/circuit.h:14-229:
// exp(-i dt Jz Z Z) on every edge, then exp(-i dt hz Z), then exp(-i dt hx X).
// exp(-i th ZZ) = cos(th) I(x)I - i sin(th) Z(x)Z, split term by term with
// the magnitude shared evenly between the two sites.
Layer kicked_ising_tpo(const Edges& edges, double Jz, double hz, double hx, double dt) {
  if (!std::isfinite(Jz) || !std::isfinite(hz) || !std::isfinite(hx) || !std::isfinite(dt))
    throw HostError(-1, "non-finite kicked-Ising parameter");
  LayerBuilder lb(edges);
  const double th = dt * Jz;
  const cd I(0, 1);
  std::vector<std::pair<std::vector<cd>, std::vector<cd>>> terms;  // (A, B) 2x2 matrices U[out][in]
  const double c = std::cos(th), s = std::sin(th);
  if (std::abs(c) > 1e-15) {
    const double a = std::sqrt(std::abs(c));
    terms.push_back({{a, 0, 0, a}, {c / a, 0, 0, c / a}});
  }
  if (std::abs(s) > 1e-15) {
    const double a = std::sqrt(std::abs(s));
    const cd b = -I * s / a;
    terms.push_back({{a, 0, 0, -a}, {b, 0, 0, -b}});
  }
  const int k = (int)terms.size();
  std::vector<cd> A(k * 4), B(k * 4);
  for (int t = 0; t < k; ++t) {
    const auto xa = one_qubit_x(terms[t].first), xb = one_qubit_x(terms[t].second);
    for (int r = 0; r < 4; ++r) { A[t + k * r] = xa[r]; B[t + k * r] = xb[r]; }
  }
  for (size_t m = 0; m < edges.size(); ++m) {
    const int sa = lb.site_index(edges[m].first), sb = lb.site_index(edges[m].second);
    attach(lb.ops[sa], {lb.leg_toward(sa, edges[m].second)}, {k}, A);
    attach(lb.ops[sb], {lb.leg_toward(sb, edges[m].first)}, {k}, B);
  }
  const std::vector<cd> Uz = {std::exp(-I * (dt * hz)), 0, 0, std::exp(I * (dt * hz))};
  const std::vector<cd> Ux = {std::cos(dt * hx), -I * std::sin(dt * hx), -I * std::sin(dt * hx), std::cos(dt * hx)};
  for (size_t si = 0; si < lb.sites.size(); ++si) attach(lb.ops[si], {}, {}, one_qubit_x(Uz));
  for (size_t si = 0; si < lb.sites.size(); ++si) attach(lb.ops[si], {}, {}, one_qubit_x(Ux));
  return pack_layer(lb);
}

// ------------------------------------------------------ TPO compression
// OptTPObySVD (include/tnbp/ptns/function/optsvdtpo.h:86-214).  For every
// edge m = (a, b) in edge order: C = O_a contracted with O_b over their
// shared bond, rows = O_a's other legs, columns = O_b's other legs (both in
// leg order, column-major); truncated SVD keeping the singular values
// > eps, at most the old bond dimension r and at least one; then
// O_a := U sqrt(s) and O_b := sqrt(s) V^H with the new bond back at the
// bond's leg position.  C = A B has rank <= r, so its SVD is taken from the
// factors: A = Ua diag(sa) Vah, W = diag(sa) Vah B = Uw diag(s) Vwh, and
// C = (Ua Uw) diag(s) Vwh.  The singular values are C's; the singular
// vectors equal an SVD of C up to a unitary on the bond, which changes no
// observable; the cost is O((m + n) r^2) instead of O(m n min(m, n)).
void opt_tpo_svd(const Edges& edges, Layer& layer, double eps) {
  const auto sites = site_labels(edges);
  const size_t ns = sites.size(), ne = edges.size();
  if (layer.edge_rank.size() != ne || layer.op_offset.size() != ns)
    throw HostError(-1, "TPO layer does not match the edge list");
  std::map<int, int> pos;
  for (size_t i = 0; i < ns; ++i) pos[sites[i]] = (int)i;
  std::vector<std::vector<int>> bonds(ns);
  for (size_t i = 0; i < ns; ++i) bonds[i] = surrounding_bonds(edges, sites[i]);

  std::vector<SiteOp> ops(ns);
  const int64_t avail = (int64_t)layer.op_data.size() / 2;
  for (size_t si = 0; si < ns; ++si) {
    auto& o = ops[si];
    int64_t n = 4;
    for (int m : bonds[si]) {
      const int r = layer.edge_rank[m];
      if (r < 1) throw HostError(-1, "TPO bond dimension < 1");
      o.shape.push_back(r);
      n *= r;
    }
    o.shape.push_back(2);
    o.shape.push_back(2);
    const int64_t off = layer.op_offset[si];
    if (off < 0 || off + n > avail) throw HostError(-1, "TPO site operator outside the op data");
    o.data.resize(n);
    for (int64_t x = 0; x < n; ++x) {
      o.data[x] = cd(layer.op_data[2 * (off + x)], layer.op_data[2 * (off + x) + 1]);
      if (!std::isfinite(o.data[x].real()) || !std::isfinite(o.data[x].imag()))
        throw HostError(-1, "non-finite TPO element");
    }
  }

  for (size_t m = 0; m < ne; ++m) {
    const int ia = pos.at(edges[m].first), ib = pos.at(edges[m].second);
    const int pa = (int)(std::find(bonds[ia].begin(), bonds[ia].end(), (int)m) - bonds[ia].begin());
    const int pb = (int)(std::find(bonds[ib].begin(), bonds[ib].end(), (int)m) - bonds[ib].begin());
    SiteOp& A = ops[ia];
    SiteOp& B = ops[ib];
    const int r = A.shape[pa];
    // A as an (ma x r) matrix, B as an (r x nb) matrix: the row (column)
    // index is lo + below * hi with lo the legs before the bond, hi after it
    int64_t below_a = 1, below_b = 1;
    for (int k = 0; k < pa; ++k) below_a *= A.shape[k];
    for (int k = 0; k < pb; ++k) below_b *= B.shape[k];
    const int ma = (int)(A.data.size() / r), nb = (int)(B.data.size() / r);
    std::vector<cd> Am(A.data.size()), Bm(B.data.size());
    for (int64_t x = 0; x < (int64_t)A.data.size(); ++x) {
      const int64_t lo = x % below_a, j = (x / below_a) % r, hi = x / (below_a * r);
      Am[lo + below_a * hi + (int64_t)ma * j] = A.data[x];
    }
    for (int64_t x = 0; x < (int64_t)B.data.size(); ++x) {
      const int64_t lo = x % below_b, j = (x / below_b) % r, hi = x / (below_b * r);
      Bm[j + (int64_t)r * (lo + below_b * hi)] = B.data[x];
    }
    std::vector<cd> Ua, Vah, Uw, Vwh;
    std::vector<double> sa, sw;
    small_svd(ma, r, Am, Ua, sa, Vah);
    const int ka = (int)sa.size();
    std::vector<cd> W((size_t)ka * nb, 0.0);
    for (int c = 0; c < nb; ++c)
      for (int j = 0; j < r; ++j) {
        const cd b = Bm[j + (size_t)r * c];
        if (b == 0.0) continue;
        for (int i = 0; i < ka; ++i) W[i + (size_t)ka * c] += sa[i] * Vah[i + (size_t)ka * j] * b;
      }
    small_svd(ka, nb, W, Uw, sw, Vwh);
    const int kw = (int)sw.size();
    int keep = 0;
    while (keep < kw && keep < r && sw[keep] > eps) ++keep;
    if (keep == 0) keep = 1;

    SiteOp nA, nB;
    nA.shape = A.shape;
    nA.shape[pa] = keep;
    nB.shape = B.shape;
    nB.shape[pb] = keep;
    nA.data.assign((size_t)ma * keep, 0.0);
    nB.data.assign((size_t)nb * keep, 0.0);
    for (int j = 0; j < keep; ++j) {
      const double sq = std::sqrt(sw[j]);
      for (int row = 0; row < ma; ++row) {
        cd u = 0;  // (Ua Uw)[row, j]
        for (int i = 0; i < ka; ++i) u += Ua[row + (size_t)ma * i] * Uw[i + (size_t)ka * j];
        const int64_t lo = row % below_a, hi = row / below_a;
        nA.data[lo + below_a * (j + (int64_t)keep * hi)] = u * sq;
      }
      for (int col = 0; col < nb; ++col) {
        const int64_t lo = col % below_b, hi = col / below_b;
        nB.data[lo + below_b * (j + (int64_t)keep * hi)] = sq * Vwh[j + (size_t)kw * col];
      }
    }
    A = std::move(nA);
    B = std::move(nB);
  }

  Layer out;
  out.edge_rank.assign(ne, 1);
  for (size_t si = 0; si < ns; ++si)
    for (size_t k = 0; k < bonds[si].size(); ++k) out.edge_rank[bonds[si][k]] = ops[si].shape[k];
  int64_t off = 0;
  for (size_t si = 0; si < ns; ++si) {
    out.op_offset.push_back(off);
    for (auto& v : ops[si].data) { out.op_data.push_back(v.real()); out.op_data.push_back(v.imag()); }
    off += (int64_t)ops[si].data.size();
  }
  layer = std::move(out);
}

// -------------------------------------------------------------- Pauli
// Rows of the observable text come from pauli_rows (qasm_text.cpp);
// classification of ClassifyOps (paulitotpo.h:99-153).
namespace {
bool adjacent(const Edges& edges, int a, int b) {
  for (int m : surrounding_bonds(edges, a)) {
    const auto& e = edges[m];
    if ((e.first == a && e.second == b) || (e.first == b && e.second == a)) return true;
  }
  return false;
}

}  // namespace

std::vector<PauliTerm> pauli_terms(const std::string& text, const Edges& edges, int64_t* n_dropped) {
  std::vector<PauliTerm> out;
  int64_t dropped = 0;
  const auto rows = pauli_rows(text);
  for (size_t row = 0; row < rows.size(); ++row) {
    const auto& ops = rows[row].ops;
    PauliTerm t;
    t.coeff_re = rows[row].re;
    t.coeff_im = rows[row].im;
    t.row = (int64_t)row;
    if (ops.size() == 1) {
      t.kind = 1; t.q0 = ops[0].first; t.q1 = -1; t.l0 = ops[0].second; t.l1 = 0;
      out.push_back(t);
    } else if (ops.size() == 2 && adjacent(edges, ops[0].first, ops[1].first)) {
      t.kind = 2; t.q0 = ops[0].first; t.q1 = ops[1].first; t.l0 = ops[0].second; t.l1 = ops[1].second;
      out.push_back(t);
    } else {
      ++dropped;
    }
  }
  if (n_dropped) *n_dropped = dropped;
  return out;
}

std::vector<PauliString> pauli_strings(const std::string& text, const Edges& edges) {
  std::vector<PauliString> out;
  for (const auto& r : pauli_rows(text)) {
    PauliString t;
    t.coeff_re = r.re;
    t.coeff_im = r.im;
    for (const auto& o : r.ops) { t.qubits.push_back(o.first); t.letters.push_back(o.second); }
    const size_t k = r.ops.size();
    t.kind = k == 0 ? 0 : k == 1 ? 1 : (k == 2 && adjacent(edges, r.ops[0].first, r.ops[1].first)) ? 2 : 3;
    out.push_back(std::move(t));
  }
  return out;
}

// PauliOpMatrix (paulitotpo.h:21-35) in the reference's tensor layout
// O[c0, c1] = list[c0 + 2 c1].
std::vector<cd> pauli_list(char l) {
  const cd I(0, 1);
  switch (l) {
    case 'I': return {1, 0, 0, 1};
    case 'X': return {0, 1, 1, 0};
    case 'Y': return {0, -I, I, 0};
    case 'Z': return {1, 0, 0, -1};
    default: throw HostError(-6, "matrix for this op not implemented");
  }
}

}  // namespace tnbp_host
