/* C++ interface of the B200 estimator engine with the names, argument
   meanings and exceptions of tnbp's estimator path, header-only over the C
   ABI of tnbp_b200.h (link libtnbp_b200.so).

   What changes against the reference's templates: the PEPS state (V, SiteIdx,
   Site_To_MpiRank, E, EdgeIdx and the F scratch of the apps) lives on the
   GPU inside a tnbp_b200::State instead of caller-owned std::vector<TenT>;
   TPO layers are packed host arrays (TpoLayer) instead of vectors of
   tensors; BeliefPropagation updates every layer and copies F -> E in one
   call (the apps call it once per layer and then copy,
   apps/estimator/main.cc:133-143).  Everything else keeps its meaning:
   edges as (site, site) pairs in edge order, site labels, leg order
   (GetSurroundingBondIndex), the first/second half message convention,
   column-major tensors with coordinate 0 fastest.

   Errors become the exceptions the reference throws (tnbp_b200.h's status
   codes): TNBP_EPARSE -> ParseError (a std::runtime_error, as
   qasm::ParseError, include/qasm/ir.h:36-41, and the sparse-Pauli reader's
   runtime_error); TNBP_EINVAL -> std::invalid_argument; TNBP_ENOMEM ->
   std::bad_alloc; TNBP_ENOTCONV -> NotConverged; anything else (a
   cancelled request, CUDA errors, no device) -> std::runtime_error with
   the engine's message. */
#pragma once

#include <algorithm>
#include <array>
#include <complex>
#include <cstdint>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tnbp_b200.h"

namespace tnbp_b200 {

using Edges = std::vector<std::pair<int, int>>;
using cplx = std::complex<double>;

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct NotConverged : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check(int rc) {
  if (rc == TNBP_OK) return;
  const std::string msg = tnbp_last_error();
  switch (rc) {
    case TNBP_EPARSE: throw ParseError(msg);
    case TNBP_EINVAL: throw std::invalid_argument(msg);
    case TNBP_ENOMEM: throw std::bad_alloc();
    case TNBP_ENOTCONV: throw NotConverged(msg);
    default: throw std::runtime_error(msg);
  }
}

namespace detail {
inline std::vector<int32_t> flat(const Edges& e) {
  std::vector<int32_t> f;
  f.reserve(2 * e.size());
  for (const auto& p : e) { f.push_back(p.first); f.push_back(p.second); }
  return f;
}
inline Edges pairs(const std::vector<int32_t>& f, int64_t n) {
  Edges e((size_t)n);
  for (int64_t i = 0; i < n; ++i) e[i] = {f[2 * i], f[2 * i + 1]};
  return e;
}
}  // namespace detail

/* ------------------------------------------------------------ graphs */

/* bond_square_lattice (include/tnbp/lattice/square.h:14-34). */
inline Edges bond_square_lattice(int Lx, int Ly) {
  int64_t n = 0;
  check(tnbp_square_lattice(Lx, Ly, nullptr, 0, &n));
  std::vector<int32_t> f(2 * n + 2);
  check(tnbp_square_lattice(Lx, Ly, f.data(), n, &n));
  return detail::pairs(f, n);
}

/* GetSiteIndexFromBond (include/tnbp/framework/graph.h:23-35): sorted labels. */
inline std::vector<int> GetSiteIndexFromBond(const Edges& edges) {
  std::vector<int> s;
  for (const auto& p : edges) { s.push_back(p.first); s.push_back(p.second); }
  std::sort(s.begin(), s.end());
  s.erase(std::unique(s.begin(), s.end()), s.end());
  return s;
}

/* GetSurroundingBondIndex (graph.h:40-55): leg k of `site` = k-th edge containing it. */
inline std::vector<int> GetSurroundingBondIndex(int site, const Edges& edges) {
  const auto f = detail::flat(edges);
  int32_t n = 0;
  check(tnbp_surrounding_bonds(f.data(), (int64_t)edges.size(), site, nullptr, 0, &n));
  std::vector<int32_t> out(n + 1);
  check(tnbp_surrounding_bonds(f.data(), (int64_t)edges.size(), site, out.data(), n, &n));
  return std::vector<int>(out.begin(), out.begin() + n);
}

/* FindShortestPath (graph.h:57-108). */
inline std::vector<int> FindShortestPath(const Edges& edges, int src, int dst) {
  const auto f = detail::flat(edges);
  int32_t n = 0;
  check(tnbp_shortest_path(f.data(), (int64_t)edges.size(), src, dst, nullptr, 0, &n));
  std::vector<int32_t> out(n + 1);
  check(tnbp_shortest_path(f.data(), (int64_t)edges.size(), src, dst, out.data(), n, &n));
  return std::vector<int>(out.begin(), out.begin() + n);
}

/* GreedyEdgeLayering (graph.h:138-170). */
inline std::vector<Edges> GreedyEdgeLayering(const Edges& edges) {
  const auto f = detail::flat(edges);
  std::vector<int32_t> layer(edges.size() + 1);
  int32_t nl = 0;
  check(tnbp_greedy_layering(f.data(), (int64_t)edges.size(), layer.data(), &nl));
  std::vector<Edges> out(nl);
  for (size_t i = 0; i < edges.size(); ++i) out[layer[i]].push_back(edges[i]);
  return out;
}

/* EdgesFromQasm (include/tnbp/parser/qasmtoedge.h:38-56) of a program's text. */
inline Edges EdgesFromQasm(const std::string& qasm_source) {
  int64_t n = 0;
  check(tnbp_qasm_edges(qasm_source.c_str(), nullptr, 0, &n));
  std::vector<int32_t> f(2 * n + 2);
  check(tnbp_qasm_edges(qasm_source.c_str(), f.data(), n, &n));
  return detail::pairs(f, n);
}

/* -------------------------------------------------------------- TPOs */

/* One TPO layer: edge_rank[e] the operator bond dimension of edge e;
   op_offset[s] the element offset of site s's operator (shape (r_legs...,
   2, 2), column-major, O[..., in, out]) in op_data. */
struct TpoLayer {
  std::vector<int32_t> edge_rank;
  std::vector<int64_t> op_offset;
  std::vector<cplx> op_data;
};

/* QasmToTPO (include/tnbp/parser/qasmtotpo.h:709-767): one layer per
   barrier-delimited block. */
inline std::vector<TpoLayer> QasmToTPO(const std::string& qasm_source, const Edges& edges) {
  const auto f = detail::flat(edges);
  const int64_t ne = (int64_t)edges.size(), ns = (int64_t)GetSiteIndexFromBond(edges).size();
  int32_t nl = 0;
  int64_t nel = 0;
  check(tnbp_qasm_tpo(qasm_source.c_str(), f.data(), ne, nullptr, nullptr, nullptr, 0, &nl, &nel));
  std::vector<int32_t> rank((size_t)nl * ne + 1);
  std::vector<int64_t> off((size_t)nl * ns + 1);
  std::vector<cplx> data((size_t)nel + 1);
  check(tnbp_qasm_tpo(qasm_source.c_str(), f.data(), ne, rank.data(), off.data(),
                      reinterpret_cast<double*>(data.data()), nel, &nl, &nel));
  std::vector<TpoLayer> out(nl);
  for (int32_t l = 0; l < nl; ++l) {
    const int64_t base = off[(size_t)l * ns];
    const int64_t end = l + 1 < nl ? off[(size_t)(l + 1) * ns] : nel;
    out[l].edge_rank.assign(rank.begin() + (size_t)l * ne, rank.begin() + (size_t)(l + 1) * ne);
    for (int64_t s = 0; s < ns; ++s) out[l].op_offset.push_back(off[(size_t)l * ns + s] - base);
    out[l].op_data.assign(data.begin() + base, data.begin() + end);
  }
  return out;
}

/* QasmToTPO with manual gate-number layering (qasmtotpo.h:709-738):
   layer m takes the next num_gates[m] instructions. */
inline std::vector<TpoLayer> QasmToTPO(const std::string& qasm_source, const Edges& edges,
                                       const std::vector<int>& num_gates) {
  const auto f = detail::flat(edges);
  const std::vector<int32_t> ng(num_gates.begin(), num_gates.end());
  const int64_t ne = (int64_t)edges.size(), ns = (int64_t)GetSiteIndexFromBond(edges).size();
  int32_t nl = 0;
  int64_t nel = 0;
  check(tnbp_qasm_tpo_counts(qasm_source.c_str(), f.data(), ne, ng.data(), (int32_t)ng.size(), nullptr, nullptr,
                             nullptr, 0, &nl, &nel));
  std::vector<int32_t> rank((size_t)nl * ne + 1);
  std::vector<int64_t> off((size_t)nl * ns + 1);
  std::vector<cplx> data((size_t)nel + 1);
  check(tnbp_qasm_tpo_counts(qasm_source.c_str(), f.data(), ne, ng.data(), (int32_t)ng.size(), rank.data(),
                             off.data(), reinterpret_cast<double*>(data.data()), nel, &nl, &nel));
  std::vector<TpoLayer> out(nl);
  for (int32_t l = 0; l < nl; ++l) {
    const int64_t base = off[(size_t)l * ns];
    const int64_t end = l + 1 < nl ? off[(size_t)(l + 1) * ns] : nel;
    out[l].edge_rank.assign(rank.begin() + (size_t)l * ne, rank.begin() + (size_t)(l + 1) * ne);
    for (int64_t s = 0; s < ns; ++s) out[l].op_offset.push_back(off[(size_t)l * ns + s] - base);
    out[l].op_data.assign(data.begin() + base, data.begin() + end);
  }
  return out;
}

/* OptTPObySVD (include/tnbp/ptns/function/optsvdtpo.h:86-214), in place. */
inline void OptTPObySVD(const Edges& edges, TpoLayer& O, double eps) {
  const auto f = detail::flat(edges);
  int64_t n = 0;
  check(tnbp_opt_tpo_svd(f.data(), (int64_t)edges.size(), eps, O.edge_rank.data(), O.op_offset.data(),
                         reinterpret_cast<double*>(O.op_data.data()), &n));
  O.op_data.resize((size_t)n);
}

/* CircuitTPO (apps/kicked_ising_lattice/circuit.h:14-229): one Floquet step. */
inline TpoLayer CircuitTPO(const Edges& edges, double Jz, double hz, double hx, double dt) {
  const auto f = detail::flat(edges);
  int64_t nel = 0;
  check(tnbp_kicked_ising_tpo(f.data(), (int64_t)edges.size(), Jz, hz, hx, dt, nullptr, nullptr, nullptr, 0, &nel));
  TpoLayer t;
  t.edge_rank.resize(edges.size());
  t.op_offset.resize(GetSiteIndexFromBond(edges).size());
  t.op_data.resize((size_t)nel);
  check(tnbp_kicked_ising_tpo(f.data(), (int64_t)edges.size(), Jz, hz, hx, dt, t.edge_rank.data(),
                              t.op_offset.data(), reinterpret_cast<double*>(t.op_data.data()), nel, &nel));
  return t;
}

/* ------------------------------------------------------ observables */

/* load_sparse_pauli_op + SparsePauliToTensorOp + ClassifyOps
   (include/pauli/sparse_pauli.h:52-97, include/tnbp/parser/paulitotpo.h:39-153)
   on the text of a .txt observable: the kept terms (kind 1: one site; 2: an
   adjacent pair) and the count of dropped ones. */
struct PauliTerms {
  std::vector<int32_t> kind, q0, q1, row;
  std::string letters;  // two per term
  std::vector<cplx> coeff;
  int64_t dropped = 0;
  size_t size() const { return kind.size(); }
};

inline PauliTerms ClassifyOps(const std::string& sparse_pauli_text, const Edges& edges) {
  const auto f = detail::flat(edges);
  int64_t nk = 0, nd = 0;
  check(tnbp_pauli_terms(sparse_pauli_text.c_str(), f.data(), (int64_t)edges.size(), nullptr, nullptr, nullptr,
                         nullptr, nullptr, nullptr, 0, &nk, &nd));
  PauliTerms t;
  t.kind.resize(nk + 1); t.q0.resize(nk + 1); t.q1.resize(nk + 1); t.row.resize(nk + 1);
  std::vector<char> l(2 * nk + 2);
  t.coeff.resize(nk + 1);
  check(tnbp_pauli_terms(sparse_pauli_text.c_str(), f.data(), (int64_t)edges.size(), t.kind.data(), t.q0.data(),
                         t.q1.data(), l.data(), reinterpret_cast<double*>(t.coeff.data()), t.row.data(), nk, &nk,
                         &nd));
  t.kind.resize(nk); t.q0.resize(nk); t.q1.resize(nk); t.row.resize(nk); t.coeff.resize(nk);
  t.letters.assign(l.begin(), l.begin() + 2 * nk);
  t.dropped = nd;
  return t;
}

/* ---------------------------------------------------------- the state */

/* The device-resident PEPS of one edge list: site tensors V (in
   GetSiteIndexFromBond order, shape (D_legs..., d)) and the 2|E| messages
   E (m < |E| computed at edges[m].first, the rest at .second). */
class State {
 public:
  explicit State(const Edges& edges, int precision = TNBP_C128, uint64_t hbm_budget_bytes = 0)
      : edges_(edges), sites_(GetSiteIndexFromBond(edges)) {
    const auto f = detail::flat(edges);
    check(tnbp_job_create(f.data(), (int64_t)edges.size(), nullptr, precision, nullptr, hbm_budget_bytes, &job_));
  }
  ~State() {
    if (job_) tnbp_job_destroy(job_);
  }
  State(const State&) = delete;
  State& operator=(const State&) = delete;
  State(State&& o) noexcept : job_(o.job_), edges_(std::move(o.edges_)), sites_(std::move(o.sites_)) { o.job_ = nullptr; }

  tnbp_job* handle() { return job_; }
  const Edges& edges() const { return edges_; }
  const std::vector<int>& sites() const { return sites_; }

  std::vector<int> bond_dims() const {
    std::vector<int32_t> d(edges_.size() + 1);
    check(tnbp_bond_dims(job_, d.data()));
    return std::vector<int>(d.begin(), d.begin() + edges_.size());
  }
  std::vector<int> site_shape(int64_t site_index) const {
    std::vector<int32_t> sh(64);
    int32_t r = 0;
    check(tnbp_site_shape(job_, site_index, sh.data(), 64, &r));
    return std::vector<int>(sh.begin(), sh.begin() + r);
  }
  std::vector<cplx> site(int64_t site_index) {
    size_t n = 1;
    for (int d : site_shape(site_index)) n *= (size_t)d;
    std::vector<cplx> v(n);
    check(tnbp_download_site(job_, site_index, reinterpret_cast<double*>(v.data()), (int64_t)n));
    return v;
  }
  std::vector<cplx> message(int64_t m) {
    int32_t D = 0;
    check(tnbp_download_message(job_, m, nullptr, 0, &D));
    std::vector<cplx> v((size_t)D * D);
    check(tnbp_download_message(job_, m, reinterpret_cast<double*>(v.data()), (int64_t)v.size(), &D));
    return v;
  }

 private:
  tnbp_job* job_ = nullptr;
  Edges edges_;
  std::vector<int> sites_;
};

/* --------------------------------------------------------- functions */

/* InitTensorProductState (include/tnbp/ptns/function/init.h:18-95): |0...0>. */
inline State InitTensorProductState(const Edges& I, int precision = TNBP_C128) { return State(I, precision); }

/* AbsorbTPO (include/tnbp/ptns/function/apply.h:15-177). */
inline void AbsorbTPO(State& W, const TpoLayer& O) {
  tnbp_tpo* t = nullptr;
  check(tnbp_tpo_create(W.handle(), O.edge_rank.data(), O.op_offset.data(),
                        reinterpret_cast<const double*>(O.op_data.data()), &t));
  const int rc = tnbp_absorb_tpo(W.handle(), t);
  tnbp_tpo_destroy(t);
  check(rc);
}

/* BeliefPropagation (include/tnbp/ptns/function/bp.h:66-261) over every
   layer, then the apps' F -> E copy: one Jacobi sweep. */
inline void BeliefPropagation(State& W) { check(tnbp_bp_sweep(W.handle())); }

/* BeliefPropagationCondition (bp.h:266-355). */
inline double BeliefPropagationCondition(State& W) {
  double r = 0.0;
  check(tnbp_bp_condition(W.handle(), &r));
  return r;
}

/* The apps' BP loop (apps/estimator/main.cc:131-157): returns (sweeps applied,
   last condition). */
inline std::pair<int, double> BeliefPropagationLoop(State& W, double tol, int max_iter) {
  int32_t it = 0;
  double c = 0.0;
  check(tnbp_bp_run(W.handle(), tol, max_iter, &it, &c));
  return {it, c};
}

/* Truncation (include/tnbp/ptns/function/truncation.h:18-222): res_bond_dim
   and res_trunc_err per edge. */
inline void Truncation(State& W, int max_dim, double eps, std::vector<int>& res_bond_dim,
                       std::vector<double>& res_trunc_err) {
  std::vector<int32_t> d(W.edges().size() + 1);
  res_trunc_err.assign(W.edges().size() + 1, 0.0);
  check(tnbp_truncate(W.handle(), max_dim, eps, d.data(), res_trunc_err.data()));
  res_bond_dim.assign(d.begin(), d.begin() + W.edges().size());
  res_trunc_err.resize(W.edges().size());
}

/* Measure, one site per entry (measure.h:15-94): Site = site labels,
   O[i] = 2x2 operator, column-major O[p, p']. */
inline std::vector<cplx> Measure(State& W, const std::vector<int>& Site, const std::vector<std::array<cplx, 4>>& O) {
  if (Site.size() != O.size()) throw std::invalid_argument("one operator per site");
  std::vector<int64_t> idx;
  for (int s : Site) {
    int64_t k = -1;
    for (size_t i = 0; i < W.sites().size(); ++i)
      if (W.sites()[i] == s) k = (int64_t)i;
    if (k < 0) throw std::invalid_argument("site " + std::to_string(s) + " is not in the edge list");
    idx.push_back(k);
  }
  std::vector<cplx> out(Site.size() + 1);
  check(tnbp_measure_1site(W.handle(), (int64_t)Site.size(), idx.data(), reinterpret_cast<const double*>(O.data()),
                           reinterpret_cast<double*>(out.data())));
  out.resize(Site.size());
  return out;
}

/* Measure, nearest-neighbour pairs (measure.h:100-300): Edge = label pairs,
   O[i] = (2,2,2,2) operator O[p_a, p_b, p_a', p_b'], column-major. */
inline std::vector<cplx> Measure(State& W, const Edges& Edge, const std::vector<std::array<cplx, 16>>& O) {
  if (Edge.size() != O.size()) throw std::invalid_argument("one operator per pair");
  const auto f = detail::flat(Edge);
  std::vector<cplx> out(Edge.size() + 1);
  check(tnbp_measure_2site(W.handle(), (int64_t)Edge.size(), f.data(), reinterpret_cast<const double*>(O.data()),
                           reinterpret_cast<double*>(out.data())));
  out.resize(Edge.size());
  return out;
}

/* sum_k c_k <P_k> over the kept terms (FP64; not in the reference, which
   prints the per-term values); per-term values into *per_term if given. */
inline cplx MeasurePauliSum(State& W, const PauliTerms& t, std::vector<cplx>* per_term = nullptr) {
  std::vector<cplx> per(t.size() + 1);
  cplx sum = 0.0;
  if (t.size())
    check(tnbp_measure_pauli_sum(W.handle(), (int64_t)t.size(), t.kind.data(), t.q0.data(), t.q1.data(),
                                 t.letters.data(), reinterpret_cast<const double*>(t.coeff.data()),
                                 reinterpret_cast<double*>(per.data()), reinterpret_cast<double*>(&sum)));
  if (per_term) per_term->assign(per.begin(), per.begin() + t.size());
  return sum;
}

/* Every row of an observable text, the rows ClassifyOps drops measured on
   their tree clusters (not in the reference): returns the all-rows sum;
   per-row values and kinds (0 identity, 1, 2 kept, 3 cluster) if given. */
inline cplx MeasurePauliText(State& W, const std::string& sparse_pauli_text, std::vector<cplx>* values = nullptr,
                             std::vector<int>* kinds = nullptr) {
  int64_t n = 0;
  check(tnbp_measure_pauli_text(W.handle(), sparse_pauli_text.c_str(), 1, nullptr, nullptr, 0, &n, nullptr));
  std::vector<cplx> v((size_t)n + 1);
  std::vector<int32_t> k((size_t)n + 1);
  cplx sum = 0.0;
  check(tnbp_measure_pauli_text(W.handle(), sparse_pauli_text.c_str(), 1, reinterpret_cast<double*>(v.data()),
                                k.data(), n, &n, reinterpret_cast<double*>(&sum)));
  if (values) values->assign(v.begin(), v.begin() + n);
  if (kinds) kinds->assign(k.begin(), k.begin() + n);
  return sum;
}

/* SaveTPS / LoadTPS (include/tnbp/ptns/function/iotps.h:37-105) of the
   state to / from a file (single rank: the restart app's
   make_rank_filename(prefix, 0) is prefix + "000000.dat"). */
inline void SaveTPS(State& W, const std::string& filename) { check(tnbp_save_state(W.handle(), filename.c_str())); }
inline void LoadTPS(State& W, const std::string& filename) { check(tnbp_load_state(W.handle(), filename.c_str())); }

/* ---------------------------------------------------- served requests */

/* The continuous-batching estimator server (tnbp_server_*): requests queue
   and are admitted by HBM footprint; every step() runs one batched BP sweep
   over all admitted requests.  result() is empty while a request runs and
   throws the request's own error (NotConverged, ..., or std::runtime_error
   for a cancelled one) if it failed. */
class Server {
 public:
  explicit Server(int precision = TNBP_MIXED, uint64_t hbm_budget_bytes = 0, int max_active = 64) {
    check(tnbp_server_create(precision, hbm_budget_bytes, max_active, &srv_));
  }
  ~Server() {
    if (srv_) tnbp_server_destroy(srv_);
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  /* Kicked Ising on an L x L lattice: n_steps of RZZ(theta_j) on every edge
     then RX(theta_h), BP to bp_tol / bp_max_iter, truncation to chi;
     observable = ClassifyOps' kept terms of `terms`. */
  int64_t submit_kicked_ising(int L, int chi, int n_steps, double theta_j, double theta_h, const PauliTerms& terms,
                              double bp_tol = 1e-8, int bp_max_iter = 50, double sv_min = 1e-8) {
    int64_t id = 0;
    check(tnbp_server_submit_kicked_ising(srv_, L, chi, n_steps, theta_j, theta_h, bp_tol, bp_max_iter, sv_min,
                                          (int64_t)terms.size(), terms.kind.data(), terms.q0.data(),
                                          terms.q1.data(), terms.letters.data(),
                                          reinterpret_cast<const double*>(terms.coeff.data()), &id));
    return id;
  }
  /* The estimator app's workload: a QASM program and a sparse-Pauli text. */
  int64_t submit_qasm(const std::string& qasm_source, const std::string& sparse_pauli_text, int chi,
                      double bp_tol = 1e-8, int bp_max_iter = 50, double sv_min = 1e-8, bool do_opt_tpo = false,
                      double eps_opt_tpo = 1e-8) {
    int64_t id = 0;
    check(tnbp_server_submit_qasm(srv_, qasm_source.c_str(), sparse_pauli_text.c_str(), chi, bp_tol, bp_max_iter,
                                  sv_min, do_opt_tpo ? 1 : 0, eps_opt_tpo, &id));
    return id;
  }
  /* One server step; returns the number of requests that finished in it. */
  int step(int* n_active = nullptr, int* n_queued = nullptr) {
    int32_t a = 0, q = 0, d = 0;
    check(tnbp_server_step(srv_, &a, &q, &d));
    if (n_active) *n_active = a;
    if (n_queued) *n_queued = q;
    return d;
  }
  /* true and the request's sum_k c_k <P_k> once it has finished. */
  bool result(int64_t id, cplx* sum) {
    double v[2] = {0.0, 0.0};
    int32_t pending = 1;
    check(tnbp_server_result(srv_, id, v, &pending));
    if (pending) return false;
    if (sum) *sum = cplx(v[0], v[1]);
    return true;
  }
  void cancel(int64_t id) { check(tnbp_server_cancel(srv_, id)); }
  /* Restart non-converging requests in complex128 (reduced-precision servers). */
  void set_escalation(bool on) { check(tnbp_server_set_escalation(srv_, on ? 1 : 0)); }
  /* Escalate only loops whose condition never fell below min_cond. */
  void set_escalation_threshold(double min_cond) { check(tnbp_server_set_escalation_threshold(srv_, min_cond)); }
  struct RequestInfo {
    int precision;
    bool escalated, bp_converged;
    int unconverged_loops;
    double worst_final_cond, worst_min_cond;
  };
  RequestInfo info(int64_t id) {
    int32_t p = 0, e = 0, c = 0, n = 0;
    double wf = 0.0, wm = 0.0;
    check(tnbp_server_request_info(srv_, id, &p, &e, &c));
    check(tnbp_server_request_bp_stats(srv_, id, &n, &wf, &wm));
    return RequestInfo{p, e != 0, c != 0, n, wf, wm};
  }

 private:
  tnbp_server* srv_ = nullptr;
};

}  // namespace tnbp_b200
