// tnbp's hot-path functions for gqten::tensor<std::complex<double>> on the
// GPU: the definitions of the overloads declared in
// include/tnbp_dropin/gqten/gqten.h.  With that header first on the include
// path, tnbp's apps compile unchanged and these functions replace tnbp's
// templates (apply.h AbsorbTPO, bp.h BeliefPropagation and
// BeliefPropagationCondition, truncation.h Truncation, measure.h Measure) on
// the same caller-owned std::vector<TenT> containers.
//
// The state stays on the device between calls: one process-wide job mirrors
// the caller's lattice.  Before each call the caller's site tensors and
// messages are compared with host copies of what the device holds and only
// tensors that changed are uploaded; results the call produces (new site
// tensors and messages) are downloaded back into the caller's vectors.  BP
// sweeps the whole lattice at once, so the app's per-layer
// BeliefPropagation calls of one iteration (each asking for the messages of
// one layer's edges) share one device sweep.  The job's arithmetic is the
// engine's complex128 path unless TNBP_DROPIN_PRECISION selects "mixed" or
// "c64".
//
// One process runs one lattice on one GPU: the site and edge index lists
// must cover every site and edge (the single-rank layout of
// InitTensorProductState); a multi-rank layout is refused.
#include <algorithm>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "gqten/gqten.h"
#include "tnbp_b200.h"

namespace {

using cd = std::complex<double>;
using Ten = tnbp::DropinTensor;
using Edges = std::vector<std::pair<int, int>>;

void ok(int rc, const char* what) {
  if (rc != TNBP_OK) throw std::runtime_error(std::string(what) + ": " + tnbp_last_error());
}

int dropin_precision() {
  const char* p = std::getenv("TNBP_DROPIN_PRECISION");
  if (!p || !*p || std::strcmp(p, "c128") == 0) return TNBP_C128;
  if (std::strcmp(p, "mixed") == 0) return TNBP_MIXED;
  if (std::strcmp(p, "c64") == 0) return TNBP_C64;
  throw std::invalid_argument("TNBP_DROPIN_PRECISION must be c128, mixed or c64");
}

struct Held {
  std::vector<int32_t> shape;
  std::vector<cd> data;
  bool same(const Ten& t) const {
    const auto sh = t.Shape();
    return sh.size() == shape.size() && std::equal(sh.begin(), sh.end(), shape.begin()) &&
           t.Size() == data.size() && std::memcmp(t.GetRaw(), data.data(), data.size() * sizeof(cd)) == 0;
  }
  void take(const Ten& t) {
    shape = t.Shape();
    data.assign(t.GetRaw(), t.GetRaw() + t.Size());
  }
  Ten tensor() const { return Ten(shape, data); }
};

struct Mirror {
  tnbp_job* job = nullptr;
  Edges edges;
  std::vector<Held> v, e;        // what the device holds
  bool f_valid = false;          // f = one sweep from (v, f_src_e)
  std::vector<Held> f, f_src_e;  // messages of that sweep, and the messages it started from
  ~Mirror() {
    if (job) tnbp_job_destroy(job);
  }
  int ns() const { return (int)v.size(); }
  int ne() const { return (int)edges.size(); }

  // the job for lattice I (created with the caller's physical dims)
  void bind(const Edges& I, const std::vector<Ten>& V) {
    if (job && I == edges) return;
    if (job) tnbp_job_destroy(job);
    job = nullptr;
    edges = I;
    std::vector<int32_t> flat;
    for (auto& p : I) { flat.push_back(p.first); flat.push_back(p.second); }
    std::vector<int32_t> pd;
    for (auto& t : V) pd.push_back(t.Shape().empty() ? 2 : t.Shape().back());
    ok(tnbp_job_create(flat.data(), (int64_t)I.size(), pd.data(), dropin_precision(), nullptr, 0, &job),
       "tnbp_job_create");
    v.assign(V.size(), Held());
    e.assign(2 * I.size(), Held());
    f_valid = false;
  }

  // upload the caller's tensors that differ from the device's (messages
  // first: they fix the bond dimensions the site shapes are checked against)
  void sync(const Edges& I, const std::vector<Ten>& V, const std::vector<Ten>& E, const std::vector<int>& SiteIdx,
            const std::vector<int>& EdgeIdx) {
    bind(I, V);
    if ((int)V.size() != ns() || (int)SiteIdx.size() != ns() || (int)EdgeIdx.size() != ne() ||
        (int)E.size() != 2 * ne())
      throw std::invalid_argument("tnbp_b200 drop-in: one process holds the whole lattice (single-rank layout)");
    bool changed = false;
    for (int m = 0; m < 2 * ne(); ++m) {
      if (e[m].same(E[m])) continue;
      const auto sh = E[m].Shape();
      if (sh.size() != 2 || sh[0] != sh[1]) throw std::invalid_argument("tnbp_b200 drop-in: a message is not D x D");
      ok(tnbp_upload_message(job, m, sh[0], reinterpret_cast<const double*>(E[m].GetRaw())), "tnbp_upload_message");
      e[m].take(E[m]);
      changed = true;
    }
    for (int s = 0; s < ns(); ++s) {
      if (v[s].same(V[s])) continue;
      const auto sh = V[s].Shape();
      ok(tnbp_upload_site(job, s, sh.data(), (int32_t)sh.size(), reinterpret_cast<const double*>(V[s].GetRaw())),
         "tnbp_upload_site");
      v[s].take(V[s]);
      changed = true;
    }
    if (changed) f_valid = false;
  }

  Held download_site(int s) {
    Held h;
    h.shape.assign(16, 0);
    int32_t r = 0;
    ok(tnbp_site_shape(job, s, h.shape.data(), 16, &r), "tnbp_site_shape");
    h.shape.resize(r);
    size_t n = 1;
    for (auto d : h.shape) n *= (size_t)d;
    h.data.resize(n);
    ok(tnbp_download_site(job, s, reinterpret_cast<double*>(h.data.data()), (int64_t)n), "tnbp_download_site");
    return h;
  }
  Held download_message(int m) {
    int32_t D = 0;
    ok(tnbp_download_message(job, m, nullptr, 0, &D), "tnbp_download_message");
    Held h;
    h.shape = {D, D};
    h.data.resize((size_t)D * D);
    ok(tnbp_download_message(job, m, reinterpret_cast<double*>(h.data.data()), (int64_t)D * D, &D),
       "tnbp_download_message");
    return h;
  }
  // the device state becomes the caller's
  void pull(std::vector<Ten>& V, std::vector<Ten>& E) {
    for (int s = 0; s < ns(); ++s) {
      v[s] = download_site(s);
      V[s] = v[s].tensor();
    }
    E.resize(2 * ne());
    for (int m = 0; m < 2 * ne(); ++m) {
      e[m] = download_message(m);
      E[m] = e[m].tensor();
    }
    f_valid = false;
  }

  int edge_index(int a, int b) const {
    for (int k = 0; k < ne(); ++k)
      if ((edges[k].first == a && edges[k].second == b) || (edges[k].first == b && edges[k].second == a)) return k;
    throw std::invalid_argument("tnbp_b200 drop-in: pair is not an edge of the lattice");
  }
};

Mirror& mirror() {
  static Mirror m;
  return m;
}

// site index of a label (SiteIdx holds the sorted labels)
int site_of(const std::vector<int>& SiteIdx, int label) {
  auto it = std::find(SiteIdx.begin(), SiteIdx.end(), label);
  if (it == SiteIdx.end()) throw std::invalid_argument("tnbp_b200 drop-in: site label not in the lattice");
  return (int)(it - SiteIdx.begin());
}

}  // namespace

namespace tnbp {

void AbsorbTPO(tci::gqten_handle&, const std::vector<DropinTensor>& O, const std::vector<std::pair<int, int>>& Edge,
               std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx, const std::map<int, int>&,
               std::vector<DropinTensor>& E, const std::vector<int>& EdgeIdx, MPI_Comm) {
  Mirror& M = mirror();
  M.sync(Edge, V, E, SiteIdx, EdgeIdx);
  if ((int)O.size() != M.ns()) throw std::invalid_argument("tnbp_b200 drop-in: one operator per site expected");
  // TPO layout of the C ABI: the rank of each edge's operator bond, each
  // site's (r_leg0..r_leg{g-1}, d, d') tensor at its offset
  std::vector<int32_t> rank(M.ne(), 1);
  std::vector<int64_t> off(M.ns());
  std::vector<double> data;
  for (int s = 0; s < M.ns(); ++s) {
    const int label = SiteIdx[s];
    std::vector<int> legs;
    for (int k = 0; k < M.ne(); ++k)
      if (Edge[k].first == label || Edge[k].second == label) legs.push_back(k);
    const auto sh = O[s].Shape();
    if (sh.size() != legs.size() + 2) throw std::invalid_argument("tnbp_b200 drop-in: operator rank != degree + 2");
    for (size_t k = 0; k < legs.size(); ++k) rank[legs[k]] = sh[k];
    off[s] = (int64_t)(data.size() / 2);
    const double* raw = reinterpret_cast<const double*>(O[s].GetRaw());
    data.insert(data.end(), raw, raw + 2 * O[s].Size());
  }
  tnbp_tpo* tpo = nullptr;
  ok(tnbp_tpo_create(M.job, rank.data(), off.data(), data.data(), &tpo), "tnbp_tpo_create");
  const int rc = tnbp_absorb_tpo(M.job, tpo);
  tnbp_tpo_destroy(tpo);
  ok(rc, "tnbp_absorb_tpo");
  M.pull(V, E);
}

void BeliefPropagation(tci::gqten_handle&, const std::vector<std::pair<int, int>>& I,
                       const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                       const std::map<int, int>&, const std::vector<std::pair<int, int>>& J,
                       const std::vector<DropinTensor>& E, const std::vector<int>& EdgeIdx, MPI_Comm,
                       std::vector<DropinTensor>& F) {
  Mirror& M = mirror();
  bool reuse = M.f_valid && M.job && I == M.edges && (int)E.size() == 2 * M.ne() && (int)V.size() == M.ns();
  for (int s = 0; reuse && s < M.ns(); ++s) reuse = M.v[s].same(V[s]);
  for (int m = 0; reuse && m < 2 * M.ne(); ++m) reuse = M.f_src_e[m].same(E[m]);
  if (!reuse) {
    M.sync(I, V, E, SiteIdx, EdgeIdx);
    std::vector<Held> src = M.e;
    ok(tnbp_bp_sweep(M.job), "tnbp_bp_sweep");  // the device now holds the new messages
    M.f.resize(2 * M.ne());
    for (int m = 0; m < 2 * M.ne(); ++m) M.f[m] = M.download_message(m);
    M.e = M.f;
    M.f_src_e = std::move(src);
    M.f_valid = true;
  }
  F.resize(2 * EdgeIdx.size());
  for (const auto& p : J) {
    const int k = M.edge_index(p.first, p.second);
    F[k] = M.f[k].tensor();
    F[k + M.ne()] = M.f[k + M.ne()].tensor();
  }
}

void BeliefPropagationCondition(tci::gqten_handle&, const std::vector<std::pair<int, int>>& I,
                                const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                const std::map<int, int>&, const std::vector<DropinTensor>& E,
                                const std::vector<int>& EdgeIdx, MPI_Comm, double& result) {
  Mirror& M = mirror();
  M.sync(I, V, E, SiteIdx, EdgeIdx);
  ok(tnbp_bp_condition(M.job, &result), "tnbp_bp_condition");
}

void Truncation(tci::gqten_handle&, const std::vector<std::pair<int, int>>& I, std::vector<DropinTensor>& V,
                const std::vector<int>& SiteIdx, const std::map<int, int>&, std::vector<DropinTensor>& E,
                const std::vector<int>& EdgeIdx, MPI_Comm, int32_t max_dim, double eps, double,
                std::vector<int32_t>& res_bond_dim, std::vector<double>& res_trunc_err) {
  Mirror& M = mirror();
  M.sync(I, V, E, SiteIdx, EdgeIdx);
  res_bond_dim.assign(M.ne(), 0);
  res_trunc_err.assign(M.ne(), 0.0);
  ok(tnbp_truncate(M.job, max_dim, eps, res_bond_dim.data(), res_trunc_err.data()), "tnbp_truncate");
  M.pull(V, E);
}

std::vector<std::complex<double>> Measure(tci::gqten_handle&, const std::vector<std::pair<int, int>>& I,
                                          const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                          const std::map<int, int>&, const std::vector<DropinTensor>& E,
                                          const std::vector<int> EdgeIdx, MPI_Comm, const std::vector<int>& Site,
                                          const std::vector<DropinTensor>& O) {
  Mirror& M = mirror();
  M.sync(I, V, E, SiteIdx, EdgeIdx);
  const size_t n = Site.size();
  std::vector<cd> out(n);
  if (n == 0) return out;
  if (O.size() != n) throw std::invalid_argument("tnbp_b200 drop-in: one operator per site expected");
  std::vector<int64_t> sites(n);
  std::vector<double> ops;
  for (size_t i = 0; i < n; ++i) {
    sites[i] = site_of(SiteIdx, Site[i]);
    if (O[i].Size() != 4) throw std::invalid_argument("tnbp_b200 drop-in: one-site operators are 2 x 2");
    const double* raw = reinterpret_cast<const double*>(O[i].GetRaw());
    ops.insert(ops.end(), raw, raw + 8);
  }
  ok(tnbp_measure_1site(M.job, (int64_t)n, sites.data(), ops.data(), reinterpret_cast<double*>(out.data())),
     "tnbp_measure_1site");
  return out;
}

std::vector<std::complex<double>> Measure(tci::gqten_handle&, const std::vector<std::pair<int, int>>& I,
                                          const std::vector<DropinTensor>& V, const std::vector<int>& SiteIdx,
                                          const std::map<int, int>&, const std::vector<DropinTensor>& E,
                                          const std::vector<int> EdgeIdx, MPI_Comm,
                                          const std::vector<std::pair<int, int>>& Edge,
                                          const std::vector<DropinTensor>& O) {
  Mirror& M = mirror();
  M.sync(I, V, E, SiteIdx, EdgeIdx);
  const size_t n = Edge.size();
  // one value per pair; at least |I| entries, the length of the reference's
  // result vector (measure.h sizes it by the edge count)
  std::vector<cd> out(std::max(n, I.size()));
  if (n == 0) return out;
  if (O.size() != n) throw std::invalid_argument("tnbp_b200 drop-in: one operator per pair expected");
  std::vector<int32_t> pairs;
  std::vector<double> ops;
  for (size_t i = 0; i < n; ++i) {
    pairs.push_back(Edge[i].first);
    pairs.push_back(Edge[i].second);
    if (O[i].Size() != 16) throw std::invalid_argument("tnbp_b200 drop-in: two-site operators are 2x2x2x2");
    const double* raw = reinterpret_cast<const double*>(O[i].GetRaw());
    ops.insert(ops.end(), raw, raw + 32);
  }
  ok(tnbp_measure_2site(M.job, (int64_t)n, pairs.data(), ops.data(), reinterpret_cast<double*>(out.data())),
     "tnbp_measure_2site");
  return out;
}

}  // namespace tnbp
