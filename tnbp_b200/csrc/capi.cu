// extern "C" entry points of include/tnbp_b200.h.  Every call catches C++
// exceptions at the boundary, records the message for tnbp_last_error() and
// returns the status code; nothing unwinds across the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/tnbp_b200.h"
#include "engine.h"
#include "host_setup.h"
#include "server.h"
#include "tps_io.h"

using tnbp::Error;

struct tnbp_job { std::unique_ptr<tnbp::Job> j; };
struct tnbp_tpo { std::unique_ptr<tnbp::Tpo> t; tnbp::Job* owner; };

namespace {
template <class F>
int guard(F&& f) {
  try {
    tnbp::g_last_error.clear();
    f();
    return TNBP_OK;
  } catch (const tnbp::Error& e) {
    tnbp::g_last_error = e.what();
    return e.code;
  } catch (const tnbp_host::HostError& e) {
    tnbp::g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    tnbp::g_last_error = "host allocation failed";
    return TNBP_ENOMEM;
  } catch (const std::exception& e) {
    tnbp::g_last_error = e.what();
    return TNBP_EINVAL;
  }
}
void need(bool c, const char* m) {
  if (!c) throw Error(TNBP_EINVAL, m);
}
tnbp_host::Edges to_edges(const int32_t* e, int64_t n) {
  need(e != nullptr || n == 0, "edges is NULL");
  tnbp_host::Edges out(n);
  for (int64_t i = 0; i < n; ++i) out[i] = {e[2 * i], e[2 * i + 1]};
  return out;
}
void put_edges(const tnbp_host::Edges& e, int32_t* out, int64_t cap, int64_t* n) {
  if (n) *n = (int64_t)e.size();
  if (out && cap >= (int64_t)e.size())
    for (size_t i = 0; i < e.size(); ++i) { out[2 * i] = e[i].first; out[2 * i + 1] = e[i].second; }
  else if (out && cap > 0) throw Error(TNBP_EINVAL, "output capacity too small");
}
void put_layers(const std::vector<tnbp_host::Layer>& layers, int64_t ne, int64_t ns, int32_t* edge_rank,
                int64_t* op_offset, double* op_data, int64_t cap, int64_t* nelems) {
  int64_t tot = 0;
  for (auto& l : layers) tot += (int64_t)l.op_data.size() / 2;
  if (nelems) *nelems = tot;
  if (cap == 0 || !op_data) return;
  if (cap < tot) throw Error(TNBP_EINVAL, "op_data capacity too small");
  int64_t base = 0;
  for (size_t li = 0; li < layers.size(); ++li) {
    const auto& l = layers[li];
    if (edge_rank) for (int64_t e = 0; e < ne; ++e) edge_rank[li * ne + e] = l.edge_rank[e];
    if (op_offset) for (int64_t s = 0; s < ns; ++s) op_offset[li * ns + s] = base + l.op_offset[s];
    std::memcpy(op_data + 2 * base, l.op_data.data(), l.op_data.size() * sizeof(double));
    base += (int64_t)l.op_data.size() / 2;
  }
}
}  // namespace

extern "C" {

const char* tnbp_last_error(void) { return tnbp::g_last_error.c_str(); }
const char* tnbp_version(void) { return "tnbp_b200 0.1 (sm_100a)"; }
int tnbp_device_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n > 0 ? 1 : 0;
}

int tnbp_square_lattice(int32_t Lx, int32_t Ly, int32_t* edges_out, int64_t cap, int64_t* n) {
  return guard([&] { put_edges(tnbp_host::square_lattice(Lx, Ly), edges_out, cap, n); });
}

int tnbp_greedy_layering(const int32_t* edges, int64_t ne, int32_t* layer_of_edge, int32_t* nl) {
  return guard([&] {
    int L = 0;
    auto l = tnbp_host::greedy_layering(to_edges(edges, ne), &L);
    if (layer_of_edge) for (int64_t i = 0; i < ne; ++i) layer_of_edge[i] = l[i];
    if (nl) *nl = L;
  });
}

int tnbp_surrounding_bonds(const int32_t* edges, int64_t ne, int32_t site, int32_t* out, int32_t cap, int32_t* n) {
  return guard([&] {
    auto b = tnbp_host::surrounding_bonds(to_edges(edges, ne), site);
    if (n) *n = (int32_t)b.size();
    if (out) {
      need(cap >= (int32_t)b.size(), "output capacity too small");
      for (size_t i = 0; i < b.size(); ++i) out[i] = b[i];
    }
  });
}

int tnbp_shortest_path(const int32_t* edges, int64_t ne, int32_t src, int32_t dst, int32_t* out, int32_t cap, int32_t* n) {
  return guard([&] {
    auto p = tnbp_host::shortest_path(to_edges(edges, ne), src, dst);
    if (n) *n = (int32_t)p.size();
    if (out) {
      need(cap >= (int32_t)p.size(), "output capacity too small");
      for (size_t i = 0; i < p.size(); ++i) out[i] = p[i];
    }
  });
}

int tnbp_qasm_edges(const char* src, int32_t* edges_out, int64_t cap, int64_t* n) {
  return guard([&] {
    need(src != nullptr, "qasm source is NULL");
    put_edges(tnbp_host::qasm_edges(tnbp_host::parse_qasm(src)), edges_out, cap, n);
  });
}

int tnbp_qasm_instructions(const char* src, int32_t* op, int32_t* nq, int32_t* qubits, int32_t* np, double* params,
                           int64_t cap, int64_t* n_out) {
  return guard([&] {
    need(src != nullptr, "qasm source is NULL");
    auto p = tnbp_host::parse_qasm(src);
    const int64_t n = (int64_t)p.instructions.size();
    if (n_out) *n_out = n;
    if (cap == 0) return;
    need(cap >= n, "output capacity too small");
    for (int64_t i = 0; i < n; ++i) {
      const auto& in = p.instructions[i];
      if (op) op[i] = (int32_t)in.op;
      if (nq) nq[i] = (int32_t)in.qubits.size();
      if (qubits) for (int k = 0; k < 4; ++k) qubits[4 * i + k] = k < (int)in.qubits.size() ? (int32_t)in.qubits[k].index : -1;
      if (np) np[i] = (int32_t)in.params.size();
      if (params) for (int k = 0; k < 3; ++k) params[3 * i + k] = k < (int)in.params.size() ? in.params[k] : 0.0;
    }
  });
}

int tnbp_pauli_terms(const char* text, const int32_t* edges, int64_t ne, int32_t* kind, int32_t* q0, int32_t* q1,
                     char* letters, double* coeff, int32_t* term_index, int64_t cap, int64_t* n_kept,
                     int64_t* n_dropped) {
  return guard([&] {
    need(text != nullptr, "text is NULL");
    int64_t dropped = 0;
    auto t = tnbp_host::pauli_terms(text, to_edges(edges, ne), &dropped);
    if (n_kept) *n_kept = (int64_t)t.size();
    if (n_dropped) *n_dropped = dropped;
    if (cap == 0) return;
    need(cap >= (int64_t)t.size(), "output capacity too small");
    for (size_t i = 0; i < t.size(); ++i) {
      if (kind) kind[i] = t[i].kind;
      if (q0) q0[i] = t[i].q0;
      if (q1) q1[i] = t[i].q1;
      if (letters) { letters[2 * i] = t[i].l0; letters[2 * i + 1] = t[i].l1 ? t[i].l1 : 'I'; }
      if (coeff) { coeff[2 * i] = t[i].coeff_re; coeff[2 * i + 1] = t[i].coeff_im; }
      if (term_index) term_index[i] = (int32_t)t[i].row;
    }
  });
}

// The size query (cap 0) and the fill call that follows it with the same
// program and edges share one build: the layers of the last call on this
// thread are kept until a call with other inputs.
namespace {
struct LastTpo {
  std::string src;
  std::vector<int32_t> edges;
  std::vector<tnbp_host::Layer> layers;
};
thread_local LastTpo g_last_tpo;
}  // namespace

int tnbp_qasm_tpo(const char* src, const int32_t* edges, int64_t ne, int32_t* edge_rank, int64_t* op_offset,
                  double* op_data, int64_t cap, int32_t* n_layers, int64_t* n_elems) {
  return guard([&] {
    need(src != nullptr, "qasm source is NULL");
    auto e = to_edges(edges, ne);
    std::vector<int32_t> key(edges, edges + 2 * ne);
    if (g_last_tpo.src != src || g_last_tpo.edges != key) {
      g_last_tpo.layers = tnbp_host::qasm_tpo(tnbp_host::parse_qasm(src), e);
      g_last_tpo.src = src;
      g_last_tpo.edges = std::move(key);
    }
    const auto& layers = g_last_tpo.layers;
    if (n_layers) *n_layers = (int32_t)layers.size();
    put_layers(layers, ne, (int64_t)tnbp_host::site_labels(e).size(), edge_rank, op_offset, op_data, cap, n_elems);
  });
}

int tnbp_qasm_tpo_counts(const char* src, const int32_t* edges, int64_t ne, const int32_t* num_gates, int32_t n_counts,
                         int32_t* edge_rank, int64_t* op_offset, double* op_data, int64_t cap, int32_t* n_layers,
                         int64_t* n_elems) {
  return guard([&] {
    need(src != nullptr && (n_counts == 0 || num_gates != nullptr), "NULL argument");
    auto e = to_edges(edges, ne);
    auto layers = tnbp_host::qasm_tpo_counts(tnbp_host::parse_qasm(src), e,
                                             std::vector<int>(num_gates, num_gates + n_counts));
    if (n_layers) *n_layers = (int32_t)layers.size();
    put_layers(layers, ne, (int64_t)tnbp_host::site_labels(e).size(), edge_rank, op_offset, op_data, cap, n_elems);
  });
}

int tnbp_kicked_ising_tpo(const int32_t* edges, int64_t ne, double Jz, double hz, double hx, double dt,
                          int32_t* edge_rank, int64_t* op_offset, double* op_data, int64_t cap, int64_t* n_elems) {
  return guard([&] {
    auto e = to_edges(edges, ne);
    std::vector<tnbp_host::Layer> layers{tnbp_host::kicked_ising_tpo(e, Jz, hz, hx, dt)};
    put_layers(layers, ne, (int64_t)tnbp_host::site_labels(e).size(), edge_rank, op_offset, op_data, cap, n_elems);
  });
}

int tnbp_opt_tpo_svd(const int32_t* edges, int64_t ne, double eps, int32_t* edge_rank, int64_t* op_offset,
                     double* op_data, int64_t* n_elems) {
  return guard([&] {
    need(edge_rank != nullptr && op_offset != nullptr && op_data != nullptr, "NULL argument");
    auto e = to_edges(edges, ne);
    const auto bonds_of = [&](int site) { return tnbp_host::surrounding_bonds(e, site); };
    const auto sites = tnbp_host::site_labels(e);
    const int64_t ns = (int64_t)sites.size();
    tnbp_host::Layer L;
    L.edge_rank.assign(edge_rank, edge_rank + ne);
    L.op_offset.assign(op_offset, op_offset + ns);
    int64_t extent = 0;  // elements the input layer spans from op_data[0]
    for (int64_t s = 0; s < ns; ++s) {
      int64_t n = 4;
      for (int m : bonds_of(sites[s])) {
        need(edge_rank[m] >= 1, "edge_rank < 1");
        n *= edge_rank[m];
      }
      need(op_offset[s] >= 0, "op_offset < 0");
      extent = std::max(extent, op_offset[s] + n);
    }
    L.op_data.assign(op_data, op_data + 2 * extent);
    tnbp_host::opt_tpo_svd(e, L, eps);
    // bond dimensions never grow, so a layer packed without overlaps fits
    const int64_t tot = (int64_t)L.op_data.size() / 2;
    need(tot <= extent, "op_data too small for the repacked layer (overlapping site operators)");
    std::copy(L.edge_rank.begin(), L.edge_rank.end(), edge_rank);
    std::copy(L.op_offset.begin(), L.op_offset.end(), op_offset);
    std::memcpy(op_data, L.op_data.data(), L.op_data.size() * sizeof(double));
    if (n_elems) *n_elems = tot;
  });
}

// ----------------------------------------------------------- checkpoints
int tnbp_tps_write(const char* path, const int32_t* edges, int64_t ne, const int32_t* bond_dim,
                   const int32_t* phys_dims, const double* site_data, const double* msg_data) {
  return guard([&] {
    need(path && bond_dim && site_data && msg_data, "NULL argument");
    auto e = to_edges(edges, ne);
    const size_t ns = tnbp_host::site_labels(e).size();
    std::vector<int> bd(bond_dim, bond_dim + ne), pd(ns, 2);
    if (phys_dims) pd.assign(phys_dims, phys_dims + ns);
    for (int d : bd) need(d >= 1, "bond dimension < 1");
    for (int d : pd) need(d >= 1, "physical dimension < 1");
    tnbp_host::tps_write(path, tnbp_host::tps_whole(e, bd, pd, reinterpret_cast<const std::complex<double>*>(site_data),
                                                    reinterpret_cast<const std::complex<double>*>(msg_data)));
  });
}

int tnbp_tps_read(const char* path, const int32_t* edges, int64_t ne, int32_t* bond_dim, int32_t* phys_dims,
                  double* site_data, int64_t site_cap, double* msg_data, int64_t msg_cap, int64_t* site_elems,
                  int64_t* msg_elems) {
  return guard([&] {
    need(path != nullptr, "path is NULL");
    auto e = to_edges(edges, ne);
    const auto st = tnbp_host::tps_read(path);
    std::vector<int> bd, pd;
    tnbp_host::tps_check_whole(st, e, bd, pd);
    int64_t nv = 0, nm = 0;
    for (const auto& t : st.V) nv += (int64_t)t.data.size();
    for (const auto& t : st.E) nm += (int64_t)t.data.size();
    if (site_elems) *site_elems = nv;
    if (msg_elems) *msg_elems = nm;
    if (bond_dim) std::copy(bd.begin(), bd.end(), bond_dim);
    if (phys_dims) std::copy(pd.begin(), pd.end(), phys_dims);
    if (site_data) {
      need(site_cap >= nv, "site_data capacity too small");
      int64_t o = 0;
      for (const auto& t : st.V) {
        std::memcpy(site_data + 2 * o, t.data.data(), t.data.size() * 16);
        o += (int64_t)t.data.size();
      }
    }
    if (msg_data) {
      need(msg_cap >= nm, "msg_data capacity too small");
      int64_t o = 0;
      for (const auto& t : st.E) {
        std::memcpy(msg_data + 2 * o, t.data.data(), t.data.size() * 16);
        o += (int64_t)t.data.size();
      }
    }
  });
}

int tnbp_save_state(tnbp_job* job, const char* path) {
  return guard([&] {
    need(job && path, "NULL argument");
    auto& J = *job->j;
    const size_t ns = J.g.labels.size(), ne = J.g.edges.size();
    std::vector<double> hv(2 * J.v_elems), hm(2 * J.m_elems);
    J.get_complex(J.V, hv.data(), J.v_elems, 0);
    J.get_complex(J.M[J.cur], hm.data(), J.m_elems, 0);
    std::vector<double> sv, mv;
    for (size_t s = 0; s < ns; ++s)
      sv.insert(sv.end(), hv.begin() + 2 * J.voff[s], hv.begin() + 2 * (J.voff[s] + J.site_elems((int)s)));
    for (size_t m = 0; m < 2 * ne; ++m) {
      const size_t dd = (size_t)J.dim[m % ne] * J.dim[m % ne];
      mv.insert(mv.end(), hm.begin() + 2 * J.moff[m], hm.begin() + 2 * (J.moff[m] + dd));
    }
    tnbp_host::tps_write(path, tnbp_host::tps_whole(J.g.edges, J.dim, J.pd,
                                                    reinterpret_cast<const std::complex<double>*>(sv.data()),
                                                    reinterpret_cast<const std::complex<double>*>(mv.data())));
  });
}

int tnbp_load_state(tnbp_job* job, const char* path) {
  return guard([&] {
    need(job && path, "NULL argument");
    auto& J = *job->j;
    const auto st = tnbp_host::tps_read(path);
    std::vector<int> bd, pd;
    tnbp_host::tps_check_whole(st, J.g.edges, bd, pd);
    need(pd == J.pd, "checkpoint physical dimensions differ from the job's");
    // New layout and buffers are built beside the job's own and swapped in
    // only after every check and allocation succeeded, so a refused or
    // failed load leaves the job's state as it was.
    const std::vector<int> old_dim = J.dim;
    const std::vector<size_t> old_voff = J.voff, old_moff = J.moff;
    const size_t old_v = J.v_elems, old_m = J.m_elems;
    J.dim = bd;
    J.layout();
    auto restore = [&] {
      J.dim = old_dim; J.voff = old_voff; J.moff = old_moff; J.v_elems = old_v; J.m_elems = old_m;
    };
    tnbp::DevBuf nV, nM0, nM1;
    try {
      const uint64_t extra = (uint64_t)(J.v_elems + 2 * J.m_elems) * J.esz;
      const uint64_t held = J.V.bytes + J.M[0].bytes + J.M[1].bytes;
      if (J.budget && J.device_bytes() - held + extra > J.budget)
        throw tnbp::Error(TNBP_ENOMEM, "checkpoint needs " + std::to_string(J.device_bytes() - held + extra) +
                                           " device bytes, budget " + std::to_string(J.budget));
      nV.alloc(J.v_elems * J.esz, J.stream);
      nM0.alloc(J.m_elems * J.esz, J.stream);
      nM1.alloc(J.m_elems * J.esz, J.stream);
    } catch (...) {
      restore();
      throw;
    }
    std::swap(J.V, nV);
    std::swap(J.M[0], nM0);
    std::swap(J.M[1], nM1);
    std::vector<double> hv(2 * J.v_elems, 0.0), hm(2 * J.m_elems, 0.0);
    for (size_t s = 0; s < st.V.size(); ++s)
      std::memcpy(hv.data() + 2 * J.voff[s], st.V[s].data.data(), st.V[s].data.size() * 16);
    for (size_t m = 0; m < st.E.size(); ++m)
      std::memcpy(hm.data() + 2 * J.moff[m], st.E[m].data.data(), st.E[m].data.size() * 16);
    J.put_complex(J.V, hv.data(), J.v_elems, 0);
    J.put_complex(J.M[0], hm.data(), J.m_elems, 0);
    J.cur = 0;
    J.shadow_dirty = true;
    J.destroy_graphs();
    J.plan = tnbp::SweepPlan();
  });
}

// ------------------------------------------------------------------ jobs
int tnbp_job_create(const int32_t* edges, int64_t ne, const int32_t* pdims, int32_t precision, void* stream,
                    uint64_t budget, tnbp_job** out) {
  return guard([&] {
    need(out != nullptr, "out is NULL");
    *out = nullptr;
    auto j = std::make_unique<tnbp_job>();
    j->j = std::make_unique<tnbp::Job>(edges, ne, pdims, precision, static_cast<cudaStream_t>(stream), budget);
    *out = j.release();
  });
}

int tnbp_job_destroy(tnbp_job* job) {
  return guard([&] { delete job; });
}

int tnbp_job_info(const tnbp_job* job, int64_t* ns, int64_t* ne, int32_t* prec) {
  return guard([&] {
    need(job, "job is NULL");
    if (ns) *ns = (int64_t)job->j->g.labels.size();
    if (ne) *ne = (int64_t)job->j->g.edges.size();
    if (prec) *prec = job->j->prec;
  });
}

int tnbp_job_device_bytes(const tnbp_job* job, uint64_t* bytes) {
  return guard([&] { need(job && bytes, "NULL argument"); *bytes = job->j->device_bytes(); });
}

int tnbp_bond_dims(const tnbp_job* job, int32_t* dims) {
  return guard([&] {
    need(job && dims, "NULL argument");
    for (size_t e = 0; e < job->j->dim.size(); ++e) dims[e] = job->j->dim[e];
  });
}

int tnbp_site_shape(const tnbp_job* job, int64_t site, int32_t* shape, int32_t cap, int32_t* rank) {
  return guard([&] {
    need(job, "job is NULL");
    need(site >= 0 && site < (int64_t)job->j->g.labels.size(), "site index out of range");
    auto sh = job->j->site_shape((int)site);
    if (rank) *rank = (int32_t)sh.size();
    if (shape) {
      need(cap >= (int32_t)sh.size(), "shape capacity too small");
      for (size_t k = 0; k < sh.size(); ++k) shape[k] = sh[k];
    }
  });
}

int tnbp_download_site(tnbp_job* job, int64_t site, double* data, int64_t cap) {
  return guard([&] {
    need(job && data, "NULL argument");
    need(site >= 0 && site < (int64_t)job->j->g.labels.size(), "site index out of range");
    const size_t n = job->j->site_elems((int)site);
    need(cap >= (int64_t)n, "capacity too small");
    job->j->get_complex(job->j->V, data, n, job->j->voff[site]);
  });
}

int tnbp_upload_site(tnbp_job* job, int64_t site, const int32_t* shape, int32_t rank, const double* data) {
  return guard([&] {
    need(job && shape && data, "NULL argument");
    auto& J = *job->j;
    need(site >= 0 && site < (int64_t)J.g.labels.size(), "site index out of range");
    auto sh = J.site_shape((int)site);
    need(rank == (int32_t)sh.size(), "rank does not match the site's degree + 1");
    for (size_t k = 0; k < sh.size(); ++k)
      need(shape[k] == sh[k], "shape does not match the current bond dimensions (upload messages first?)");
    J.put_complex(J.V, data, J.site_elems((int)site), J.voff[site]);
  });
}

int tnbp_download_message(tnbp_job* job, int64_t m, double* data, int64_t cap, int32_t* dim_out) {
  return guard([&] {
    need(job, "job is NULL");
    auto& J = *job->j;
    const int64_t ne = (int64_t)J.g.edges.size();
    need(m >= 0 && m < 2 * ne, "message index out of range");
    const int D = J.dim[m % ne];
    if (dim_out) *dim_out = D;
    if (!data) return;
    need(cap >= (int64_t)D * D, "capacity too small");
    J.get_complex(J.M[J.cur], data, (size_t)D * D, J.moff[m]);
  });
}

int tnbp_upload_message(tnbp_job* job, int64_t m, int32_t dim, const double* data) {
  return guard([&] {
    need(job && data, "NULL argument");
    auto& J = *job->j;
    const int64_t ne = (int64_t)J.g.edges.size();
    need(m >= 0 && m < 2 * ne, "message index out of range");
    if (dim != J.dim[m % ne]) {
      // a new bond dimension: re-layout (site tensors of both endpoints are
      // left stale until they are uploaded with matching shapes)
      std::vector<double> keepM(2 * J.m_elems);
      J.get_complex(J.M[J.cur], keepM.data(), J.m_elems, 0);
      std::vector<double> keepV(2 * J.v_elems);
      J.get_complex(J.V, keepV.data(), J.v_elems, 0);
      const auto odim = J.dim;
      const auto omoff = J.moff;
      const auto ovoff = J.voff;
      std::vector<size_t> oelems(J.g.labels.size());
      for (size_t s = 0; s < oelems.size(); ++s) oelems[s] = J.site_elems((int)s);
      J.dim[m % ne] = dim;
      J.layout();
      J.V.alloc(J.v_elems * J.esz, J.stream);
      J.shadow_dirty = true;
      J.M[0].alloc(J.m_elems * J.esz, J.stream);
      J.M[1].alloc(J.m_elems * J.esz, J.stream);
      for (size_t s = 0; s < oelems.size(); ++s)
        if (J.site_elems((int)s) == oelems[s]) J.put_complex(J.V, keepV.data() + 2 * ovoff[s], oelems[s], J.voff[s]);
      for (int64_t k = 0; k < 2 * ne; ++k)
        if (J.dim[k % ne] == odim[k % ne])
          J.put_complex(J.M[0], keepM.data() + 2 * omoff[k], (size_t)odim[k % ne] * odim[k % ne], J.moff[k]);
      J.cur = 0;
      J.destroy_graphs();
      J.plan = tnbp::SweepPlan();
    }
    J.put_complex(J.M[J.cur], data, (size_t)dim * dim, J.moff[m]);
  });
}

int tnbp_tpo_create(tnbp_job* job, const int32_t* edge_rank, const int64_t* op_offset, const double* op_data,
                    tnbp_tpo** out) {
  return guard([&] {
    need(job && edge_rank && op_offset && op_data && out, "NULL argument");
    auto& J = *job->j;
    const int ns = (int)J.g.labels.size(), ne = (int)J.g.edges.size();
    auto t = std::make_unique<tnbp::Tpo>();
    t->rank.assign(edge_rank, edge_rank + ne);
    for (int r : t->rank) need(r >= 1, "TPO bond rank must be >= 1");
    t->op_offset.assign(op_offset, op_offset + ns);
    t->dout.resize(ns);
    int64_t total = 0;
    for (int s = 0; s < ns; ++s) {
      int64_t n = 1;
      for (int e : J.g.legs[s]) n *= t->rank[e];
      n *= (int64_t)J.pd[s] * J.pd[s];
      t->dout[s] = J.pd[s];
      total = std::max(total, t->op_offset[s] + n);
    }
    for (int64_t i = 0; i < 2 * total; ++i) need(std::isfinite(op_data[i]), "non-finite TPO element");
    t->ops.alloc((size_t)total * sizeof(double2), J.stream);
    CK(cudaMemcpyAsync(t->ops.p, op_data, (size_t)total * sizeof(double2), cudaMemcpyHostToDevice, J.stream));
    CK(cudaStreamSynchronize(J.stream));
    auto h = std::make_unique<tnbp_tpo>();
    h->t = std::move(t);
    h->owner = job->j.get();
    *out = h.release();
  });
}

int tnbp_tpo_destroy(tnbp_tpo* tpo) { return guard([&] { delete tpo; }); }

int tnbp_absorb_tpo(tnbp_job* job, const tnbp_tpo* tpo) {
  return guard([&] {
    need(job && tpo, "NULL argument");
    need(tpo->owner == job->j.get(), "TPO was created for another job");
    job->j->absorb_tpo(*tpo->t);
  });
}

int tnbp_bp_sweep(tnbp_job* job) { return guard([&] { need(job, "job is NULL"); job->j->bp_sweep(); }); }

int tnbp_bp_condition(tnbp_job* job, double* result) {
  return guard([&] {
    need(job && result, "NULL argument");
    *result = job->j->bp_condition();
  });
}

int tnbp_bp_run(tnbp_job* job, double tol, int32_t max_iter, int32_t* iters, double* cond) {
  return guard([&] {
    need(job, "job is NULL");
    int it = 0;
    double c = 0;
    job->j->bp_run(tol, max_iter, &it, &c);
    if (iters) *iters = it;
    if (cond) *cond = c;
  });
}

int tnbp_truncate(tnbp_job* job, int32_t chi_max, double sv_min, int32_t* dims, double* errs) {
  return guard([&] {
    need(job, "job is NULL");
    job->j->truncate(chi_max, sv_min, dims, errs);
  });
}

int tnbp_measure_1site(tnbp_job* job, int64_t n, const int64_t* sites, const double* ops, double* out) {
  return guard([&] {
    need(job && (n == 0 || (sites && ops && out)), "NULL argument");
    auto& J = *job->j;
    std::vector<tnbp::TermSpec> terms(n);
    for (int64_t i = 0; i < n; ++i) {
      need(sites[i] >= 0 && sites[i] < (int64_t)J.g.labels.size(), "site index out of range");
      need(J.pd[sites[i]] == 2, "one-site operators are 2x2");
      auto& t = terms[i];
      std::memset(&t, 0, sizeof(t));
      t.kind = 1;
      t.site_a = (int)sites[i];
      std::memcpy(t.op, ops + 8 * i, 8 * sizeof(double));
    }
    J.measure_terms(terms, out, nullptr);
  });
}

int tnbp_measure_2site(tnbp_job* job, int64_t n, const int32_t* pairs, const double* ops, double* out) {
  return guard([&] {
    need(job && (n == 0 || (pairs && ops && out)), "NULL argument");
    auto& J = *job->j;
    std::vector<tnbp::TermSpec> terms(n);
    for (int64_t i = 0; i < n; ++i) {
      auto& t = terms[i];
      std::memset(&t, 0, sizeof(t));
      t.kind = 2;
      t.edge = J.edge_of(pairs[2 * i], pairs[2 * i + 1]);
      need(t.edge >= 0, "pair is not an edge of the lattice");
      t.label_a = pairs[2 * i];
      std::memcpy(t.op, ops + 32 * i, 32 * sizeof(double));
    }
    J.measure_terms(terms, out, nullptr);
  });
}

}  // extern "C"

namespace {
// One kept term of ClassifyOps as the device measurement takes it.
tnbp::TermSpec term_spec(const tnbp::Job& J, int kind, int q0, int q1, char l0, char l1, double cre, double cim) {
  tnbp::TermSpec t;
  std::memset(&t, 0, sizeof(t));
  t.kind = kind;
  t.coeff[0] = cre;
  t.coeff[1] = cim;
  if (kind == 1) {
    auto it = J.g.index_of.find(q0);
    need(it != J.g.index_of.end(), "one-site term on a qubit outside the lattice");
    t.site_a = it->second;
    auto P = tnbp_host::pauli_list(l0);
    for (int k = 0; k < 4; ++k) { t.op[2 * k] = P[k].real(); t.op[2 * k + 1] = P[k].imag(); }
  } else if (kind == 2) {
    t.edge = J.edge_of(q0, q1);
    need(t.edge >= 0, "two-site term on a non-adjacent pair");
    t.label_a = q0;
    auto Pa = tnbp_host::pauli_list(l0);
    auto Pb = tnbp_host::pauli_list(l1);
    // O[i0, i1, i2, i3] = Pa[i0, i2] Pb[i1, i3]  (paulitotpo.h:73-91)
    for (int i0 = 0; i0 < 2; ++i0)
      for (int i1 = 0; i1 < 2; ++i1)
        for (int i2 = 0; i2 < 2; ++i2)
          for (int i3 = 0; i3 < 2; ++i3) {
            const auto v = Pa[i0 + 2 * i2] * Pb[i1 + 2 * i3];
            const int idx = i0 + 2 * i1 + 4 * i2 + 8 * i3;
            t.op[2 * idx] = v.real();
            t.op[2 * idx + 1] = v.imag();
          }
  } else {
    throw Error(TNBP_EINVAL, "term kind must be 1 or 2");
  }
  return t;
}
}  // namespace

extern "C" {

int tnbp_measure_pauli_sum(tnbp_job* job, int64_t n, const int32_t* kind, const int32_t* q0, const int32_t* q1,
                           const char* letters, const double* coeff, double* per_term, double* sum) {
  return guard([&] {
    need(job && (n == 0 || (kind && q0 && q1 && letters && coeff)), "NULL argument");
    auto& J = *job->j;
    std::vector<tnbp::TermSpec> terms;
    for (int64_t i = 0; i < n; ++i)
      terms.push_back(term_spec(J, kind[i], q0[i], q1[i], letters[2 * i], letters[2 * i + 1], coeff[2 * i],
                                coeff[2 * i + 1]));
    J.measure_terms(terms, per_term, sum);
  });
}

int tnbp_measure_cluster(tnbp_job* job, int64_t n, const int32_t* n_qubits, const int32_t* qubits,
                         const char* letters, const double* coeff, double* values, double* sum) {
  return guard([&] {
    need(job && (n == 0 || (n_qubits && qubits && letters && coeff)), "NULL argument");
    std::vector<tnbp::ClusterTerm> terms(n);
    int64_t o = 0;
    for (int64_t i = 0; i < n; ++i) {
      need(n_qubits[i] >= 2 && n_qubits[i] <= 64, "a cluster term has 2 to 64 qubits");
      terms[i].labels.assign(qubits + o, qubits + o + n_qubits[i]);
      for (int k = 0; k < n_qubits[i]; ++k) terms[i].letters.push_back((char)std::toupper((unsigned char)letters[o + k]));
      terms[i].coeff[0] = coeff[2 * i];
      terms[i].coeff[1] = coeff[2 * i + 1];
      o += n_qubits[i];
    }
    job->j->measure_clusters(terms, values, sum);
  });
}

int tnbp_measure_pauli_text(tnbp_job* job, const char* text, int32_t clusters, double* values, int32_t* kinds,
                            int64_t cap, int64_t* n_rows, double* sum) {
  return guard([&] {
    need(job && text, "NULL argument");
    auto& J = *job->j;
    const auto rows = tnbp_host::pauli_strings(text, J.g.edges);
    const int64_t n = (int64_t)rows.size();
    if (n_rows) *n_rows = n;
    if (!values && !kinds && !sum) return;  // sizing call
    need(!(values || kinds) || cap >= n, "output capacity too small");
    std::vector<tnbp::TermSpec> kept;
    std::vector<int64_t> kept_row;
    std::vector<tnbp::ClusterTerm> cl;
    std::vector<int64_t> cl_row;
    std::vector<double> out(2 * std::max<int64_t>(n, 1), std::nan(""));
    double sr = 0.0, si = 0.0;  // identity terms
    for (int64_t r = 0; r < n; ++r) {
      const auto& t = rows[r];
      if (kinds) kinds[r] = t.kind;
      if (t.kind == 0) {
        out[2 * r] = 1.0;
        out[2 * r + 1] = 0.0;
        if (clusters) { sr += t.coeff_re; si += t.coeff_im; }
      } else if (t.kind == 1 || t.kind == 2) {
        kept.push_back(term_spec(J, t.kind, t.qubits[0], t.kind == 2 ? t.qubits[1] : -1, t.letters[0],
                                 t.kind == 2 ? t.letters[1] : 'I', t.coeff_re, t.coeff_im));
        kept_row.push_back(r);
      } else if (clusters) {
        tnbp::ClusterTerm c;
        c.labels = t.qubits;
        c.letters.assign(t.letters.begin(), t.letters.end());
        c.coeff[0] = t.coeff_re;
        c.coeff[1] = t.coeff_im;
        cl.push_back(c);
        cl_row.push_back(r);
      }
    }
    std::vector<double> kv(2 * std::max<size_t>(kept.size(), 1)), cv(2 * std::max<size_t>(cl.size(), 1));
    double ks[2] = {0.0, 0.0}, cs[2] = {0.0, 0.0};
    if (!kept.empty()) J.measure_terms(kept, kv.data(), ks);
    if (!cl.empty()) J.measure_clusters(cl, cv.data(), cs);
    for (size_t k = 0; k < kept.size(); ++k) { out[2 * kept_row[k]] = kv[2 * k]; out[2 * kept_row[k] + 1] = kv[2 * k + 1]; }
    for (size_t k = 0; k < cl.size(); ++k) { out[2 * cl_row[k]] = cv[2 * k]; out[2 * cl_row[k] + 1] = cv[2 * k + 1]; }
    if (values) std::memcpy(values, out.data(), 2 * n * sizeof(double));
    if (sum) { sum[0] = ks[0] + cs[0] + sr; sum[1] = ks[1] + cs[1] + si; }
  });
}

unsigned long long tnbp_kernel_launches(void) { return tnbp::g_launches.load(); }

int tnbp_sweep_totals(const tnbp_job* job, double* total_ms, double* total_flops, double* total_bytes,
                      int64_t* n_sweeps) {
  return guard([&] {
    need(job, "job is NULL");
    if (total_ms) *total_ms = job->j->total_sweep_ms;
    if (total_flops) *total_flops = job->j->total_sweep_flops;
    if (total_bytes) *total_bytes = job->j->total_sweep_bytes;
    if (n_sweeps) *n_sweeps = job->j->timed_sweeps;
  });
}

int tnbp_sweep_stats(const tnbp_job* job, double* ms, double* flops, double* bytes) {
  return guard([&] {
    need(job, "job is NULL");
    if (ms) *ms = job->j->last_sweep_ms;
    if (flops) *flops = job->j->plan.flops;
    if (bytes) *bytes = job->j->plan.bytes_alg;
  });
}

}  // extern "C"
