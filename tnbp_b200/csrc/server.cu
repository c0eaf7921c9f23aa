// Continuous-batching request loop (the served estimator path).
//
// Requests wait in a FIFO queue and are admitted while their estimated peak
// HBM footprint fits the budget and a slot is free.  Each admitted request
// owns a device-resident Job (site tensors, messages, sweep plan) for its
// whole life.  Every server step:
//   1. admits queued requests;
//   2. absorbs the next TPO layer for requests entering a Floquet step;
//   3. runs ONE batched BP sweep over all requests in their BP phase: the
//      leg-contraction, Gram and message kernels each take the concatenated
//      task lists of every such job (uneven lattices and bond dimensions share
//      each launch), with one condition per job;
//   4. truncates requests whose BP loop ended, and measures finished ones.
// Requests that arrive while others are on the GPU join at the next step, so
// their sweeps overlap with the sweeps already in flight.  The BP stopping
// rule per job is the one of Job::bp_run (the apps' loop), so a request's
// result does not depend on what it was batched with.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/tnbp_b200.h"
#include "host_setup.h"
#include "server.h"
#include "trace.h"

namespace tnbp {

Server::Server(int precision, uint64_t budget_bytes, int max_active_jobs)
    : prec(precision), budget(budget_bytes), max_active(max_active_jobs) {
  if (precision != TNBP_C128 && precision != TNBP_C64 && precision != TNBP_MIXED)
    throw Error(TNBP_EINVAL, "unknown precision");
  if (max_active < 1) throw Error(TNBP_EINVAL, "max_active must be >= 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw Error(TNBP_ENOGPU, "no CUDA device visible: the B200 engine has no CPU path");
  }
  keep_pool_memory();
  CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  if (budget == 0) {
    const size_t fr = device_bytes_available();
    const size_t reserve = (size_t)4 << 30;
    budget = fr > 2 * reserve ? fr - reserve : fr / 2;
  }
}

Server::~Server() {
  sweeps.clear();
  for (auto& kv : reqs) { kv.second->job.reset(); kv.second->tpos.reset(); }
  tpo_cache.clear();
  for (auto& h : hconds)
    if (h.p) cudaFreeHost(h.p);
  if (stream2) { cudaStreamSynchronize(stream2); cudaStreamDestroy(stream2); }
  if (stream) { cudaStreamSynchronize(stream); cudaStreamDestroy(stream); }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
}

// Sweep scratch slots of a degree-g site under the tree schedule of
// Job::build_plan: S(1) = 0, S(n) = n + S(n/2) + S(n - n/2).
static int sweep_slots(int g) {
  if (g <= 1) return 0;
  const int h = g / 2;
  return g + sweep_slots(h) + sweep_slots(g - h);
}

// Peak device bytes of a job on `edges` whose BP runs at bond dimension
// D[e] on edge e (physical dimension 2): per site the tensor, its spare
// buffer and the complex64 sweep copy (TNBP_MIXED); the two chain buffers of
// truncation and measurement (at most the chain cap each); the sweep scratch
// slots of the largest wave; both message arenas twice; per-edge truncation
// work and Gram partials; plus extra_bytes; 10 % and 8 MiB of margin.
uint64_t footprint_estimate(const std::vector<std::pair<int, int>>& edges, const std::vector<double>& D, int prec,
                            uint64_t extra_bytes) {
  const double esz = prec == TNBP_C64 ? 8.0 : 16.0;   // stored element
  const double wsz = prec == TNBP_C128 ? 16.0 : 8.0;  // sweep element
  const double shadow = prec == TNBP_MIXED ? 8.0 : 0.0;
  const size_t ne = edges.size();
  const auto sites = tnbp_host::site_labels(edges);
  std::map<int, size_t> pos;
  for (size_t i = 0; i < sites.size(); ++i) pos[sites[i]] = i;
  std::vector<double> n(sites.size(), 2.0);  // elements of each site tensor
  std::vector<int> deg(sites.size(), 0);
  for (size_t e = 0; e < ne; ++e)
    for (int v : {edges[e].first, edges[e].second}) {
      n[pos[v]] *= D[e];
      ++deg[pos[v]];
    }
  double bytes = 0.0, slots_all = 0.0, unit_max = 0.0, chain_all = 0.0;
  for (size_t i = 0; i < sites.size(); ++i) {
    bytes += n[i] * (2.0 * esz + shadow);  // V, spare, sweep copy
    chain_all += n[i] * esz;
    slots_all += n[i] * wsz * sweep_slots(deg[i]);
    unit_max = std::max(unit_max, n[i] * wsz * std::max(1, deg[i]));
  }
  bytes += 2.0 * std::min(chain_all, (double)chain_cap_bytes());
  // sweep scratch: one wave's units at a time (a wave stays within the wave
  // budget, at most the scratch cap, unless it is a single unit)
  const double cap = (double)scratch_cap_bytes();
  double wave = (double)wave_budget_bytes();
  if (wave <= 0.0 || wave > cap) wave = cap;
  bytes += std::min(slots_all, std::max(wave, unit_max));
  for (size_t e = 0; e < ne; ++e) {
    const double dd = D[e] * D[e];
    bytes += 4.0 * 2.0 * dd * esz;   // message arenas (old + new)
    bytes += 8.0 * dd * 16.0;        // truncation work
    bytes += 2.0 * 16.0 * dd * 16.0; // Gram partials (upper bound)
  }
  bytes += (double)extra_bytes;
  return (uint64_t)(bytes * 1.1) + (8ull << 20);
}

// Peak device bytes of a request.  Bond dimension during BP on edge e: at
// most chi times the largest TPO rank on e, and at most the product of the
// ranks absorbed since |0...0>; plus the request's TPO layers.
uint64_t Server::footprint(const Request& r) const {
  const TpoSet& ts = *r.tpos;
  const auto& edges = ts.edges;
  const size_t ne = edges.size();
  const int nsteps = r.source == Request::QASM ? (int)ts.layers.size() : r.steps;
  std::vector<double> D(ne);
  for (size_t e = 0; e < ne; ++e) {
    const double cap = (double)r.chi * ts.rank_max[e];
    double prod = 1.0;
    for (int t = 0; t < nsteps && prod < cap; ++t)
      prod *= ts.layers[r.source == Request::QASM ? t : 0]->rank[e];
    D[e] = std::max(1.0, std::min(cap, prod));
  }
  return footprint_estimate(edges, D, r.prec, ts.device_bytes);
}

// The TPO layers of a circuit, built and uploaded on the first request that
// names it and shared with every later one while it stays in the cache.
std::shared_ptr<const TpoSet> Server::tpo_set(
    const std::string& key,
    const std::function<void(tnbp_host::Edges&, std::vector<tnbp_host::Layer>&)>& build) {
  auto it = tpo_cache.find(key);
  if (it != tpo_cache.end()) {
    ++cache_hits;
    tpo_lru.remove(key);
    tpo_lru.push_back(key);
    return it->second;
  }
  ++cache_misses;
  TNBP_TRACE_SCOPE("server.tpo_build");
  auto ts = std::make_shared<TpoSet>();
  std::vector<tnbp_host::Layer> layers;
  build(ts->edges, layers);
  if (ts->edges.empty()) throw Error(TNBP_EINVAL, "the circuit has no two-qubit gate (no edges)");
  const size_t ne = ts->edges.size(), ns = tnbp_host::site_labels(ts->edges).size();
  ts->rank_max.assign(ne, 1);
  for (const auto& L : layers) {
    auto t = std::make_unique<Tpo>();
    t->rank.assign(L.edge_rank.begin(), L.edge_rank.end());
    for (size_t e = 0; e < ne; ++e) ts->rank_max[e] = std::max(ts->rank_max[e], t->rank[e]);
    t->op_offset = L.op_offset;
    t->dout.assign(ns, 2);
    t->ops.alloc(L.op_data.size() * sizeof(double), stream);
    CK(cudaMemcpyAsync(t->ops.p, L.op_data.data(), L.op_data.size() * sizeof(double), cudaMemcpyHostToDevice,
                       stream));
    ts->device_bytes += L.op_data.size() * sizeof(double);
    ts->layers.push_back(std::move(t));
  }
  CK(cudaStreamSynchronize(stream));
  tpo_cache[key] = ts;
  tpo_lru.push_back(key);
  while (tpo_cache.size() > tpo_cache_cap) {
    tpo_cache.erase(tpo_lru.front());
    tpo_lru.pop_front();
  }
  return ts;
}

int64_t Server::submit(std::unique_ptr<Request> r) {
  if (!r->tpos) throw Error(TNBP_EINVAL, "request without TPO layers");
  if (r->source == Request::KICKED_ISING && r->L < 2) throw Error(TNBP_EINVAL, "lattice side must be >= 2");
  if (r->chi < 1 || r->steps < 0 || r->maxit < 0) throw Error(TNBP_EINVAL, "bad request parameters");
  r->prec = prec;
  r->footprint = footprint(*r);
  if (r->footprint > budget) throw Error(TNBP_ENOMEM, "request footprint exceeds the server's HBM budget");
  r->id = next_id++;
  const int64_t id = r->id;
  queue.push_back(id);
  reqs[id] = std::move(r);
  return id;
}

void Server::start(Request& r) {
  const auto& edges = r.tpos->edges;
  std::vector<int32_t> e(2 * edges.size());
  for (size_t i = 0; i < edges.size(); ++i) { e[2 * i] = edges[i].first; e[2 * i + 1] = edges[i].second; }
  r.job = std::make_unique<Job>(e.data(), (int64_t)edges.size(), nullptr, r.prec, stream, 0);
  r.job->scratch_cap = scratch_cap_bytes();  // the footprint estimate counts this cap
  r.step = 0;
  r.bp_converged = true;
  r.unconv_loops = 0;
  r.worst_final_cond = 0;
  r.worst_min_cond = 0;
  r.phase = r.steps > 0 ? Request::ABSORB : Request::MEASURE;
}

void Server::finish(Request& r) {
  std::vector<TermSpec> terms(r.kind.size());
  for (size_t i = 0; i < r.kind.size(); ++i) {
    TermSpec& t = terms[i];
    std::memset(&t, 0, sizeof(t));
    t.kind = r.kind[i];
    t.coeff[0] = r.coeff[2 * i];
    t.coeff[1] = r.coeff[2 * i + 1];
    if (t.kind == 1) {
      auto it = r.job->g.index_of.find(r.q0[i]);
      if (it == r.job->g.index_of.end()) throw Error(TNBP_EINVAL, "term on a qubit outside the lattice");
      t.site_a = it->second;
      auto P = tnbp_host::pauli_list(r.letters[2 * i]);
      for (int k = 0; k < 4; ++k) { t.op[2 * k] = P[k].real(); t.op[2 * k + 1] = P[k].imag(); }
    } else {
      t.edge = r.job->edge_of(r.q0[i], r.q1[i]);
      if (t.edge < 0) throw Error(TNBP_EINVAL, "two-site term on a non-adjacent pair");
      t.label_a = r.q0[i];
      auto Pa = tnbp_host::pauli_list(r.letters[2 * i]);
      auto Pb = tnbp_host::pauli_list(r.letters[2 * i + 1]);
      for (int i0 = 0; i0 < 2; ++i0)
        for (int i1 = 0; i1 < 2; ++i1)
          for (int i2 = 0; i2 < 2; ++i2)
            for (int i3 = 0; i3 < 2; ++i3) {
              const auto v = Pa[i0 + 2 * i2] * Pb[i1 + 2 * i3];
              const int idx = i0 + 2 * i1 + 4 * i2 + 8 * i3;
              t.op[2 * idx] = v.real();
              t.op[2 * idx + 1] = v.imag();
            }
    }
  }
  r.job->measure_terms(terms, nullptr, r.result);
  r.job.reset();
  r.tpos.reset();
  r.phase = Request::DONE;
}

// A request whose own work raises an error (a non-finite BP condition, a
// truncation that reports non-finite messages or an SVD sweep limit) is
// finished with that error; the other requests are not affected.
void Server::fail(Request& r, int code, const std::string& msg) {
  r.error_code = code;
  r.error = msg;
  r.result[0] = r.result[1] = std::nan("");
  r.job.reset();
  r.tpos.reset();
  r.phase = Request::DONE;
}

void Server::cancel(int64_t id) {
  auto it = reqs.find(id);
  if (it == reqs.end()) throw Error(TNBP_EINVAL, "unknown request id");
  Request& r = *it->second;
  if (r.phase == Request::DONE) return;
  const bool admitted = r.phase != Request::QUEUED;
  queue.erase(std::remove(queue.begin(), queue.end(), id), queue.end());
  active.erase(std::remove(active.begin(), active.end(), id), active.end());
  if (admitted) in_use -= r.footprint;
  fail(r, TNBP_ECANCELED, "request cancelled");
}

// Restart a request from |0...0> in complex128 (see Server::escalate); its
// footprint is re-counted for the complex128 job.
void Server::restart_c128(Request& r) {
  r.job.reset();
  in_use -= r.footprint;
  r.prec = TNBP_C128;
  r.escalated = true;
  r.footprint = footprint(r);
  in_use += r.footprint;
  start(r);
}

// The batched BP sweep of one group of requests whose jobs all have
// precision gprec: its task arrays built (on the server's stream, where the
// jobs' own work runs) and, once launched, its read-back and the BP-loop
// decision of each request.
Server::GroupSweep Server::prepare_group(int gprec, const std::vector<Request*>& inbp) {
  TNBP_TRACE_SCOPE("server.3_sweep");
  GroupSweep g;
  g.gprec = gprec;
  g.reqs = inbp;
  std::vector<BatchEntry> entries;
  for (auto* r : inbp) {
    r->job->sync_shadow();
    if (!r->job->plan.valid) r->job->build_plan();
    entries.push_back({r->job.get(), r->job->cur});
  }
  prepare_kernels(gprec);
  std::vector<uint64_t> key;
  for (auto& e : entries) key.push_back(2 * e.job->plan_serial + (uint64_t)e.parity);
  auto it = sweeps.find(key);
  if (it == sweeps.end()) {
    auto cs = std::make_unique<CachedSweep>();
    build_batch(entries, cs->batch, stream);
    it = sweeps.emplace(key, std::move(cs)).first;
    sweeps_lru.push_back(key);
    while (sweeps.size() > sweeps_cap) {
      if (sweeps_lru.front() == key) {  // never the batch about to run
        sweeps_lru.splice(sweeps_lru.end(), sweeps_lru, sweeps_lru.begin());
        continue;
      }
      sweeps.erase(sweeps_lru.front());
      sweeps_lru.pop_front();
    }
  } else {
    sweeps_lru.remove(key);
    sweeps_lru.push_back(key);
  }
  g.cs = it->second.get();
  return g;
}

// Launches a prepared group on stream s (captured as a CUDA graph on its
// second use, relaunched as that graph after) and queues the read-back of
// its conditions into the pinned buffer h.
void Server::launch_group(GroupSweep& g, cudaStream_t s, PinnedConds& h) {
  CachedSweep& cs = *g.cs;
  SweepBatch& batch = cs.batch;
  if (cs.uses == 1 && !batch.graph) {
    TNBP_TRACE_SCOPE("server.3_graph_capture");
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      batch.nkernels = launch_batch(batch, g.gprec, s);
    } catch (...) {
      cudaStreamEndCapture(s, &graph);
      throw;
    }
    CK(cudaStreamEndCapture(s, &graph));
    CK(cudaGraphInstantiate(&batch.graph, graph, 0));
    cudaGraphDestroy(graph);
  }
  if (batch.graph) {
    CK(cudaGraphLaunch(batch.graph, s));
    note_launch(batch.nkernels);
    ++graph_launches;
  } else {
    note_launch(launch_batch(batch, g.gprec, s));
    ++eager_launches;
  }
  ++cs.uses;
  if (h.cap < g.reqs.size()) {
    if (h.p) cudaFreeHost(h.p);
    h.p = nullptr;
    h.cap = std::max<size_t>(64, 2 * g.reqs.size());
    CK(cudaMallocHost(&h.p, h.cap * sizeof(double)));
  }
  g.h = h.p;
  CK(cudaMemcpyAsync(h.p, batch.cond.p, g.reqs.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
}

// After the group's stream has finished: each request's BP-loop decision.
void Server::finish_group(GroupSweep& g) {
  for (size_t i = 0; i < g.reqs.size(); ++i) {
    Request& r = *g.reqs[i];
    Job& j = *r.job;
    if (r.bp_iters == 0) {  // first sweep of the loop: always kept
      j.cur = 1 - j.cur;
      r.bp_iters = 1;
      continue;
    }
    const double c = g.h[i];
    if (!std::isfinite(c)) {
      fail(r, TNBP_ENOTCONV, "BP condition is not finite (non-finite messages)");
      continue;
    }
    const bool conv = c < effective_tol(g.gprec, r.tol);
    r.loop_min_cond = std::min(r.loop_min_cond, c);
    if (conv || r.bp_iters >= r.maxit || stop_on_growth(g.gprec, r.prev_cond, c)) {
      r.phase = Request::TRUNC;  // keep the current messages
      if (!conv && r.bp_iters >= r.maxit) {
        r.bp_converged = false;
        ++r.unconv_loops;
        r.worst_final_cond = std::max(r.worst_final_cond, c);
        r.worst_min_cond = std::max(r.worst_min_cond, r.loop_min_cond);
        if (escalate && r.prec != TNBP_C128 && r.loop_min_cond > escalate_min_cond) restart_c128(r);
      }
    } else {
      r.prev_cond = c;
      j.cur = 1 - j.cur;
      ++r.bp_iters;
    }
  }
}

void Server::step(int* n_active, int* n_queued, int* n_done) {
  TNBP_TRACE_SCOPE("server.step");
  int done = 0;
  // 1. admission by HBM footprint and free slots
  TNBP_TRACE_SCOPE("server.1_admit_absorb");
  while (!queue.empty() && (int)active.size() < max_active) {
    Request& r = *reqs[queue.front()];
    if (!active.empty() && in_use + r.footprint > budget) break;
    queue.pop_front();
    start(r);
    in_use += r.footprint;
    active.push_back(r.id);
  }
  // 2. TPO absorption for requests entering a Floquet step
  for (int64_t id : active) {
    Request& r = *reqs[id];
    if (r.phase == Request::ABSORB) {
      r.job->absorb_tpo(*r.tpos->layers[r.source == Request::QASM ? r.step : 0]);
      r.phase = Request::BP;
      r.bp_iters = 0;
      r.prev_cond = INFINITY;
      r.loop_min_cond = INFINITY;
      if (r.maxit <= 0) r.phase = Request::TRUNC;
    }
  }
  // 3. one batched BP sweep over every request in its BP phase, one batch
  // per job precision.  Requests escalated to complex128 sweep apart, on a
  // second stream forked from the server's stream before the first batch
  // and joined back after, so the two batches can run side by side; the host
  // waits once for both.
  {
    std::vector<Request*> grp[2];
    for (int64_t id : active) {
      Request& r = *reqs[id];
      if (r.phase == Request::BP) grp[r.prec == prec ? 0 : 1].push_back(&r);
    }
    std::vector<GroupSweep> gs;
    if (!grp[0].empty()) gs.push_back(prepare_group(prec, grp[0]));
    if (!grp[1].empty()) gs.push_back(prepare_group(TNBP_C128, grp[1]));
    if (gs.size() == 2) CK(cudaEventRecord(ev_fork, stream));
    for (size_t k = 0; k < gs.size(); ++k) {
      if (k == 1) {
        CK(cudaStreamWaitEvent(stream2, ev_fork, 0));
        launch_group(gs[k], stream2, hconds[1]);
        CK(cudaEventRecord(ev_join, stream2));
        CK(cudaStreamWaitEvent(stream, ev_join, 0));
      } else {
        launch_group(gs[k], stream, hconds[0]);
      }
    }
    if (!gs.empty()) {
      CK(cudaStreamSynchronize(stream));
      if (gs.size() == 2) CK(cudaStreamSynchronize(stream2));
      if (reduced_sweeps(prec)) check_tc_error(stream);
      for (auto& g : gs) finish_group(g);
    }
  }
  // 4. truncation, next step or measurement
  TNBP_TRACE_SCOPE("server.4_trunc_measure");
  for (int64_t id : active) {
    Request& r = *reqs[id];
    try {
      if (r.phase == Request::TRUNC) {
        r.job->truncate(r.chi, r.sv_min, nullptr, nullptr);
        ++r.step;
        r.phase = r.step < r.steps ? Request::ABSORB : Request::MEASURE;
      }
      if (r.phase == Request::MEASURE) finish(r);
    } catch (const Error& e) {
      if (e.code == TNBP_ECUDA) throw;  // the device context is not usable
      fail(r, e.code, e.what());
    }
    if (r.phase == Request::DONE) {
      in_use -= r.footprint;
      ++done;
    }
  }
  active.erase(std::remove_if(active.begin(), active.end(),
                              [&](int64_t id) { return reqs[id]->phase == Request::DONE; }),
               active.end());
  if (n_active) *n_active = (int)active.size();
  if (n_queued) *n_queued = (int)queue.size();
  if (n_done) *n_done = done;
}

}  // namespace tnbp

// ------------------------------------------------------------------ C ABI
struct tnbp_server { std::unique_ptr<tnbp::Server> s; };

namespace {
template <class F>
int sguard(F&& f) {
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
  } catch (const std::exception& e) {
    tnbp::g_last_error = e.what();
    return TNBP_EINVAL;
  }
}
}  // namespace

extern "C" {

int tnbp_server_create(int32_t precision, uint64_t budget, int32_t max_active, tnbp_server** out) {
  return sguard([&] {
    if (!out) throw tnbp::Error(TNBP_EINVAL, "out is NULL");
    *out = nullptr;
    auto s = std::make_unique<tnbp_server>();
    s->s = std::make_unique<tnbp::Server>(precision, budget, max_active);
    *out = s.release();
  });
}

int tnbp_server_destroy(tnbp_server* srv) { return sguard([&] { delete srv; }); }

int tnbp_server_submit_kicked_ising(tnbp_server* srv, int32_t L, int32_t chi, int32_t n_steps, double theta_j,
                                    double theta_h, double bp_tol, int32_t bp_max_iter, double sv_min,
                                    int64_t n_terms, const int32_t* kind, const int32_t* q0, const int32_t* q1,
                                    const char* letters, const double* coeff, int64_t* request_id) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    if (n_terms > 0 && !(kind && q0 && q1 && letters && coeff)) throw tnbp::Error(TNBP_EINVAL, "NULL term arrays");
    auto r = std::make_unique<tnbp::Request>();
    r->L = L; r->chi = chi; r->steps = n_steps; r->theta_j = theta_j; r->theta_h = theta_h;
    r->tol = bp_tol; r->maxit = bp_max_iter; r->sv_min = sv_min;
    r->kind.assign(kind, kind + n_terms);
    r->q0.assign(q0, q0 + n_terms);
    r->q1.assign(q1, q1 + n_terms);
    r->letters.assign(letters, letters + 2 * n_terms);
    r->coeff.assign(coeff, coeff + 2 * n_terms);
    for (int64_t i = 0; i < n_terms; ++i)
      if (r->kind[i] != 1 && r->kind[i] != 2) throw tnbp::Error(TNBP_EINVAL, "term kind must be 1 or 2");
    if (L < 2) throw tnbp::Error(TNBP_EINVAL, "lattice side must be >= 2");
    if (!std::isfinite(theta_j) || !std::isfinite(theta_h) || !std::isfinite(bp_tol) || !std::isfinite(sv_min))
      throw tnbp::Error(TNBP_EINVAL, "non-finite request parameter");
    for (int64_t i = 0; i < 2 * n_terms; ++i)
      if (!std::isfinite(coeff[i])) throw tnbp::Error(TNBP_EINVAL, "non-finite term coefficient");
    // RZZ(theta_j) = exp(-i theta_j/2 ZZ), RX(theta_h) = exp(-i theta_h/2 X)
    char key[96];
    std::snprintf(key, sizeof(key), "kicked_ising %d %a %a", L, theta_j, theta_h);
    r->tpos = srv->s->tpo_set(key, [&](tnbp_host::Edges& e, std::vector<tnbp_host::Layer>& layers) {
      e = tnbp_host::square_lattice(L, L);
      layers.push_back(tnbp_host::kicked_ising_tpo(e, theta_j / 2.0, 0.0, theta_h / 2.0, 1.0));
    });
    const int64_t id = srv->s->submit(std::move(r));
    if (request_id) *request_id = id;
  });
}

int tnbp_server_submit_qasm(tnbp_server* srv, const char* qasm_src, const char* pauli_text, int32_t chi,
                            double bp_tol, int32_t bp_max_iter, double sv_min, int32_t do_opt_tpo,
                            double eps_opt_tpo, int64_t* request_id) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    if (!qasm_src || !pauli_text) throw tnbp::Error(TNBP_EINVAL, "NULL program or observable");
    if (!std::isfinite(bp_tol) || !std::isfinite(sv_min) || !std::isfinite(eps_opt_tpo))
      throw tnbp::Error(TNBP_EINVAL, "non-finite request parameter");
    auto r = std::make_unique<tnbp::Request>();
    r->source = tnbp::Request::QASM;
    r->chi = chi; r->tol = bp_tol; r->maxit = bp_max_iter; r->sv_min = sv_min;
    char opts[64];
    std::snprintf(opts, sizeof(opts), "qasm opt=%d eps=%a\n", do_opt_tpo ? 1 : 0, do_opt_tpo ? eps_opt_tpo : 0.0);
    r->tpos = srv->s->tpo_set(std::string(opts) + qasm_src,
                              [&](tnbp_host::Edges& e, std::vector<tnbp_host::Layer>& layers) {
                                const auto prog = tnbp_host::parse_qasm(qasm_src);
                                e = tnbp_host::qasm_edges(prog);
                                layers = tnbp_host::qasm_tpo(prog, e);
                                if (do_opt_tpo)
                                  for (auto& l : layers) tnbp_host::opt_tpo_svd(e, l, eps_opt_tpo);
                              });
    r->steps = (int)r->tpos->layers.size();
    // the estimator app's observable: load_sparse_pauli_op + ClassifyOps
    int64_t dropped = 0;
    const auto terms = tnbp_host::pauli_terms(pauli_text, r->tpos->edges, &dropped);
    const auto labels = tnbp_host::site_labels(r->tpos->edges);
    for (const auto& t : terms) {
      if (t.kind == 1 && !std::binary_search(labels.begin(), labels.end(), t.q0))
        throw tnbp::Error(TNBP_EINVAL, "one-site term on qubit " + std::to_string(t.q0) + " that no two-qubit gate touches");
      r->kind.push_back(t.kind);
      r->q0.push_back(t.q0);
      r->q1.push_back(t.q1);
      r->letters.push_back(t.l0);
      r->letters.push_back(t.kind == 2 ? t.l1 : 'I');
      r->coeff.push_back(t.coeff_re);
      r->coeff.push_back(t.coeff_im);
    }
    const int64_t id = srv->s->submit(std::move(r));
    if (request_id) *request_id = id;
  });
}

int tnbp_footprint_estimate(const int32_t* edges, int64_t n_edges, const int32_t* bond_dim, int32_t precision,
                            uint64_t* bytes) {
  return sguard([&] {
    if (!bytes || !bond_dim || (n_edges > 0 && !edges)) throw tnbp::Error(TNBP_EINVAL, "NULL argument");
    if (precision != TNBP_C128 && precision != TNBP_C64 && precision != TNBP_MIXED)
      throw tnbp::Error(TNBP_EINVAL, "unknown precision");
    std::vector<std::pair<int, int>> e(n_edges);
    std::vector<double> D(n_edges);
    for (int64_t i = 0; i < n_edges; ++i) {
      e[i] = {edges[2 * i], edges[2 * i + 1]};
      if (bond_dim[i] < 1) throw tnbp::Error(TNBP_EINVAL, "bond dimension < 1");
      D[i] = bond_dim[i];
    }
    *bytes = tnbp::footprint_estimate(e, D, precision, 0);
  });
}

int tnbp_server_tpo_cache_stats(tnbp_server* srv, int64_t* hits, int64_t* misses, int64_t* entries) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    if (hits) *hits = srv->s->cache_hits;
    if (misses) *misses = srv->s->cache_misses;
    if (entries) *entries = (int64_t)srv->s->tpo_cache.size();
  });
}

int tnbp_server_step(tnbp_server* srv, int32_t* n_active, int32_t* n_queued, int32_t* n_done) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    int a = 0, q = 0, d = 0;
    srv->s->step(&a, &q, &d);
    if (n_active) *n_active = a;
    if (n_queued) *n_queued = q;
    if (n_done) *n_done = d;
  });
}

int tnbp_server_cancel(tnbp_server* srv, int64_t id) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    srv->s->cancel(id);
  });
}

int tnbp_server_result(tnbp_server* srv, int64_t id, double* sum, int32_t* pending) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    auto it = srv->s->reqs.find(id);
    if (it == srv->s->reqs.end()) throw tnbp::Error(TNBP_EINVAL, "unknown request id");
    const bool done = it->second->phase == tnbp::Request::DONE;
    if (pending) *pending = done ? 0 : 1;
    if (done && it->second->error_code) throw tnbp::Error(it->second->error_code, it->second->error);
    if (sum && done) { sum[0] = it->second->result[0]; sum[1] = it->second->result[1]; }
  });
}

int tnbp_server_set_escalation(tnbp_server* srv, int32_t on) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    srv->s->escalate = on != 0;
  });
}

int tnbp_server_set_escalation_threshold(tnbp_server* srv, double min_cond) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    if (!(min_cond >= 0.0) || !std::isfinite(min_cond))
      throw tnbp::Error(TNBP_EINVAL, "escalation threshold must be finite and >= 0");
    srv->s->escalate_min_cond = min_cond;
  });
}

int tnbp_server_request_bp_stats(tnbp_server* srv, int64_t id, int32_t* unconverged_loops,
                                 double* worst_final_cond, double* worst_min_cond) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    auto it = srv->s->reqs.find(id);
    if (it == srv->s->reqs.end()) throw tnbp::Error(TNBP_EINVAL, "unknown request id");
    const tnbp::Request& r = *it->second;
    if (unconverged_loops) *unconverged_loops = r.unconv_loops;
    if (worst_final_cond) *worst_final_cond = r.worst_final_cond;
    if (worst_min_cond) *worst_min_cond = r.worst_min_cond;
  });
}

int tnbp_server_request_info(tnbp_server* srv, int64_t id, int32_t* precision, int32_t* escalated,
                             int32_t* bp_converged) {
  return sguard([&] {
    if (!srv) throw tnbp::Error(TNBP_EINVAL, "server is NULL");
    auto it = srv->s->reqs.find(id);
    if (it == srv->s->reqs.end()) throw tnbp::Error(TNBP_EINVAL, "unknown request id");
    const tnbp::Request& r = *it->second;
    if (precision) *precision = r.prec;
    if (escalated) *escalated = r.escalated ? 1 : 0;
    if (bp_converged) *bp_converged = r.bp_converged ? 1 : 0;
  });
}

}  // extern "C"
