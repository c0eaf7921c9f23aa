// Device-resident BP-PEPS estimator engine behind the C ABI of
// include/tnbp_b200.h.  One job = one PEPS (site tensors V, two message
// arenas E/F) on one GPU stream.  Host code only builds task descriptors;
// all tensor arithmetic runs in the kernels of kernels.cuh, truncate.cuh and
// measure.cuh.  There is no CPU fallback: without a device every state call
// fails with TNBP_ENOGPU.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <fstream>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tnbp_b200.h"
#include "engine.h"
#include "host_setup.h"
#include "kernels.cuh"
#include "measure.cuh"
#include "tc_leg.cuh"
#include "tc_leg_bulk.cuh"
#include "tc_gram.cuh"
#include "tc_leg64.cuh"
#include "tc_leg_gram.cuh"
#include "site_sweep.cuh"
#include "trace.h"
#include "truncate.cuh"

namespace tnbp {

thread_local std::string g_last_error;
std::atomic<unsigned long long> g_launches{0};
void note_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    throw Error(TNBP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                                std::to_string(line) + ")");
  }
}

// Per-device one-time settings (the memory pool's release threshold, the
// opt-in dynamic shared memory of the sweep kernels) belong to a device
// context: each kernel family records, per
// device ordinal, that they were set, under one mutex, so several devices
// and threads may share the library.
static std::mutex g_attr_mu;
static bool attr_done(std::vector<char>& flags) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if ((int)flags.size() <= dev) flags.resize(dev + 1, 0);
  return flags[dev] != 0;
}
static void attr_mark(std::vector<char>& flags) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  flags[dev] = 1;
}

// ----------------------------------------------------------------- memory
DevBuf::~DevBuf() { release(); }
void DevBuf::release() {
  if (p) {
    cudaFreeAsync(p, stream);
    p = nullptr;
  }
  bytes = 0;
}
void DevBuf::alloc(size_t nbytes, cudaStream_t s) {
  release();
  stream = s;
  if (nbytes == 0) return;
  cudaError_t e = cudaMallocAsync(&p, nbytes, s);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    throw Error(TNBP_ENOMEM, "device allocation of " + std::to_string(nbytes) + " bytes failed: " +
                                 cudaGetErrorString(e));
  }
  bytes = nbytes;
}

template <typename T>
static void upload_vec(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
  b.alloc(std::max<size_t>(sizeof(T), v.size() * sizeof(T)), s);
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

static inline size_t align_elems(size_t n) { return (n + 31) & ~size_t(31); }

// Site tensors are re-laid out at every AbsorbTPO and truncation; keep the
// stream-ordered pool's memory mapped across synchronizations instead of
// returning it to the driver each time (the default threshold of 0 makes
// every large re-allocation map fresh pages).
void keep_pool_memory() {
  static std::vector<char> flags;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (attr_done(flags)) return;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  attr_mark(flags);
}

// ------------------------------------------------------------------ graph
Graph::Graph(const int32_t* e, int64_t n) {
  if (n <= 0 || !e) throw Error(TNBP_EINVAL, "edge list is empty");
  edges.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    edges[i] = {e[2 * i], e[2 * i + 1]};
    if (edges[i].first == edges[i].second) throw Error(TNBP_EINVAL, "self-loop edge");
  }
  // GetSiteIndexFromBond (graph.h:23-35): sorted distinct labels
  for (auto& p : edges) { labels.push_back(p.first); labels.push_back(p.second); }
  std::sort(labels.begin(), labels.end());
  labels.erase(std::unique(labels.begin(), labels.end()), labels.end());
  for (size_t s = 0; s < labels.size(); ++s) index_of[labels[s]] = (int)s;
  // GetSurroundingBondIndex (graph.h:40-55): incident edges in edge order
  legs.assign(labels.size(), {});
  leg_a.resize(n);
  leg_b.resize(n);
  site_a.resize(n);
  site_b.resize(n);
  for (int64_t m = 0; m < n; ++m) {
    const int a = index_of[edges[m].first], b = index_of[edges[m].second];
    site_a[m] = a;
    site_b[m] = b;
    leg_a[m] = (int)legs[a].size();
    legs[a].push_back((int)m);
    leg_b[m] = (int)legs[b].size();
    legs[b].push_back((int)m);
  }
  for (auto& l : legs)
    if ((int)l.size() > kMaxLegs) throw Error(TNBP_EINVAL, "site degree above " + std::to_string(kMaxLegs));
}

// message index computed at site s along its leg k, and the one it absorbs
int Graph::out_msg(int s, int k) const {
  const int e = legs[s][k];
  return site_a[e] == s ? e : e + (int)edges.size();
}
int Graph::in_msg(int s, int k) const {
  const int e = legs[s][k];
  return site_a[e] == s ? e + (int)edges.size() : e;
}

// Page-locked 64-byte slots for the jobs' condition read-backs.  A
// cudaMallocHost and cudaFreeHost per job cost milliseconds (page locking,
// and the free synchronizes the device): a job takes a slot from blocks
// allocated once per process and gives it back when it is destroyed (after
// its stream is idle, so no copy into the slot is pending).
namespace {
struct PinnedSlots {
  std::mutex mu;
  std::vector<double*> free;
};
PinnedSlots& pinned_slots() {
  static PinnedSlots* p = new PinnedSlots();  // blocks live until exit
  return *p;
}
constexpr size_t kSlotBytes = 64, kSlotsPerBlock = 1024;
double* pinned_slot_get() {
  PinnedSlots& P = pinned_slots();
  std::lock_guard<std::mutex> lk(P.mu);
  if (P.free.empty()) {
    void* b = nullptr;
    CK(cudaMallocHost(&b, kSlotBytes * kSlotsPerBlock));
    for (size_t i = kSlotsPerBlock; i-- > 0;)
      P.free.push_back(reinterpret_cast<double*>(static_cast<char*>(b) + i * kSlotBytes));
  }
  double* slot = P.free.back();
  P.free.pop_back();
  return slot;
}
void pinned_slot_put(double* slot) {
  PinnedSlots& P = pinned_slots();
  std::lock_guard<std::mutex> lk(P.mu);
  P.free.push_back(slot);
}
}  // namespace

// -------------------------------------------------------------------- job
Job::Job(const int32_t* e, int64_t n, const int32_t* pdims, int precision, cudaStream_t s,
         uint64_t budget)
    : g(e, n), prec(precision), budget(budget) {
  if (precision != TNBP_C128 && precision != TNBP_C64 && precision != TNBP_MIXED)
    throw Error(TNBP_EINVAL, "unknown precision");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    throw Error(TNBP_ENOGPU, "no CUDA device visible: the B200 engine has no CPU path");
  }
  sprec = prec == TNBP_C64 ? TNBP_C64 : TNBP_C128;
  esz = sprec == TNBP_C128 ? 16 : 8;
  wsz = prec == TNBP_C128 ? 16 : 8;
  keep_pool_memory();
  if (s) {
    stream = s;
  } else {
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  host_scalar = pinned_slot_get();
  const int ns = (int)g.labels.size();
  pd.assign(ns, 2);
  if (pdims) for (int i = 0; i < ns; ++i) pd[i] = pdims[i];
  dim.assign(g.edges.size(), 1);
  layout();
  V.alloc(v_elems * esz, stream);
  M[0].alloc(m_elems * esz, stream);
  M[1].alloc(m_elems * esz, stream);
  // |0...0>: V_s = e_0 on the physical leg; messages = [1] (init.h:40-61)
  std::vector<double> hv(2 * v_elems, 0.0), hm(2 * m_elems, 0.0);
  for (int s = 0; s < ns; ++s) hv[2 * voff[s]] = 1.0;
  for (size_t m = 0; m < moff.size(); ++m) hm[2 * moff[m]] = 1.0;
  put_complex(V, hv.data(), v_elems, 0);
  put_complex(M[0], hm.data(), m_elems, 0);
  cur = 0;
  CK(cudaStreamSynchronize(stream));
  check_budget();
}

Job::~Job() {
  destroy_graphs();
  cudaStreamSynchronize(stream);
  V.release(); M[0].release(); M[1].release(); V32.release();
  ws_scratch.release(); ws_chain[0].release(); ws_chain[1].release(); Vspare.release();
  plan = SweepPlan();
  if (host_scalar) pinned_slot_put(host_scalar);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  cudaStreamSynchronize(stream);
  if (own_stream) cudaStreamDestroy(stream);
}

std::vector<int> Job::site_shape(int s) const {
  std::vector<int> sh;
  for (int e : g.legs[s]) sh.push_back(dim[e]);
  sh.push_back(pd[s]);
  return sh;
}
size_t Job::site_elems(int s) const {
  size_t n = pd[s];
  for (int e : g.legs[s]) n *= dim[e];
  return n;
}

void Job::layout() {
  const int ns = (int)g.labels.size();
  const int ne = (int)g.edges.size();
  voff.assign(ns, 0);
  size_t o = 0;
  for (int s = 0; s < ns; ++s) { voff[s] = o; o += align_elems(site_elems(s)); }
  v_elems = std::max<size_t>(o, 32);
  moff.assign(2 * ne, 0);
  o = 0;
  for (int m = 0; m < 2 * ne; ++m) {
    const size_t dd = (size_t)dim[m % ne] * dim[m % ne];
    moff[m] = o;
    o += align_elems(dd);
  }
  m_elems = std::max<size_t>(o, 32);
}

void Job::put_complex(DevBuf& dst, const double* src, size_t n, size_t elem_off) {
  if (n == 0) return;
  if (&dst == &V) shadow_dirty = true;
  if (sprec == TNBP_C128) {
    CK(cudaMemcpyAsync(static_cast<char*>(dst.p) + elem_off * 16, src, n * 16, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  } else {
    std::vector<float> f(2 * n);
    for (size_t i = 0; i < 2 * n; ++i) f[i] = (float)src[i];
    CK(cudaMemcpyAsync(static_cast<char*>(dst.p) + elem_off * 8, f.data(), n * 8, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
}
void Job::get_complex(const DevBuf& src, double* dst, size_t n, size_t elem_off) {
  if (n == 0) return;
  if (sprec == TNBP_C128) {
    CK(cudaMemcpyAsync(dst, static_cast<const char*>(src.p) + elem_off * 16, n * 16, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  } else {
    std::vector<float> f(2 * n);
    CK(cudaMemcpyAsync(f.data(), static_cast<const char*>(src.p) + elem_off * 8, n * 8, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < 2 * n; ++i) dst[i] = f[i];
  }
}

uint64_t Job::device_bytes() const {
  return V.bytes + M[0].bytes + M[1].bytes + V32.bytes + ws_scratch.bytes + ws_chain[0].bytes +
         ws_chain[1].bytes + Vspare.bytes + plan.bytes();
}
void Job::check_budget() const {
  if (budget && device_bytes() > budget)
    throw Error(TNBP_ENOMEM, "job needs " + std::to_string(device_bytes()) + " device bytes, budget " +
                                 std::to_string(budget));
}

void* Job::vptr(int s) const { return static_cast<char*>(V.p) + voff[s] * esz; }
void* Job::sweep_vptr(int s) const {
  return prec == TNBP_MIXED ? static_cast<char*>(V32.p) + voff[s] * 8 : vptr(s);
}

// TNBP_MIXED: round the complex128 site tensors to the complex64 copy that
// the sweeps read (the copy only grows).  A re-allocated copy invalidates the
// sweep plan (its tasks and graphs hold the old addresses).
void Job::sync_shadow() {
  if (prec != TNBP_MIXED || !shadow_dirty) return;
  TNBP_TRACE_SCOPE("sweep.sync_shadow");
  if (V32.ensure(v_elems * 8, stream)) {
    destroy_graphs();
    plan = SweepPlan();
  }
  const unsigned grid = (unsigned)std::min<size_t>((v_elems + 255) / 256, (size_t)8 * num_sms());
  k_narrow<<<grid, 256, 0, stream>>>(static_cast<const double2*>(V.p), static_cast<float2*>(V32.p), v_elems);
  CK(cudaGetLastError());
  note_launch();
  shadow_dirty = false;
}
void* Job::mptr(int arena, int m) const { return static_cast<char*>(M[arena].p) + moff[m] * esz; }

void Job::destroy_graphs() {
  plan.single[0].reset_graph();
  plan.single[1].reset_graph();
}

void SweepBatch::reset_graph() {
  if (graph) {
    cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
}
SweepBatch& SweepBatch::operator=(SweepBatch&& o) noexcept {
  if (this != &o) {
    reset_graph();
    arena = std::move(o.arena);
    cond = std::move(o.cond);
    launches = std::move(o.launches);
    nkernels = o.nkernels;
    uses = o.uses;
    graph = o.graph;
    o.graph = nullptr;
  }
  return *this;
}

SweepPlan::~SweepPlan() {}
uint64_t SweepPlan::bytes() const {
  return partial.bytes + dist.bytes + single[0].bytes() + single[1].bytes();
}

// --------------------------------------------------------------- sweep plan
// Messages T_t = V x_{k != t} E_k for all targets t of a site share partial
// products: targets are split in halves, the legs of the other half are
// absorbed once for each half, and the recursion continues.  A degree-4
// site needs 8 leg contractions instead of the 12 of the leg-by-leg
// schedule of bp.h:137-154 (the same products in another association; the
// per-leg normalizations of bp.h:153 only rescale, and the final
// normalization of bp.h:166 removes the scale).  The two top-level halves
// of a site's tree ("units") are independent: each starts from V.
namespace {
struct PlanOp { int site, src, dst, leg, level, unit; };
struct SitePlanner {
  int site;
  std::vector<PlanOp>* ops;
  int next_slot = 0;
  std::vector<int> result;       // slot holding T_t (-1 = V itself)
  std::vector<int> result_unit;  // unit whose ops produce T_t
  int chain(int src, int level, int unit, const std::vector<int>& legs, int* out_level) {
    int cur = src, lv = level;
    for (int leg : legs) {
      const int dst = next_slot++;
      ops->push_back({site, cur, dst, leg, lv, unit});
      cur = dst;
      ++lv;
    }
    *out_level = lv;
    return cur;
  }
  // unit < 0: the top of the tree (its two halves become units 0 and 1)
  void rec(int src, int level, int unit, const std::vector<int>& targets, std::vector<char> absorbed, int g) {
    if (targets.size() == 1) {
      const int u = unit < 0 ? 0 : unit;
      std::vector<int> rest;
      for (int k = 0; k < g; ++k) if (k != targets[0] && !absorbed[k]) rest.push_back(k);
      int lv;
      result[targets[0]] = chain(src, level, u, rest, &lv);
      result_unit[targets[0]] = u;
      return;
    }
    const size_t h = targets.size() / 2;
    std::vector<int> h1(targets.begin(), targets.begin() + h), h2(targets.begin() + h, targets.end());
    for (int part = 0; part < 2; ++part) {
      const int u = unit < 0 ? part : unit;
      const auto& keep = part == 0 ? h1 : h2;
      const auto& other = part == 0 ? h2 : h1;
      std::vector<int> legs;
      for (int k : other) if (!absorbed[k]) legs.push_back(k);
      int lv;
      const int x = chain(src, level, u, legs, &lv);
      auto ab = absorbed;
      for (int k : legs) ab[k] = 1;
      rec(x, lv, u, keep, ab, g);
    }
  }
};

// One unit of a site's tree with its intermediate slots mapped onto as few
// site-sized buffers as their lifetimes allow: ops of one level run in one
// launch, so a buffer read at level l is free for outputs of level l + 1;
// the T_t results (or, for a fused target, the input X of its last
// absorption) stay live until the Gram stage.  A fused target's last
// absorption is not an op of the unit: k_leg_gram_tc does it on chip.
struct Fused { int target, src, leg; };
struct Unit {
  int site = 0;
  std::vector<PlanOp> ops;
  std::vector<int> targets;  // targets with a plain Gram (of result[t])
  std::vector<Fused> fused;  // targets with the fused absorption + Gram
  std::map<int, int> buf_of_slot;
  int nbuf = 0;
  int nlevels = 0;
};

template <typename FuseFn>
Unit make_unit(int site, int u, const std::vector<PlanOp>& all, const SitePlanner& sp, FuseFn fuse) {
  Unit U;
  U.site = site;
  std::vector<char> skip(all.size(), 0);
  for (size_t t = 0; t < sp.result.size(); ++t) {
    if (sp.result_unit[t] != u) continue;
    const int r = sp.result[t];
    int fi = -1;
    if (r >= 0)
      for (size_t i = 0; i < all.size(); ++i)
        if (all[i].site == site && all[i].dst == r) fi = (int)i;
    if (fi >= 0 && fuse((int)t, all[fi].leg)) {
      skip[fi] = 1;
      U.fused.push_back({(int)t, all[fi].src, all[fi].leg});
    } else {
      U.targets.push_back((int)t);
    }
  }
  for (size_t i = 0; i < all.size(); ++i)
    if (all[i].site == site && all[i].unit == u && !skip[i]) U.ops.push_back(all[i]);
  std::stable_sort(U.ops.begin(), U.ops.end(), [](const PlanOp& a, const PlanOp& b) { return a.level < b.level; });
  constexpr int kForever = 1 << 30;
  std::map<int, int> last_read;
  for (const auto& op : U.ops)
    if (op.src >= 0) last_read[op.src] = std::max(last_read[op.src], op.level);
  for (int t : U.targets)
    if (sp.result[t] >= 0) last_read[sp.result[t]] = kForever;
  for (const auto& f : U.fused)
    if (f.src >= 0) last_read[f.src] = kForever;
  std::vector<int> busy_until;  // per buffer: last level its content is read
  for (const auto& op : U.ops) {
    int b = -1;
    for (size_t i = 0; i < busy_until.size(); ++i)
      if (busy_until[i] < op.level) { b = (int)i; break; }
    if (b < 0) { b = (int)busy_until.size(); busy_until.push_back(0); }
    U.buf_of_slot[op.dst] = b;
    auto it = last_read.find(op.dst);
    busy_until[b] = it == last_read.end() ? op.level : it->second;
    U.nlevels = std::max(U.nlevels, op.level + 1);
  }
  U.nbuf = (int)busy_until.size();
  return U;
}
}  // namespace

// Bytes of site tensors plus intermediate slots one wave may hold; 0 puts
// every unit of the sweep in one wave.  TNBP_WAVE_MB fixes it for every job
// (no autotuning); otherwise a job uses the autotuned budget of its shape
// class (below) or this default of one wave: on the 16x16 D = 32 sweep one
// wave measured 25.5 ms against 50.5 ms at 96 MiB (L2-sized waves), whose
// many small launches cost more than the L2 reuse saves.
size_t wave_budget_bytes() {
  static const size_t v = [] {
    const char* e = std::getenv("TNBP_WAVE_MB");
    if (e && *e) return (size_t)std::strtoull(e, nullptr, 10) << 20;
    return size_t(0);
  }();
  return v;
}
// Sweep scratch a served job's plan holds at most (TNBP_SCRATCH_CAP_MB,
// default 8 GiB; the server's footprint estimate counts the same): a sweep
// whose slots exceed it (a 10x10 lattice at D = 64 holds about 140 GB of
// slots in one wave) runs in waves of this many bytes; a wave of 8 GiB still
// holds tens of site tensors at D = 64, enough work for every SM.  A job
// created on its own (tnbp_job_create) keeps one wave while its slots fit in
// half of the device memory still available (Job::scratch_limit): on the
// 16x16 D = 32 workload three 8 GiB waves made the solve 30 % slower than one.
size_t scratch_cap_bytes() {
  static const size_t v = [] {
    const char* e = std::getenv("TNBP_SCRATCH_CAP_MB");
    if (e && *e && std::strtoull(e, nullptr, 10) > 0) return (size_t)std::strtoull(e, nullptr, 10) << 20;
    return size_t(8) << 30;
  }();
  return v;
}

// Free device memory plus what the stream-ordered pool holds unused (the
// engine keeps freed blocks in the pool, see keep_pool_memory).
size_t device_bytes_available() {
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t reserved = 0, used = 0;
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  if (reserved > used) fr += (size_t)(reserved - used);
  return fr;
}

size_t Job::scratch_limit() const {
  if (scratch_cap) return scratch_cap;
  return std::max(scratch_cap_bytes(), (device_bytes_available() + ws_scratch.bytes) / 2);
}

static bool wave_budget_fixed() {
  const char* e = std::getenv("TNBP_WAVE_MB");
  return e && *e;
}

// ---------------------------------------------------------------- autotuner
// The wave budget is tuned in place, per shape class and per device: the
// first time a job of a class with a large sweep (at least 2e11 algorithmic
// flops) starts a BP loop, each candidate budget gets a plan, one warm-up
// sweep and two timed sweeps (CUDA events), all writing only the message
// arena the loop overwrites next, and the fastest is kept (a candidate must
// beat the one before it by 3 %).  The wave budget
// only groups tasks into launches; every task's kernel and arithmetic are the
// same under every budget, so tuning never changes a result.  Choices are
// kept in a table per device (name and SM count) in $TNBP_TUNE_DIR (default
// $HOME/.cache/tnbp_b200), one line per class: class, budget in MiB, best
// and default sweep ms.  TNBP_AUTOTUNE=0 turns the tuner off.
// TNBP_TUNE_LOG=1 prints every candidate's timing to stderr.
static bool tune_log_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_TUNE_LOG");
    return e && e[0] == '1';
  }();
  return on;
}

bool autotune_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_AUTOTUNE");
    return !(e && e[0] == '0');
  }();
  return on;
}

namespace {
// one wave first: the largest scratch is allocated once and every later
// candidate reuses it (the buffer only grows), so tuning does not churn the
// allocator
constexpr size_t kWaveCandidatesMb[] = {0, 32, 64, 96, 128, 192};
constexpr double kTuneMinFlops = 2e11;

struct TuneTable {
  std::mutex mu;
  std::map<int, bool> loaded;                        // per device ordinal
  std::map<int, std::map<std::string, size_t>> mb;   // device -> class -> MiB
  std::map<int, std::string> path;
};
TuneTable& tune_table() {
  static TuneTable t;
  return t;
}

std::string tune_file(int dev) {
  cudaDeviceProp p{};
  CK(cudaGetDeviceProperties(&p, dev));
  std::string name(p.name);
  for (char& c : name)
    if (!std::isalnum((unsigned char)c)) c = '_';
  std::string dir;
  if (const char* d = std::getenv("TNBP_TUNE_DIR")) dir = d;
  else if (const char* h = std::getenv("HOME")) dir = std::string(h) + "/.cache/tnbp_b200";
  else dir = "/tmp/tnbp_b200";
  return dir + "/waves_" + name + "_" + std::to_string(p.multiProcessorCount) + "sm.tsv";
}

// Loads the device's table once (caller holds the mutex).
std::map<std::string, size_t>& device_table(int dev) {
  TuneTable& T = tune_table();
  if (!T.loaded[dev]) {
    T.loaded[dev] = true;
    T.path[dev] = tune_file(dev);
    std::ifstream f(T.path[dev]);
    std::string key;
    size_t mb = 0;
    double best = 0, dflt = 0;
    while (f >> key >> mb >> best >> dflt) T.mb[dev][key] = mb;
  }
  return T.mb[dev];
}
}  // namespace

// Shape class of a job: precision, largest bond dimension, largest site
// degree and the site count rounded up to a power of two.
std::string Job::tune_key() const {
  int maxd = 1, maxg = 0;
  for (int d : dim) maxd = std::max(maxd, d);
  for (auto& l : g.legs) maxg = std::max(maxg, (int)l.size());
  size_t ns = 1;
  while (ns < g.labels.size()) ns <<= 1;
  const char* pn = prec == TNBP_C128 ? "c128" : prec == TNBP_C64 ? "c64" : "mixed";
  return std::string(pn) + "_D" + std::to_string(maxd) + "_g" + std::to_string(maxg) + "_n" + std::to_string(ns);
}

void Job::choose_wave_budget() {
  wave_budget = wave_budget_bytes();
  if (wave_budget_fixed() || !autotune_enabled()) return;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  TuneTable& T = tune_table();
  std::lock_guard<std::mutex> lk(T.mu);
  auto& tab = device_table(dev);
  auto it = tab.find(tune_key());
  if (it != tab.end()) wave_budget = it->second << 20;
}

void Job::autotune_waves() {
  if (wave_budget_fixed() || !autotune_enabled() || plan.flops < kTuneMinFlops) return;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const std::string key = tune_key();
  {
    TuneTable& T = tune_table();
    std::lock_guard<std::mutex> lk(T.mu);
    if (device_table(dev).count(key)) return;
  }
  TNBP_TRACE_SCOPE("sweep.autotune");
  struct Flag {
    bool& f;
    explicit Flag(bool& x) : f(x) { f = true; }
    ~Flag() { f = false; }
  } flag(tuning);
  double best_ms = INFINITY, default_ms = INFINITY;
  size_t best_mb = wave_budget_bytes() >> 20;
  for (size_t mb : kWaveCandidatesMb) {
    wave_budget = mb << 20;
    destroy_graphs();
    plan = SweepPlan();
    build_plan();
    run_sweep(cur);  // warm-up (and graph capture); the state is unchanged
    double ms = 0.0;
    for (int rep = 0; rep < 2; ++rep) {
      run_sweep(cur);
      CK(cudaStreamSynchronize(stream));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev0, ev1));
      ms += t;
    }
    if (reduced_sweeps(prec)) check_tc_error(stream);
    ms /= 2.0;
    if (tune_log_enabled())
      std::fprintf(stderr, "tnbp autotune %s: wave budget %zu MiB (0 = one wave), %zu waves, %.3f ms per sweep\n",
                   key.c_str(), mb, plan.waves.size(), ms);
    if (mb == (wave_budget_bytes() >> 20)) default_ms = ms;
    // a later (smaller) budget must be 3 % faster to replace an earlier one:
    // two timed sweeps do not resolve smaller differences
    if (ms < 0.97 * best_ms) { best_ms = ms; best_mb = mb; }
  }
  wave_budget = best_mb << 20;
  destroy_graphs();
  plan = SweepPlan();
  TuneTable& T = tune_table();
  std::lock_guard<std::mutex> lk(T.mu);
  device_table(dev)[key] = best_mb;
  const std::string& path = T.path[dev];
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    // create the directory chain (best effort: an unwritable cache only
    // means the tuning is redone by the next process)
    for (size_t i = 1; i <= slash; ++i)
      if (path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
  }
  std::ofstream f(path, std::ios::app);
  if (f) f << key << '\t' << best_mb << '\t' << best_ms << '\t' << default_ms << '\n';
}

void Job::build_plan() {
  TNBP_TRACE_SCOPE("sweep.build_plan");
  {
    TNBP_TRACE_SCOPE("sweep.build_plan.release");
    destroy_graphs();
    plan = SweepPlan();
  }
  const int ns = (int)g.labels.size();
  const int ne = (int)g.edges.size();
  // 1. each site's tree, split into its units
  std::vector<std::vector<int>> result(ns);
  std::vector<Unit> units;
  std::vector<int> small_sites;
  for (int s = 0; s < ns; ++s) {
    const int gs = (int)g.legs[s].size();
    if (site_whole(s)) {
      small_sites.push_back(s);
      continue;
    }
    std::vector<PlanOp> ops;
    SitePlanner sp;
    sp.site = s;
    sp.ops = &ops;
    sp.result.assign(gs, -1);
    sp.result_unit.assign(gs, 0);
    std::vector<int> targets(gs);
    std::iota(targets.begin(), targets.end(), 0);
    sp.rec(-1, 0, -1, targets, std::vector<char>(gs, 0), gs);
    result[s] = sp.result;
    const auto sh = site_shape(s);
    // the last absorption of a target runs fused with its Gram on tcgen05
    // (complex64 sweeps, both dims <= 32); decided from this job alone
    auto fuse = [&](int t, int w) {
      return reduced_sweeps(prec) && tcgen05_enabled() && leg_gram_enabled() && tc::leg_gram_ok(sh[t], sh[w]);
    };
    const int nunits = gs >= 2 ? 2 : 1;
    for (int u = 0; u < nunits; ++u) units.push_back(make_unit(s, u, ops, sp, fuse));
  }
  // 2. waves of consecutive units within the byte budget (at least one unit)
  if (!tuning) choose_wave_budget();
  size_t cap = 0;
  {
    TNBP_TRACE_SCOPE("sweep.build_plan.scratch_limit");
    cap = scratch_limit();
  }
  const size_t budget = wave_budget && wave_budget < cap ? wave_budget : cap;
  std::vector<std::vector<int>> waves;
  {
    size_t bytes = 0;
    int last_site = -1;
    for (size_t i = 0; i < units.size(); ++i) {
      const Unit& U = units[i];
      const size_t site_b = align_elems(site_elems(U.site)) * wsz;
      const size_t add = (size_t)U.nbuf * site_b + (U.site == last_site ? 0 : site_b);
      if (waves.empty() || (budget && bytes + add > budget && !waves.back().empty())) {
        waves.emplace_back();
        bytes = site_b + (size_t)U.nbuf * site_b;
      } else {
        bytes += add;
      }
      waves.back().push_back((int)i);
      last_site = U.site;
    }
  }
  // 3. slot buffers: a wave's units side by side, every wave at offset 0
  std::vector<size_t> unit_base(units.size(), 0);
  size_t scratch = 0;
  for (auto& w : waves) {
    size_t o = 0;
    for (int ui : w) {
      unit_base[ui] = o;
      o += (size_t)units[ui].nbuf * align_elems(site_elems(units[ui].site));
    }
    scratch = std::max(scratch, o);
  }
  {
    TNBP_TRACE_SCOPE("sweep.build_plan.scratch_alloc");
    ws_scratch.ensure(std::max<size_t>(scratch, 32) * wsz, stream);
  }
  auto slot_ptr = [&](int ui, int slot) -> void* {
    const Unit& U = units[ui];
    if (slot < 0) return sweep_vptr(U.site);
    return static_cast<char*>(ws_scratch.p) +
           (unit_base[ui] + (size_t)U.buf_of_slot.at(slot) * align_elems(site_elems(U.site))) * wsz;
  };
  // 4. tasks
  plan.flops = 0.0;
  plan.bytes_alg = 0.0;
  for (int s = 0; s < ns; ++s) {
    const auto sh = site_shape(s);
    const int gs = (int)g.legs[s].size();
    const double n = (double)site_elems(s);
    double sumD = 0;
    for (int k = 0; k < gs; ++k) sumD += sh[k];
    // algorithmic work of bp.h's schedule: 8 d prod(D) sum(D) flops per message
    plan.flops += gs * 8.0 * n * sumD;
    plan.bytes_alg += n * wsz;  // each site tensor read once (as the sweep reads it)
    for (int t = 0; t < gs; ++t) plan.bytes_alg += 2.0 * sh[t] * sh[t] * esz;  // message in + out
  }
  plan.waves.assign(waves.size(), WaveHost());
  size_t max_part = 1;
  struct Pending { int s, t; size_t part_off; int nchunk, C; };
  std::vector<Pending> pend;      // one per target, in message order
  std::vector<size_t> gram_part;  // pend index of each plain Gram task
  std::vector<size_t> lg_part;    // pend index of each fused task
  for (size_t w = 0; w < waves.size(); ++w) {
    WaveHost& W = plan.waves[w];
    int nlev = 0;
    for (int ui : waves[w]) nlev = std::max(nlev, units[ui].nlevels);
    W.levels.assign(nlev, LevelHost());
    size_t part = 0;
    for (int ui : waves[w]) {
      const Unit& U = units[ui];
      const auto sh = site_shape(U.site);
      for (const auto& op : U.ops) {
        long long L = 1, R = 1;
        for (int k = 0; k < op.leg; ++k) L *= sh[k];
        for (size_t k = op.leg + 1; k < sh.size(); ++k) R *= sh[k];
        for (int par = 0; par < 2; ++par) {
          LegTask lt;
          lt.in = slot_ptr(ui, op.src);
          lt.out = slot_ptr(ui, op.dst);
          lt.mat = mptr(par, g.in_msg(op.site, op.leg));
          lt.L = L; lt.R = R; lt.Din = sh[op.leg]; lt.Dout = sh[op.leg];
          set_leg_divisors(lt);
          lt.block_begin = 0;  // assigned when a batch is built
          W.levels[op.level].tasks[par].push_back(lt);
        }
      }
      for (int t : U.targets) {
        GramTask g1;
        g1.A = slot_ptr(ui, result[U.site][t]);
        g1.B = sweep_vptr(U.site);
        long long L = 1, M = 1;
        for (int k = 0; k < t; ++k) L *= sh[k];
        for (size_t k = t + 1; k < sh.size(); ++k) M *= sh[k];
        g1.L = L; g1.M = M; g1.D = sh[t]; g1.P = 1; g1.C = sh[t];
        g1.ctiles = (g1.C + kColTile - 1) / kColTile;
        g1.Q = L * M;
        // chunks of about Q/16 rows (multiples of 64, 256..4096): FP64
        // partials of one sweep stay a small fraction of its traffic, and
        // one wave of all sites gives every SM work.  The chunking does not
        // depend on the wave budget, so neither does the rounding.
        long long cr = ((g1.Q / 16) + 63) / 64 * 64;
        cr = std::max<long long>(256, std::min<long long>(4096, cr));
        g1.chunk_rows = cr;
        g1.nchunk = (int)((g1.Q + cr - 1) / cr);
        g1.partial = nullptr;
        g1.block_begin = 0;
        W.grams.push_back((int)plan.gram.size());
        W.msgs.push_back((int)pend.size());
        gram_part.push_back(pend.size());
        pend.push_back({U.site, t, part, g1.nchunk, g1.C});
        part += (size_t)g1.nchunk * g1.C * g1.C;
        plan.gram.push_back(g1);
        plan.gram_blocks.push_back((long long)g1.nchunk * g1.ctiles * g1.ctiles);
      }
      for (const auto& f : U.fused) {
        const int t = f.target, w2 = f.leg, p1 = std::min(t, w2), p2 = std::max(t, w2);
        long long L1 = 1, Mid = 1, R = 1;
        for (int k = 0; k < p1; ++k) L1 *= sh[k];
        for (int k = p1 + 1; k < p2; ++k) Mid *= sh[k];
        for (size_t k = p2 + 1; k < sh.size(); ++k) R *= sh[k];
        LegGramTask lg;
        lg.X = slot_ptr(ui, f.src);
        lg.V = sweep_vptr(U.site);
        lg.E = nullptr;  // per parity below
        lg.st = 1; lg.sw = 1;
        for (int k = 0; k < t; ++k) lg.st *= sh[k];
        for (int k = 0; k < w2; ++k) lg.sw *= sh[k];
        lg.L1 = L1; lg.Mid = Mid;
        lg.s_mid = L1 * sh[p1];
        lg.s_r = L1 * sh[p1] * Mid * sh[p2];
        lg.n_outer = L1 * Mid * R;
        lg.Dt = sh[t]; lg.Dw = sh[w2];
        // thread order along the unit-stride index: c (t = leg 0), j
        // (w = leg 0) or the outer index
        lg.mode = t == 0 ? 0 : (w2 == 0 ? 1 : 2);
        const long long tiles = (lg.n_outer + tc::kLgOuter - 1) / tc::kLgOuter;
        lg.chunk_tiles = (int)std::max<long long>(1, std::min<long long>(16, tiles / 128));
        lg.nchunk = (int)((tiles + lg.chunk_tiles - 1) / lg.chunk_tiles);
        lg.partial = nullptr;
        lg.block_begin = 0;
        W.lgs.push_back((int)plan.lg[0].size());
        W.msgs.push_back((int)pend.size());
        lg_part.push_back(pend.size());
        pend.push_back({U.site, t, part, lg.nchunk, lg.Dt});
        part += (size_t)lg.nchunk * lg.Dt * lg.Dt;
        for (int par = 0; par < 2; ++par) {
          LegGramTask l2 = lg;
          l2.E = mptr(par, g.in_msg(U.site, w2));
          plan.lg[par].push_back(l2);
        }
      }
    }
    max_part = std::max(max_part, part);
  }
  // Gram partials are finalized at the end of their wave, so one wave's
  // worth of partials is enough
  plan.partial.alloc(max_part * sizeof(double2), stream);
  plan.dist.alloc(std::max<size_t>(2 * ne, 1) * sizeof(double), stream);
  for (int par = 0; par < 2; ++par) plan.site[par].clear();
  for (int s : small_sites) {
    const auto sh = site_shape(s);
    const int gs = (int)g.legs[s].size();
    for (int par = 0; par < 2; ++par) {
      SiteTask st{};
      st.V = sweep_vptr(s);
      st.g = gs;
      st.d = pd[s];
      st.n = (int)site_elems(s);
      for (int k = 0; k < gs; ++k) {
        const int mo = g.out_msg(s, k);
        st.D[k] = sh[k];
        st.E[k] = mptr(par, g.in_msg(s, k));
        st.out[k] = mptr(1 - par, mo);
        st.old[k] = mptr(par, mo);
        st.dist[k] = static_cast<double*>(plan.dist.p) + mo;
      }
      plan.site[par].push_back(st);
    }
  }
  double2* partial = static_cast<double2*>(plan.partial.p);
  for (size_t i = 0; i < plan.gram.size(); ++i) plan.gram[i].partial = partial + pend[gram_part[i]].part_off;
  for (size_t i = 0; i < lg_part.size(); ++i)
    for (int par = 0; par < 2; ++par) plan.lg[par][i].partial = partial + pend[lg_part[i]].part_off;
  for (int par = 0; par < 2; ++par) plan.msg[par].clear();
  for (size_t i = 0; i < pend.size(); ++i) {
    const int mo = g.out_msg(pend[i].s, pend[i].t);
    for (int par = 0; par < 2; ++par) {
      MsgTask m;
      m.partial = partial + pend[i].part_off;
      m.nchunk = pend[i].nchunk;
      m.C = pend[i].C;
      m.out = mptr(1 - par, mo);
      m.old = mptr(par, mo);
      m.dist = static_cast<double*>(plan.dist.p) + mo;
      m.norm_out = nullptr;
      plan.msg[par].push_back(m);
    }
  }
  plan.valid = true;
  static std::atomic<uint64_t> serials{0};
  plan_serial = ++serials;
  // the per-job launch sequences (plan.single) are built on first use: a
  // served job only ever runs inside batches.  Every allocation above is
  // stream-ordered and every upload is staged before it returns, so no
  // synchronization is needed here.
  check_budget();
}

// Concatenate the sweep tasks of several jobs (each at its own message
// parity) into one launch sequence: wave k of the batch holds wave k of
// every job, block offsets are re-based so uneven jobs share every launch,
// and all task arrays go to the device in one copy.
void build_batch(const std::vector<BatchEntry>& entries, SweepBatch& b, cudaStream_t stream) {
  TNBP_TRACE_SCOPE("sweep.build_batch");
  b.reset_graph();
  b.launches.clear();
  size_t nw = 0;
  for (auto& e : entries) {
    if (!e.job->plan.valid) e.job->build_plan();
    nw = std::max(nw, e.job->plan.waves.size());
  }
  std::vector<unsigned char> host;
  auto put = [&](const void* p, size_t bytes) -> size_t {
    const size_t off = (host.size() + 255) & ~size_t(255);
    host.resize(off + std::max<size_t>(bytes, 16));
    if (bytes) std::memcpy(host.data() + off, p, bytes);
    return off;
  };
  auto add = [&](int kind, const auto& tasks, const std::vector<long long>& begins, long long nblocks, int max_din) {
    if (tasks.empty()) return;
    SweepLaunch L;
    L.kind = kind;
    L.tasks_off = put(tasks.data(), tasks.size() * sizeof(tasks[0]));
    L.begins_off = begins.empty() ? 0 : put(begins.data(), begins.size() * sizeof(long long));
    L.ntask = (int)tasks.size();
    L.nblocks = nblocks;
    L.max_din = max_din;
    b.launches.push_back(L);
  };
  // The kernel is chosen per task, never per launch: complex64 tasks whose
  // tile is a contiguous byte range (tc::bulk_mode) run on the bulk-staged
  // tcgen05 kernel, other tasks with Din, Dout <= 32 on the register-staged
  // tcgen05 kernel, every other task on the CUDA-core kernel, whatever else
  // shares the batch.  A request's rounding therefore does not depend on
  // what it is batched with.
  const bool tc_ok = !entries.empty() && reduced_sweeps(entries[0].job->prec) && tcgen05_enabled();
  {
    // small sites: one CTA each, every message of the site on chip
    std::vector<SiteTask> sts;
    size_t smem = 0;
    for (auto& e : entries)
      for (const SiteTask& st : e.job->plan.site[e.parity]) {
        sts.push_back(st);
        smem = std::max(smem, site_sweep_smem_bytes(st.D, st.g, st.d));
      }
    add(SweepLaunch::SITE, sts, {}, (long long)sts.size(), (int)smem);
  }
  for (size_t w = 0; w < nw; ++w) {
    size_t nlev = 0;
    for (auto& e : entries)
      if (w < e.job->plan.waves.size()) nlev = std::max(nlev, e.job->plan.waves[w].levels.size());
    for (size_t lv = 0; lv < nlev; ++lv) {
      std::vector<LegTask> t, t2, t3, t4;
      std::vector<long long> beg, b2, b3, b4;
      long long nb = 0, nb2 = 0, nb3 = 0, nb4 = 0;
      int maxdin = 1;
      for (auto& e : entries) {
        const auto& P = e.job->plan;
        if (w >= P.waves.size() || lv >= P.waves[w].levels.size()) continue;
        for (LegTask lt : P.waves[w].levels[lv].tasks[e.parity]) {
          if (tc_ok && bulk_leg_enabled() && tc::bulk_mode(lt.L, lt.Din, lt.Dout) != 0) {
            lt.block_begin = nb3;
            b3.push_back(nb3);
            nb3 += (lt.L * lt.R + tc::kTcRows - 1) / tc::kTcRows;
            t3.push_back(lt);
          } else if (tc_ok && tc::leg64_ok(lt.Din, lt.Dout)) {
            lt.block_begin = nb4;
            b4.push_back(nb4);
            nb4 += (lt.L * lt.R + tc::kTcRows - 1) / tc::kTcRows;
            t4.push_back(lt);
          } else if (tc_ok && lt.Din <= tc::kTcMaxD && lt.Dout <= tc::kTcMaxD) {
            lt.block_begin = nb2;
            b2.push_back(nb2);
            nb2 += (lt.L * lt.R + tc::kTcRows - 1) / tc::kTcRows;
            t2.push_back(lt);
          } else {
            lt.block_begin = nb;
            beg.push_back(nb);
            nb += (lt.L * lt.R + kRowTile - 1) / kRowTile;
            maxdin = std::max(maxdin, lt.Din);
            t.push_back(lt);
          }
        }
      }
      add(SweepLaunch::LEG_BULK, t3, b3, nb3, 0);
      add(SweepLaunch::LEG_T64, t4, b4, nb4, 0);
      add(SweepLaunch::LEG_TC, t2, b2, nb2, 0);
      add(SweepLaunch::LEG_CORE, t, beg, nb, maxdin);
    }
    // Gram tasks: the fused absorption + Gram kernel, then per task the
    // tcgen05 kernels (one CTA per chunk) for the complex64 sweeps with C <=
    // 64, else the CUDA-core kernel; then the wave's messages are finalized
    std::vector<GramTask> gt, gt2, gt3;
    std::vector<long long> gb, gb2, gb3, lb;
    std::vector<LegGramTask> lt;
    std::vector<MsgTask> mt;
    long long nb = 0, nb2 = 0, nb3 = 0, nlb = 0;
    for (auto& e : entries) {
      const auto& P = e.job->plan;
      if (w >= P.waves.size()) continue;
      for (int li : P.waves[w].lgs) {
        LegGramTask l1 = P.lg[e.parity][li];
        l1.block_begin = nlb;
        lb.push_back(nlb);
        nlb += l1.nchunk;
        lt.push_back(l1);
      }
      for (int mi : P.waves[w].msgs) mt.push_back(P.msg[e.parity][mi]);
      for (int gi : P.waves[w].grams) {
        GramTask g1 = P.gram[gi];
        if (tc_ok && tc::gram_tc_ok(g1.C, g1.P)) {
          g1.block_begin = nb2;
          gb2.push_back(nb2);
          nb2 += g1.nchunk;
          gt2.push_back(g1);
        } else if (tc_ok && tc::gram64_ok(g1.C, g1.P)) {
          g1.block_begin = nb3;
          gb3.push_back(nb3);
          nb3 += g1.nchunk;
          gt3.push_back(g1);
        } else {
          g1.block_begin = nb;
          gb.push_back(nb);
          nb += P.gram_blocks[gi];
          gt.push_back(g1);
        }
      }
    }
    add(SweepLaunch::LEG_GRAM, lt, lb, nlb, 0);
    add(SweepLaunch::GRAM_TC, gt2, gb2, nb2, 0);
    add(SweepLaunch::GRAM_T64, gt3, gb3, nb3, 0);
    add(SweepLaunch::GRAM_CORE, gt, gb, nb, 0);
    add(SweepLaunch::MSG, mt, {}, (long long)mt.size(), 0);
  }
  // one condition per job
  b.cond.ensure(std::max<size_t>(entries.size(), 1) * sizeof(double), stream);
  std::vector<SumTask> st;
  for (size_t ei = 0; ei < entries.size(); ++ei) {
    const auto& P = entries[ei].job->plan;
    SumTask s1;
    s1.x = static_cast<const double*>(P.dist.p);
    s1.n = (int)(2 * entries[ei].job->g.edges.size());  // every message's distance
    s1.scale = 1.0 / (2.0 * (double)entries[ei].job->g.edges.size());
    s1.out = static_cast<double*>(b.cond.p) + ei;
    st.push_back(s1);
  }
  add(SweepLaunch::SUM, st, {}, (long long)st.size(), 0);
  b.arena.ensure(std::max<size_t>(host.size(), 256), stream);
  CK(cudaMemcpyAsync(b.arena.p, host.data(), host.size(), cudaMemcpyHostToDevice, stream));
  b.nkernels = (int)b.launches.size();
}

template <typename R>
static size_t leg_smem(int max_din) {
  return (size_t)(kRowTile * (max_din + 1) + max_din * (kColTile + 1)) * sizeof(typename cvec<R>::type);
}

// Largest dynamic shared memory any leg-apply launch may ask for.
template <typename R, typename MR>
static void leg_apply_attr() {
  static std::vector<char> flags;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (attr_done(flags)) return;
  CK(cudaFuncSetAttribute(k_leg_apply<R, MR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)leg_smem<R>(128)));
  CK(cudaFuncSetAttribute(k_site_sweep<R, MR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSiteSmemMax));
  attr_mark(flags);
}

template <typename R, typename MR>
static int launch_batch_t(const SweepBatch& b, cudaStream_t stream) {
  const char* base = static_cast<const char*>(b.arena.p);
  for (const SweepLaunch& L : b.launches) {
    const void* tasks = base + L.tasks_off;
    const long long* begins = reinterpret_cast<const long long*>(base + L.begins_off);
    switch (L.kind) {
      case SweepLaunch::LEG_BULK: {
        // persistent: one CTA per SM (about 193 KB of shared memory each)
        const long long grid = std::min<long long>(L.nblocks, num_sms());
        k_leg_apply_tc_bulk<MR><<<(unsigned)grid, 256, tc::bulk_smem_bytes(), stream>>>(
            static_cast<const LegTask*>(tasks), begins, L.ntask, L.nblocks);
        break;
      }
      case SweepLaunch::LEG_T64: {
        // persistent: one 256-thread CTA per SM (about 193 KB of shared memory)
        const long long grid = std::min<long long>(L.nblocks, num_sms());
        k_leg_apply_tc64<MR><<<(unsigned)grid, 256, tc::leg64_smem_bytes(), stream>>>(
            static_cast<const LegTask*>(tasks), begins, L.ntask, L.nblocks);
        break;
      }
      case SweepLaunch::LEG_TC: {
        // persistent: up to 2 CTAs per SM, each over a contiguous range of tiles
        const long long grid = std::min<long long>(L.nblocks, 2LL * num_sms());
        k_leg_apply_tc<MR><<<(unsigned)grid, 128, tc::leg_smem_bytes(), stream>>>(
            static_cast<const LegTask*>(tasks), begins, L.ntask, L.nblocks);
        break;
      }
      case SweepLaunch::LEG_CORE: {
        if (L.max_din > 128) throw Error(TNBP_EUNSUPPORTED, "bond dimension above 128 during BP");
        k_leg_apply<R, MR><<<(unsigned)L.nblocks, kThreads, leg_smem<R>(L.max_din), stream>>>(
            static_cast<const LegTask*>(tasks), begins, L.ntask, L.max_din);
        break;
      }
      case SweepLaunch::GRAM_TC:
        k_gram_tc<<<(unsigned)L.nblocks, 256, tc::gram_smem_bytes(), stream>>>(
            static_cast<const GramTask*>(tasks), begins, L.ntask);
        break;
      case SweepLaunch::GRAM_T64:
        k_gram_tc64<<<(unsigned)L.nblocks, 256, tc::gram64_smem_bytes(), stream>>>(
            static_cast<const GramTask*>(tasks), begins, L.ntask);
        break;
      case SweepLaunch::LEG_GRAM:
        k_leg_gram_tc<MR><<<(unsigned)L.nblocks, 256, tc::leg_gram_smem_bytes(), stream>>>(
            static_cast<const LegGramTask*>(tasks), begins, L.ntask);
        break;
      case SweepLaunch::GRAM_CORE:
        k_gram<R><<<(unsigned)L.nblocks, kThreads, 0, stream>>>(static_cast<const GramTask*>(tasks), begins, L.ntask);
        break;
      case SweepLaunch::MSG:
        k_msg_finalize<R, MR><<<L.ntask, kThreads, 0, stream>>>(static_cast<const MsgTask*>(tasks));
        break;
      case SweepLaunch::SITE:  // max_din holds the launch's shared memory bytes
        k_site_sweep<R, MR><<<L.ntask, kThreads, (size_t)L.max_din, stream>>>(static_cast<const SiteTask*>(tasks));
        break;
      case SweepLaunch::SUM:
        k_segmented_sum<<<L.ntask, kThreads, 0, stream>>>(static_cast<const SumTask*>(tasks));
        break;
    }
    CK(cudaGetLastError());
  }
  return (int)b.launches.size();
}

// Sweep kernels: TNBP_C128 all complex128; TNBP_C64 all complex64;
// TNBP_MIXED complex64 tensors with complex128 messages.
int launch_batch(const SweepBatch& b, int prec, cudaStream_t stream) {
  if (prec == TNBP_C128) return launch_batch_t<double, double>(b, stream);
  if (prec == TNBP_C64) return launch_batch_t<float, float>(b, stream);
  return launch_batch_t<float, double>(b, stream);
}

template <typename MR>
static void tc_attr() {
  static std::vector<char> flags, gram_flags;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (attr_done(flags)) return;
  CK(cudaFuncSetAttribute(k_leg_apply_tc<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)tc::leg_smem_bytes()));
  CK(cudaFuncSetAttribute(k_leg_apply_tc_bulk<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)tc::bulk_smem_bytes()));
  CK(cudaFuncSetAttribute(k_leg_apply_tc64<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)tc::leg64_smem_bytes()));
  CK(cudaFuncSetAttribute(k_leg_gram_tc<MR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)tc::leg_gram_smem_bytes()));
  if (!attr_done(gram_flags)) {
    CK(cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::gram_smem_bytes()));
    CK(cudaFuncSetAttribute(k_gram_tc64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)tc::gram64_smem_bytes()));
    attr_mark(gram_flags);
  }
  attr_mark(flags);
}

void prepare_kernels(int prec) {
  if (prec == TNBP_C128) {
    leg_apply_attr<double, double>();
  } else if (prec == TNBP_C64) {
    leg_apply_attr<float, float>();
    tc_attr<float>();
  } else {
    leg_apply_attr<float, double>();
    tc_attr<double>();
  }
}

int num_sms() {
  static std::vector<int> per_dev;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if ((int)per_dev.size() <= dev) per_dev.resize(dev + 1, 0);
  if (!per_dev[dev]) CK(cudaDeviceGetAttribute(&per_dev[dev], cudaDevAttrMultiProcessorCount, dev));
  return per_dev[dev];
}

// The tcgen05 leg kernel serves complex64 levels with dims <= 32; setting
// TNBP_DISABLE_TCGEN05=1 routes them to the CUDA-core kernel instead (both do
// the full contraction; used to compare the two).
bool tcgen05_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_DISABLE_TCGEN05");
    return !(e && e[0] == '1');
  }();
  return on;
}

// The bulk-staged leg kernel (k_leg_apply_tc_bulk) is selected with
// TNBP_LEG_BULK=1.  Default: the register-staged kernel, measured faster on
// the 16x16 D = 32 sweep (30.9 ms vs 33.2 ms): with its 224 KB of shared
// memory the bulk kernel runs one CTA per SM and is bound by the bytes it
// keeps in flight, the register-staged one runs two.
bool bulk_leg_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_LEG_BULK");
    return e && e[0] == '1';
  }();
  return on;
}

// TNBP_LEG_GRAM=1 runs the last absorption of every target with dims <= 32
// fused with its Gram (k_leg_gram_tc) on the reduced-precision paths; by
// default those targets use the separate leg and Gram kernels, which
// measured faster (16x16 D = 32 sweep in one wave: 25.5 ms separate, 34.7
// ms fused).  Both compute the same contraction.
bool leg_gram_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_LEG_GRAM");
    return e && e[0] == '1';
  }();
  return on;
}

// Every site whose tensor, two work buffers, messages and Gram partials fit
// kSiteSmemMax of shared memory is swept whole by one CTA (k_site_sweep);
// the other sites take the per-level path.  Measured on the random-circuit
// workload (10x10, BP at D <= 8): BP loops 4.6-5.7 ms per solve against
// 23-33 ms per-level (mixed), 4.9-6.3 against 8.0-8.5 ms (complex128); the
// 16x16 headline unchanged within run-to-run noise.  TNBP_SITE_SWEEP=0
// sends every site to the per-level path.
bool site_sweep_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_SITE_SWEEP");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool Job::site_whole(int s) const {
  const int gs = (int)g.legs[s].size();
  if (!site_sweep_enabled() || gs < 1 || gs > kMaxLegs) return false;
  const auto sh = site_shape(s);
  return site_sweep_smem_bytes(sh.data(), gs, pd[s]) <= kSiteSmemMax;
}

// A tcgen05 CTA that gave up waiting for its MMAs records it in g_tc_error.
void check_tc_error(cudaStream_t stream) {
  int err = 0;
  CK(cudaMemcpyFromSymbolAsync(&err, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (err) {
    const int zero = 0;
    CK(cudaMemcpyToSymbolAsync(g_tc_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    throw Error(TNBP_ECUDA, "a tcgen05 tile reached its wait limit (MMA completion not observed)");
  }
}

// A sweep's launch sequence (one per message-arena parity) runs kernel by
// kernel on its first kEagerSweeps uses and is captured as a CUDA graph on
// the next, then relaunched as that graph.  Shapes change at every AbsorbTPO
// and truncation, so a plan lives for one BP loop: on small lattices (the
// random-circuit workload's BP at D <= 4, two or three sweeps per loop)
// capturing both parities at once cost more host time (about 0.3 ms per
// capture) than the sweeps themselves.
constexpr int kEagerSweeps = 2;

void Job::run_sweep(int par) {
  sync_shadow();
  if (!plan.valid) build_plan();
  SweepBatch& b = plan.single[par];
  if (b.launches.empty()) build_batch({{this, par}}, b, stream);
  if (!b.graph && b.uses < kEagerSweeps) {
    prepare_kernels(prec);
    CK(cudaEventRecord(ev0, stream));
    note_launch(launch_batch(b, prec, stream));
    CK(cudaEventRecord(ev1, stream));
    ++b.uses;
    last_par = par;
    sweeps_run++;
    return;
  }
  if (!b.graph) {
    TNBP_TRACE_SCOPE("sweep.graph_capture");
    prepare_kernels(prec);
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      b.nkernels = launch_batch(b, prec, stream);
    } catch (...) {
      cudaStreamEndCapture(stream, &graph);
      throw;
    }
    CK(cudaStreamEndCapture(stream, &graph));
    CK(cudaGraphInstantiate(&b.graph, graph, 0));
    cudaGraphDestroy(graph);
  }
  CK(cudaEventRecord(ev0, stream));
  CK(cudaGraphLaunch(b.graph, stream));
  note_launch(b.nkernels);
  CK(cudaEventRecord(ev1, stream));
  ++b.uses;
  last_par = par;
  sweeps_run++;
}

double Job::read_cond() {
  TNBP_TRACE_SCOPE("sweep.cond_wait");
  CK(cudaMemcpyAsync(host_scalar, plan.single[last_par].cond.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (reduced_sweeps(prec)) check_tc_error(stream);
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) {
    last_sweep_ms = ms;
    total_sweep_ms += ms;
    total_sweep_flops += plan.flops;
    total_sweep_bytes += plan.bytes_alg;
    ++timed_sweeps;
  }
  return host_scalar[0];
}
void Job::bp_sweep() {
  run_sweep(cur);
  cur = 1 - cur;
  CK(cudaStreamSynchronize(stream));
  if (reduced_sweeps(prec)) check_tc_error(stream);
}

double Job::bp_condition() {
  run_sweep(cur);  // writes the other arena; state (cur) unchanged
  return read_cond();
}

// The condition of the complex64 path cannot go below its rounding floor
// (about 1e-7 per sweep for normalized messages); a tolerance under the
// floor would run every sweep to max_iter and let unstable BP modes grow
// from rounding noise.  The mixed path therefore stops at
// max(tol, kC64TolFloor) (1e-7: a floor of 1e-6 left the messages about
// 1e-6 from the fixed point and the expectation values as far from the
// plain path's).
double effective_tol(int prec, double tol) {
  return reduced_sweeps(prec) ? std::max(tol, kC64TolFloor) : tol;
}

// The mixed path also stops when the condition grows once it is within two
// decades of its rounding floor (prev < kC64GrowthGate): past the minimum
// the unstable BP mode amplifies rounding noise every sweep.  Growth at
// larger conditions is ordinary BP dynamics, which the plain path sees too,
// and does not stop the loop.  The plain path keeps the reference's rule
// exactly.
bool stop_on_growth(int prec, double prev, double c) {
  return reduced_sweeps(prec) && prev < kC64GrowthGate && c > prev;
}

void Job::bp_run(double tol_in, int max_iter, int* iters, double* cond) {
  TNBP_TRACE_SCOPE("bp_run");
  const double tol = effective_tol(prec, tol_in);
  *iters = 0;
  *cond = std::nan("");
  if (max_iter <= 0) return;
  sync_shadow();
  if (!plan.valid) build_plan();
  autotune_waves();
  run_sweep(cur);
  cur = 1 - cur;
  *iters = 1;
  double prev = INFINITY;
  while (true) {
    run_sweep(cur);
    const double c = read_cond();
    *cond = c;
    if (!std::isfinite(c)) throw Error(TNBP_ENOTCONV, "BP condition is not finite (non-finite messages)");
    if (c < tol) break;
    if (*iters >= max_iter) break;
    if (stop_on_growth(prec, prev, c)) break;
    prev = c;
    cur = 1 - cur;
    ++*iters;
  }
}

// --------------------------------------------------------------- AbsorbTPO
Tpo::~Tpo() {}

void Job::absorb_tpo(const Tpo& tpo) {
  TNBP_TRACE_SCOPE("absorb");
  shadow_dirty = true;
  const int ns = (int)g.labels.size();
  const int ne = (int)g.edges.size();
  if ((int)tpo.rank.size() != ne) throw Error(TNBP_EINVAL, "TPO edge count mismatch");
  std::vector<int> ndim(ne);
  for (int e = 0; e < ne; ++e) ndim[e] = dim[e] * tpo.rank[e];
  const std::vector<int> odim = dim;
  const std::vector<size_t> ovoff = voff, omoff = moff;
  // new layout
  dim = ndim;
  layout();
  DevBuf nM0, nM1;
  DevBuf& nV = Vspare;
  nV.ensure(v_elems * esz, stream);
  nM0.alloc(m_elems * esz, stream);
  nM1.alloc(m_elems * esz, stream);
  std::vector<AbsorbTask> at;
  std::vector<long long> ab;
  long long nb = 0;
  for (int s = 0; s < ns; ++s) {
    AbsorbTask t{};
    t.V = static_cast<char*>(V.p) + ovoff[s] * esz;
    t.out = static_cast<char*>(nV.p) + voff[s] * esz;
    t.O = static_cast<const double2*>(tpo.ops.p) + tpo.op_offset[s];
    t.g = (int)g.legs[s].size();
    t.d = pd[s];
    t.dout = tpo.dout[s];
    for (int k = 0; k < t.g; ++k) {
      t.Dv[k] = odim[g.legs[s][k]];
      t.r[k] = tpo.rank[g.legs[s][k]];
      t.div_m[k] = make_fastdiv((uint32_t)(t.Dv[k] * t.r[k]));
      t.div_v[k] = make_fastdiv((uint32_t)t.Dv[k]);
    }
    t.n_out = (long long)site_elems(s);
    if (t.n_out >= (1ll << 31)) throw Error(TNBP_EUNSUPPORTED, "site tensor of 2^31 or more elements");
    t.block_begin = nb;
    ab.push_back(nb);
    nb += (t.n_out + kThreads - 1) / kThreads;
    at.push_back(t);
  }
  std::vector<MsgExpandTask> mt;
  std::vector<long long> mb;
  long long nmb = 0;
  for (int m = 0; m < 2 * ne; ++m) {
    MsgExpandTask t;
    t.E = static_cast<char*>(M[cur].p) + omoff[m] * esz;
    t.out = static_cast<char*>(nM0.p) + moff[m] * esz;
    t.D = odim[m % ne];
    t.r = tpo.rank[m % ne];
    t.block_begin = nmb;
    mb.push_back(nmb);
    const long long N = (long long)t.D * t.r;
    nmb += (N * N + kThreads - 1) / kThreads;
    mt.push_back(t);
  }
  DevBuf dat, dab, dmt, dmb;
  upload_vec(dat, at, stream);
  upload_vec(dab, ab, stream);
  upload_vec(dmt, mt, stream);
  upload_vec(dmb, mb, stream);
  if (sprec == TNBP_C128) {
    (k_absorb_sites<double><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<AbsorbTask*>(dat.p), static_cast<long long*>(dab.p), (int)at.size()), note_launch());
    (k_expand_msgs<double><<<(unsigned)nmb, kThreads, 0, stream>>>(static_cast<MsgExpandTask*>(dmt.p), static_cast<long long*>(dmb.p), (int)mt.size()), note_launch());
  } else {
    (k_absorb_sites<float><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<AbsorbTask*>(dat.p), static_cast<long long*>(dab.p), (int)at.size()), note_launch());
    (k_expand_msgs<float><<<(unsigned)nmb, kThreads, 0, stream>>>(static_cast<MsgExpandTask*>(dmt.p), static_cast<long long*>(dmb.p), (int)mt.size()), note_launch());
  }
  CK(cudaGetLastError());
  std::swap(V, nV);
  std::swap(M[0], nM0);
  std::swap(M[1], nM1);
  cur = 0;
  plan.valid = false;
  destroy_graphs();
  plan = SweepPlan();
  CK(cudaStreamSynchronize(stream));
  check_budget();
}

// ------------------------------------------------- generic leg-apply helper
// Applies, for every entry, a chain of leg contractions to a site tensor and
// writes the result to dst.  Used by truncation (projectors) and
// measurement (incoming messages).
struct ChainEntry {
  int site;
  const void* src;
  void* dst;                        // final output
  std::vector<int> legs;            // legs to contract, in order
  std::vector<const void*> mats;    // Din x Dout matrices (storage precision)
  std::vector<int> dout;            // output dims
};

// Chain buffer capacity: chains run in batches whose intermediates fit in
// this many bytes per buffer, so that truncating a large lattice (2 x 35 GB
// of intermediates for a 10x10 lattice at D = 64 in complex128) needs two
// bounded buffers instead.
size_t chain_cap_bytes() { return size_t(8) << 30; }

void Job::run_chains(std::vector<ChainEntry>& chains) {
  TNBP_TRACE_SCOPE("chains");
  if (chains.empty()) return;
  // largest intermediate of each chain (its input and final output live
  // outside the chain buffers)
  std::vector<size_t> inter(chains.size(), 0);
  for (size_t i = 0; i < chains.size(); ++i) {
    auto sh = site_shape(chains[i].site);
    size_t n = site_elems(chains[i].site);
    for (size_t k = 0; k + 1 < chains[i].legs.size(); ++k) {
      n = n / sh[chains[i].legs[k]] * chains[i].dout[k];
      sh[chains[i].legs[k]] = chains[i].dout[k];
      inter[i] = std::max(inter[i], n);
    }
  }
  const size_t cap = chain_cap_bytes() / esz;
  DevBuf* buf = ws_chain;
  for (size_t i0 = 0; i0 < chains.size();) {
    // the next batch: chains [i0, i1) whose intermediates fit one buffer
    // (a single chain larger than the cap runs alone)
    std::vector<size_t> base;
    size_t tot = 0, i1 = i0, maxlen = 0;
    while (i1 < chains.size() && (i1 == i0 || tot + align_elems(inter[i1]) <= cap)) {
      base.push_back(tot);
      tot += align_elems(inter[i1]);
      maxlen = std::max(maxlen, chains[i1].legs.size());
      ++i1;
    }
    buf[0].ensure(std::max<size_t>(tot, 32) * esz, stream);
    buf[1].ensure(std::max<size_t>(tot, 32) * esz, stream);
    for (size_t lv = 0; lv < maxlen; ++lv) {
      std::vector<LegTask> t;
      std::vector<long long> b;
      long long nb = 0;
      int maxdin = 1;
      for (size_t i = i0; i < i1; ++i) {
        auto& c = chains[i];
        if (lv >= c.legs.size()) continue;
        auto sh = site_shape(c.site);
        for (size_t k = 0; k < lv; ++k) sh[c.legs[k]] = c.dout[k];
        const int leg = c.legs[lv];
        long long L = 1, R = 1;
        for (int k = 0; k < leg; ++k) L *= sh[k];
        for (size_t k = leg + 1; k < sh.size(); ++k) R *= sh[k];
        LegTask lt;
        lt.in = lv == 0 ? c.src : static_cast<char*>(buf[(lv - 1) & 1].p) + base[i - i0] * esz;
        lt.out = (lv + 1 == c.legs.size()) ? c.dst : static_cast<char*>(buf[lv & 1].p) + base[i - i0] * esz;
        lt.mat = c.mats[lv];
        lt.L = L; lt.R = R; lt.Din = sh[leg]; lt.Dout = c.dout[lv];
        set_leg_divisors(lt);
        lt.block_begin = nb;
        b.push_back(nb);
        nb += (L * R + kRowTile - 1) / kRowTile;
        maxdin = std::max(maxdin, lt.Din);
        t.push_back(lt);
      }
      DevBuf dt, db;
      upload_vec(dt, t, stream);
      upload_vec(db, b, stream);
      if (maxdin > 128) throw Error(TNBP_EUNSUPPORTED, "bond dimension above 128");
      prepare_kernels(sprec);
      if (sprec == TNBP_C128) {
        const size_t smem = leg_smem<double>(maxdin);
        (k_leg_apply<double><<<(unsigned)nb, kThreads, smem, stream>>>(static_cast<LegTask*>(dt.p), static_cast<long long*>(db.p), (int)t.size(), maxdin), note_launch());
      } else {
        const size_t smem = leg_smem<float>(maxdin);
        (k_leg_apply<float><<<(unsigned)nb, kThreads, smem, stream>>>(static_cast<LegTask*>(dt.p), static_cast<long long*>(db.p), (int)t.size(), maxdin), note_launch());
      }
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(stream));
    }
    i0 = i1;
  }
}

// --------------------------------------------------------------- truncation
void Job::truncate(int chi_max, double sv_min, int32_t* dims_out, double* err_out) {
  TNBP_TRACE_SCOPE("truncate");
  shadow_dirty = true;
  if (chi_max < 1) throw Error(TNBP_EINVAL, "chi_max must be >= 1");
  const int ns = (int)g.labels.size();
  const int ne = (int)g.edges.size();
  // per-edge scratch
  std::vector<size_t> woff(ne), poff(ne), soff(ne);
  size_t wtot = 0, ptot = 0, stot = 0;
  for (int e = 0; e < ne; ++e) {
    const size_t nn = (size_t)dim[e] * dim[e];
    woff[e] = wtot; wtot += 8 * nn;
    poff[e] = ptot; ptot += align_elems(nn);
    soff[e] = stot; stot += (size_t)dim[e];
  }
  DevBuf work, sv, perm, Pa, Pb, skeep, keep, err, status;
  work.alloc(wtot * sizeof(double2), stream);
  sv.alloc(3 * stot * sizeof(double), stream);
  perm.alloc(3 * stot * sizeof(int), stream);
  Pa.alloc(ptot * esz, stream);
  Pb.alloc(ptot * esz, stream);
  skeep.alloc(stot * sizeof(double), stream);
  keep.alloc(ne * sizeof(int), stream);
  err.alloc(ne * sizeof(double), stream);
  status.alloc(ne * sizeof(int), stream);
  std::vector<TruncTask> tt(ne);
  for (int e = 0; e < ne; ++e) {
    TruncTask& t = tt[e];
    t.Ma = mptr(cur, e);
    t.Mb = mptr(cur, e + ne);
    t.D = dim[e];
    t.work = static_cast<double2*>(work.p) + woff[e];
    t.sv = static_cast<double*>(sv.p) + 3 * soff[e];
    t.perm = static_cast<int*>(perm.p) + 3 * soff[e];
    t.Pa = static_cast<char*>(Pa.p) + poff[e] * esz;
    t.Pb = static_cast<char*>(Pb.p) + poff[e] * esz;
    t.s_keep = static_cast<double*>(skeep.p) + soff[e];
    t.keep_out = static_cast<int*>(keep.p) + e;
    t.err_out = static_cast<double*>(err.p) + e;
    t.status = static_cast<int*>(status.p) + e;
  }
  DevBuf dtt;
  upload_vec(dtt, tt, stream);
  if (sprec == TNBP_C128) (k_truncate_edges<double><<<ne, kThreads, 0, stream>>>(static_cast<TruncTask*>(dtt.p), chi_max, sv_min), note_launch());
  else (k_truncate_edges<float><<<ne, kThreads, 0, stream>>>(static_cast<TruncTask*>(dtt.p), chi_max, sv_min), note_launch());
  CK(cudaGetLastError());
  std::vector<int> hkeep(ne), hstatus(ne);
  std::vector<double> herr(ne);
  {
    TNBP_TRACE_SCOPE("truncate.svd_wait");
    CK(cudaMemcpyAsync(hkeep.data(), keep.p, ne * sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(herr.data(), err.p, ne * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(hstatus.data(), status.p, ne * sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  // new site tensors: V_s x_k P_k for every leg, then normalize
  const std::vector<int> odim = dim;
  const std::vector<size_t> ovoff = voff;
  dim.assign(hkeep.begin(), hkeep.end());
  layout();
  DevBuf& nV = Vspare;
  nV.ensure(v_elems * esz, stream);
  std::vector<ChainEntry> chains;
  {
    const std::vector<int> ndim = dim;
    dim = odim;  // site_shape() inside run_chains must see the old dims
    std::vector<size_t> nvoff = voff;
    for (int s = 0; s < ns; ++s) {
      ChainEntry c;
      c.site = s;
      c.src = static_cast<char*>(V.p) + ovoff[s] * esz;
      c.dst = static_cast<char*>(nV.p) + nvoff[s] * esz;
      for (size_t k = 0; k < g.legs[s].size(); ++k) {
        const int e = g.legs[s][k];
        c.legs.push_back((int)k);
        c.mats.push_back(static_cast<char*>(g.site_a[e] == s ? Pa.p : Pb.p) + poff[e] * esz);
        c.dout.push_back(ndim[e]);
      }
      chains.push_back(c);
    }
    run_chains(chains);
    dim = ndim;
    voff = nvoff;
  }
  std::swap(V, nV);
  normalize_sites();
  // messages = diag(s)
  DevBuf nM0, nM1;
  nM0.alloc(m_elems * esz, stream);
  nM1.alloc(m_elems * esz, stream);
  std::vector<DiagTask> dt;
  for (int m = 0; m < 2 * ne; ++m) {
    DiagTask t;
    t.s = static_cast<double*>(skeep.p) + soff[m % ne];
    t.out = static_cast<char*>(nM0.p) + moff[m] * esz;
    t.n = dim[m % ne];
    dt.push_back(t);
  }
  DevBuf ddt;
  upload_vec(ddt, dt, stream);
  if (sprec == TNBP_C128) (k_write_diag<double><<<2 * ne, 128, 0, stream>>>(static_cast<DiagTask*>(ddt.p)), note_launch());
  else (k_write_diag<float><<<2 * ne, 128, 0, stream>>>(static_cast<DiagTask*>(ddt.p)), note_launch());
  CK(cudaGetLastError());
  std::swap(M[0], nM0);
  std::swap(M[1], nM1);
  cur = 0;
  plan.valid = false;
  destroy_graphs();
  plan = SweepPlan();
  // no synchronization: the kept dims and errors are already on the host,
  // the buffers above are freed in stream order and the uploads were staged
  // before they returned, so the host goes on while the projectors run
  if (dims_out) for (int e = 0; e < ne; ++e) dims_out[e] = hkeep[e];
  if (err_out) for (int e = 0; e < ne; ++e) err_out[e] = herr[e];
  int bad = 0, nonfinite = 0;
  for (int e = 0; e < ne; ++e) {
    bad += hstatus[e] == 1;
    nonfinite += hstatus[e] == 2;
  }
  if (nonfinite)
    throw Error(TNBP_ENOTCONV, std::to_string(nonfinite) + " edge(s) with non-finite messages at truncation");
  if (bad) throw Error(TNBP_ENOTCONV, std::to_string(bad) + " edge SVD(s) reached the Jacobi sweep limit");
  check_budget();
}

void Job::normalize_sites() {
  TNBP_TRACE_SCOPE("normalize");
  shadow_dirty = true;
  const int ns = (int)g.labels.size();
  const int per_thread = 8;
  std::vector<RangeTask> rt;
  std::vector<long long> rb;
  long long nb = 0;
  size_t npart = 0;
  for (int s = 0; s < ns; ++s) {
    RangeTask t;
    t.data = vptr(s);
    t.n = (long long)site_elems(s);
    t.nblocks = (int)((t.n + (long long)kThreads * per_thread - 1) / ((long long)kThreads * per_thread));
    t.block_begin = nb;
    t.partial = reinterpret_cast<double*>(npart);  // patched below
    rb.push_back(nb);
    nb += t.nblocks;
    npart += t.nblocks;
    rt.push_back(t);
  }
  DevBuf part;
  part.alloc(npart * sizeof(double), stream);
  for (auto& t : rt) t.partial = static_cast<double*>(part.p) + reinterpret_cast<size_t>(t.partial);
  DevBuf drt, drb;
  upload_vec(drt, rt, stream);
  upload_vec(drb, rb, stream);
  if (sprec == TNBP_C128) {
    (k_sumsq_partial<double><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<RangeTask*>(drt.p), static_cast<long long*>(drb.p), ns, per_thread), note_launch());
    (k_scale_ranges<double><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<RangeTask*>(drt.p), static_cast<long long*>(drb.p), ns, per_thread), note_launch());
  } else {
    (k_sumsq_partial<float><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<RangeTask*>(drt.p), static_cast<long long*>(drb.p), ns, per_thread), note_launch());
    (k_scale_ranges<float><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<RangeTask*>(drt.p), static_cast<long long*>(drb.p), ns, per_thread), note_launch());
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(stream));
}

// -------------------------------------------------------------- measurement
// Environments of single sites as FP64 Gram matrices: for request r,
//   W = V_site with a matrix absorbed on every leg except keep_leg (the
//       incoming BP message, or r.mats[k] when that is set: a D x D matrix in
//       storage precision applied as W[..j..] = sum_i V[..i..] M[i, j]),
//   env[(t + D p), (t' + D p')] = sum_x W[x, t, p] conj(V[x, t', p'])
// over the kept leg t (D = its dimension) and the physical leg p; with
// keep_leg = -1 every bond leg is absorbed and env is the d x d one-site
// rho.  Outputs are packed in request order; off[i] is request i's offset
// (double2 elements).
void Job::env_grams(const std::vector<EnvReq>& reqs, DevBuf& out, std::vector<size_t>& off) {
  std::vector<size_t> woff(reqs.size());
  size_t wtot = 0;
  for (size_t i = 0; i < reqs.size(); ++i) { woff[i] = wtot; wtot += align_elems(site_elems(reqs[i].site)); }
  DevBuf W;
  W.alloc(std::max<size_t>(wtot, 32) * esz, stream);
  std::vector<ChainEntry> chains;
  std::vector<size_t> copy_only;
  for (size_t i = 0; i < reqs.size(); ++i) {
    ChainEntry c;
    c.site = reqs[i].site;
    c.src = vptr(c.site);
    c.dst = static_cast<char*>(W.p) + woff[i] * esz;
    const auto sh = site_shape(c.site);
    for (size_t k = 0; k < g.legs[c.site].size(); ++k) {
      if ((int)k == reqs[i].keep_leg) continue;
      const void* m = k < reqs[i].mats.size() ? reqs[i].mats[k] : nullptr;
      c.legs.push_back((int)k);
      c.mats.push_back(m ? m : mptr(cur, g.in_msg(c.site, (int)k)));
      c.dout.push_back(sh[k]);
    }
    if (c.legs.empty()) copy_only.push_back(i);
    else chains.push_back(c);
  }
  for (size_t i : copy_only)
    CK(cudaMemcpyAsync(static_cast<char*>(W.p) + woff[i] * esz, vptr(reqs[i].site), site_elems(reqs[i].site) * esz,
                       cudaMemcpyDeviceToDevice, stream));
  run_chains(chains);
  // Gram partials
  std::vector<GramTask> gt;
  std::vector<long long> gb;
  std::vector<PartialSumTask> pt;
  long long nb = 0;
  size_t ptot = 0, otot = 0;
  std::vector<size_t> poff;
  off.clear();
  for (size_t i = 0; i < reqs.size(); ++i) {
    const int s = reqs[i].site;
    const auto sh = site_shape(s);
    const int gs = (int)g.legs[s].size();
    GramTask t;
    t.A = static_cast<char*>(W.p) + woff[i] * esz;
    t.B = vptr(s);
    if (reqs[i].keep_leg < 0) {
      long long L = 1;
      for (int k = 0; k < gs; ++k) L *= sh[k];
      t.L = L; t.M = 1; t.D = sh[gs]; t.P = 1;
    } else {
      const int kl = reqs[i].keep_leg;
      long long L = 1, M = 1;
      for (int k = 0; k < kl; ++k) L *= sh[k];
      for (int k = kl + 1; k < gs; ++k) M *= sh[k];
      t.L = L; t.M = M; t.D = sh[kl]; t.P = sh[gs];
    }
    t.C = t.D * t.P;
    t.ctiles = (t.C + kColTile - 1) / kColTile;
    t.Q = t.L * t.M;
    long long cr = ((t.Q / 16) + kRowTile - 1) / kRowTile * kRowTile;
    t.chunk_rows = std::max<long long>(256, std::min<long long>(4096, cr));
    t.nchunk = (int)((t.Q + t.chunk_rows - 1) / t.chunk_rows);
    t.block_begin = nb;
    gb.push_back(nb);
    nb += (long long)t.nchunk * t.ctiles * t.ctiles;
    poff.push_back(ptot);
    ptot += (size_t)t.nchunk * t.C * t.C;
    off.push_back(otot);
    otot += (size_t)t.C * t.C;
    gt.push_back(t);
  }
  DevBuf part;
  part.alloc(std::max<size_t>(ptot, 1) * sizeof(double2), stream);
  out.alloc(std::max<size_t>(otot, 1) * sizeof(double2), stream);
  for (size_t i = 0; i < gt.size(); ++i) {
    gt[i].partial = static_cast<double2*>(part.p) + poff[i];
    PartialSumTask p;
    p.partial = gt[i].partial;
    p.nchunk = gt[i].nchunk;
    p.n = gt[i].C * gt[i].C;
    p.out = static_cast<double2*>(out.p) + off[i];
    pt.push_back(p);
  }
  DevBuf dgt, dgb, dpt;
  upload_vec(dgt, gt, stream);
  upload_vec(dgb, gb, stream);
  upload_vec(dpt, pt, stream);
  if (!gt.empty()) {
    if (sprec == TNBP_C128) (k_gram<double><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<GramTask*>(dgt.p), static_cast<long long*>(dgb.p), (int)gt.size()), note_launch());
    else (k_gram<float><<<(unsigned)nb, kThreads, 0, stream>>>(static_cast<GramTask*>(dgt.p), static_cast<long long*>(dgb.p), (int)gt.size()), note_launch());
    CK(cudaGetLastError());
    (k_partial_sum<<<(unsigned)pt.size(), kThreads, 0, stream>>>(static_cast<PartialSumTask*>(dpt.p)), note_launch());
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(stream));
}

// Reduced density matrices: one-site rho over the physical leg
// (measure.h:46-89), two-site environments over (target leg, physical leg)
// (measure.h:168-245).  Returns device buffers holding FP64 matrices.
void Job::compute_envs(const std::vector<int>& sites1, const std::vector<std::pair<int, int>>& sidelegs,
                       DevBuf& out1, DevBuf& out2, std::vector<size_t>& off2) {
  std::vector<EnvReq> r1, r2;
  for (int s : sites1) r1.push_back({s, -1, {}});
  for (auto& p : sidelegs) r2.push_back({p.first, p.second, {}});
  std::vector<size_t> off1;
  env_grams(r1, out1, off1);
  env_grams(r2, out2, off2);
}

void Job::measure_terms(const std::vector<TermSpec>& terms, double* values, double* sum) {
  TNBP_TRACE_SCOPE("measure");
  // distinct one-site requests and two-site sides
  std::vector<int> sites1;
  std::map<int, int> pos1;
  std::vector<std::pair<int, int>> sides;
  std::map<std::pair<int, int>, int> pos2;
  struct Where { int a, b, edge; };
  std::vector<Where> where(terms.size());
  for (size_t i = 0; i < terms.size(); ++i) {
    const auto& t = terms[i];
    if (t.kind == 1) {
      if (!pos1.count(t.site_a)) { pos1[t.site_a] = (int)sites1.size(); sites1.push_back(t.site_a); }
    } else {
      const int e = t.edge;
      const std::pair<int, int> sa{g.site_a[e], g.leg_a[e]}, sb{g.site_b[e], g.leg_b[e]};
      if (!pos2.count(sa)) { pos2[sa] = (int)sides.size(); sides.push_back(sa); }
      if (!pos2.count(sb)) { pos2[sb] = (int)sides.size(); sides.push_back(sb); }
    }
  }
  DevBuf r1, r2;
  std::vector<size_t> off2;
  compute_envs(sites1, sides, r1, r2, off2);
  std::vector<TermTask> tt(terms.size());
  for (size_t i = 0; i < terms.size(); ++i) {
    const auto& t = terms[i];
    TermTask& k = tt[i];
    k.kind = t.kind;
    k.coeff = make_double2(t.coeff[0], t.coeff[1]);
    for (int j = 0; j < 16; ++j) k.op[j] = make_double2(t.op[2 * j], t.op[2 * j + 1]);
    if (t.kind == 1) {
      k.d = pd[t.site_a];
      k.D = 1;
      size_t off = 0;
      for (int q = 0; q < pos1[t.site_a]; ++q) off += (size_t)pd[sites1[q]] * pd[sites1[q]];
      k.rho_a = static_cast<const double2*>(r1.p) + off;
      k.rho_b = nullptr;
    } else {
      const int e = t.edge;
      // measure.h:126-127: site a = first label of the requested pair
      const bool flip = g.labels[g.site_a[e]] != t.label_a;
      const std::pair<int, int> sa{g.site_a[e], g.leg_a[e]}, sb{g.site_b[e], g.leg_b[e]};
      const auto& A = flip ? sb : sa;
      const auto& B = flip ? sa : sb;
      k.d = pd[A.first];
      k.D = dim[e];
      k.rho_a = static_cast<const double2*>(r2.p) + off2[pos2[A]];
      k.rho_b = static_cast<const double2*>(r2.p) + off2[pos2[B]];
    }
  }
  DevBuf dtt, dvals, dsum;
  upload_vec(dtt, tt, stream);
  dvals.alloc(std::max<size_t>(terms.size(), 1) * sizeof(double2), stream);
  dsum.alloc(sizeof(double2), stream);
  if (!tt.empty()) {
    (k_terms<<<(unsigned)tt.size(), kThreads, 0, stream>>>(static_cast<TermTask*>(dtt.p), static_cast<double2*>(dvals.p)), note_launch());
    (k_weighted_sum<<<1, kThreads, 0, stream>>>(static_cast<TermTask*>(dtt.p), static_cast<double2*>(dvals.p), (int)tt.size(), static_cast<double2*>(dsum.p)), note_launch());
    CK(cudaGetLastError());
  }
  std::vector<double> hv(2 * std::max<size_t>(terms.size(), 1), 0.0);
  double hs[2] = {0.0, 0.0};
  if (!tt.empty()) {
    CK(cudaMemcpyAsync(hv.data(), dvals.p, terms.size() * sizeof(double2), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(hs, dsum.p, sizeof(double2), cudaMemcpyDeviceToHost, stream));
  }
  CK(cudaStreamSynchronize(stream));
  if (values) std::memcpy(values, hv.data(), terms.size() * 2 * sizeof(double));
  if (sum) { sum[0] = hs[0]; sum[1] = hs[1]; }
}

// Pauli products on any set of distinct sites -- the terms ClassifyOps drops
// (paulitotpo.h:111-132: pairs that are not adjacent, three or more qubits)
// -- measured on a tree cluster T: the union of the shortest paths
// (FindShortestPath, graph.h:57-108) from the lowest-numbered qubit's site to
// every other qubit's site (so the cluster does not depend on the order in
// which a term lists its qubits).  T's ket and bra layers, the term's Pauli on its qubit
// sites and the incoming BP messages on every leg that leaves T are
// contracted leaf to root: a tree site absorbs its children's results on
// their legs (as BP messages are absorbed) and BP messages on its other
// legs; its Gram environment over (leg toward its parent, physical leg)
// contracted with its one-site operator is its result X[t, t'].  At the root,
// its environment toward its first child, contracted with its operator,
// meets that child's result: Z = sum_{t,t'} X_child[t,t'] X_root[t,t'], the
// pairing of the two-site measurement (measure.h:255-294).  The value is
// Z(P) / Z(identity).  On a tree graph BP messages are exact environments,
// so the value is exact there; for an adjacent pair it is the two-site
// measurement.  Tree levels of every term are batched into shared launches.
void Job::measure_clusters(const std::vector<ClusterTerm>& terms, double* values, double* sum) {
  TNBP_TRACE_SCOPE("measure.clusters");
  struct Node {
    int site;
    int parent = -1;      // node index
    int parent_leg = -1;  // leg of this site toward its parent
    std::vector<int> children;
    std::vector<int> child_leg;  // leg of this site toward each child
    char letter = 'I';
    int height = 0;
  };
  const auto leg_of = [&](int s, int e) {
    const auto& L = g.legs[s];
    return (int)(std::find(L.begin(), L.end(), e) - L.begin());
  };
  std::vector<std::vector<Node>> trees(terms.size());
  int max_height = 0;
  for (size_t i = 0; i < terms.size(); ++i) {
    if (terms[i].labels.size() < 2 || terms[i].labels.size() != terms[i].letters.size())
      throw Error(TNBP_EINVAL, "a cluster term needs two or more qubits, one letter each");
    ClusterTerm t = terms[i];  // qubits in ascending order: the first is the root
    {
      std::vector<std::pair<int, char>> q;
      for (size_t k = 0; k < t.labels.size(); ++k) q.push_back({t.labels[k], t.letters[k]});
      std::stable_sort(q.begin(), q.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      for (size_t k = 0; k < q.size(); ++k) { t.labels[k] = q[k].first; t.letters[k] = q[k].second; }
    }
    auto& nodes = trees[i];
    std::map<int, int> node_of;  // site -> node
    for (size_t k = 0; k < t.labels.size(); ++k) {
      auto it = g.index_of.find(t.labels[k]);
      if (it == g.index_of.end())
        throw Error(TNBP_EINVAL, "term on qubit " + std::to_string(t.labels[k]) + " outside the graph");
      if (pd[it->second] != 2) throw Error(TNBP_EUNSUPPORTED, "cluster terms need physical dimension 2");
      const char l = t.letters[k];
      if (l != 'X' && l != 'Y' && l != 'Z' && l != 'I') throw Error(TNBP_EINVAL, "Pauli letters are I, X, Y, Z");
      const auto path = tnbp_host::shortest_path(g.edges, t.labels[0], t.labels[k]);
      if (path.empty()) throw Error(TNBP_EINVAL, "term qubits in different components of the graph");
      int prev = -1;
      for (size_t j = 0; j < path.size(); ++j) {
        const int s = g.index_of.at(path[j]);
        auto nt = node_of.find(s);
        if (nt == node_of.end()) {
          Node n;
          n.site = s;
          if (prev >= 0) {
            const int e = edge_of(g.labels[nodes[prev].site], path[j]);
            n.parent = prev;
            n.parent_leg = leg_of(s, e);
            nodes[prev].children.push_back((int)nodes.size());
            nodes[prev].child_leg.push_back(leg_of(nodes[prev].site, e));
          }
          node_of[s] = (int)nodes.size();
          nodes.push_back(n);
          prev = (int)nodes.size() - 1;
        } else {
          if (prev >= 0 && nodes[nt->second].parent != prev)
            throw Error(TNBP_EUNSUPPORTED, "shortest paths from the first qubit do not form a tree");
          prev = nt->second;
        }
      }
      Node& q = nodes[node_of.at(g.index_of.at(t.labels[k]))];
      if (q.letter != 'I' || (k > 0 && q.site == nodes[0].site)) throw Error(TNBP_EINVAL, "repeated qubit in a term");
      q.letter = l == 'I' ? 'i' : l;  // 'i': named identity, still a qubit of the term
    }
    // heights: children are created after their parents
    for (int n = (int)nodes.size() - 1; n >= 0; --n)
      for (int c : nodes[n].children) nodes[n].height = std::max(nodes[n].height, nodes[c].height + 1);
    max_height = std::max(max_height, nodes[0].height);
  }
  // result slots: per (term, chain, node), D x D with D the dimension of the
  // edge toward the parent (the root: toward its first child)
  const auto slot_dim = [&](const std::vector<Node>& nodes, int n) {
    const Node& nd = nodes[n];
    const int leg = nd.parent >= 0 ? nd.parent_leg : nd.child_leg[0];
    return dim[g.legs[nd.site][leg]];
  };
  std::vector<std::vector<size_t>> off(2 * terms.size());
  size_t tot = 0;
  for (size_t i = 0; i < terms.size(); ++i)
    for (int ch = 0; ch < 2; ++ch) {
      auto& o = off[2 * i + ch];
      for (size_t n = 0; n < trees[i].size(); ++n) {
        o.push_back(tot);
        const size_t D = (size_t)slot_dim(trees[i], (int)n);
        tot += align_elems(D * D);
      }
    }
  DevBuf xs, x64, zbuf;
  xs.alloc(std::max<size_t>(tot, 32) * esz, stream);
  x64.alloc(std::max<size_t>(tot, 32) * sizeof(double2), stream);
  zbuf.alloc(std::max<size_t>(2 * terms.size(), 1) * sizeof(double2), stream);
  const auto pauli_op = [](char l, double2* op) {
    const auto P = tnbp_host::pauli_list(l == 'i' ? 'I' : l);
    for (int k = 0; k < 4; ++k) op[k] = make_double2(P[k].real(), P[k].imag());
  };
  // levels 0 .. max_height; the roots are done at their own height
  for (int h = 0; h <= max_height; ++h) {
    std::vector<EnvReq> reqs;
    struct Out { size_t term; int ch; int node; };
    std::vector<Out> outs;
    for (size_t i = 0; i < terms.size(); ++i)
      for (int ch = 0; ch < 2; ++ch)
        for (size_t n = 0; n < trees[i].size(); ++n) {
          const Node& nd = trees[i][n];
          if (nd.height != h) continue;
          EnvReq r;
          r.site = nd.site;
          const bool root = nd.parent < 0;
          r.keep_leg = root ? nd.child_leg[0] : nd.parent_leg;
          r.mats.assign(g.legs[nd.site].size(), nullptr);
          for (size_t c = root ? 1 : 0; c < nd.children.size(); ++c)
            r.mats[nd.child_leg[c]] = static_cast<char*>(xs.p) + off[2 * i + ch][nd.children[c]] * esz;
          reqs.push_back(r);
          outs.push_back({i, ch, (int)n});
        }
    if (reqs.empty()) continue;
    DevBuf env;
    std::vector<size_t> eoff;
    env_grams(reqs, env, eoff);
    std::vector<EnvOpTask> et(reqs.size());
    for (size_t k = 0; k < reqs.size(); ++k) {
      const Out& o = outs[k];
      const Node& nd = trees[o.term][o.node];
      EnvOpTask& t = et[k];
      t.env = static_cast<const double2*>(env.p) + eoff[k];
      t.D = slot_dim(trees[o.term], o.node);
      t.d = 2;
      pauli_op(o.ch == 0 ? nd.letter : 'I', t.op);
      t.out64 = static_cast<double2*>(x64.p) + off[2 * o.term + o.ch][o.node];
      t.out = nd.parent >= 0 ? static_cast<char*>(xs.p) + off[2 * o.term + o.ch][o.node] * esz : nullptr;
    }
    DevBuf det;
    upload_vec(det, et, stream);
    if (sprec == TNBP_C128) (k_env_op<double><<<(unsigned)et.size(), kThreads, 0, stream>>>(static_cast<EnvOpTask*>(det.p)), note_launch());
    else (k_env_op<float><<<(unsigned)et.size(), kThreads, 0, stream>>>(static_cast<EnvOpTask*>(det.p)), note_launch());
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream));
  }
  // the root meets its first child
  std::vector<PairTask> pt;
  for (size_t i = 0; i < terms.size(); ++i)
    for (int ch = 0; ch < 2; ++ch) {
      const auto& nodes = trees[i];
      const int D = slot_dim(nodes, 0);
      PairTask p;
      p.a = static_cast<const double2*>(x64.p) + off[2 * i + ch][nodes[0].children[0]];
      p.b = static_cast<const double2*>(x64.p) + off[2 * i + ch][0];
      p.n = D * D;
      p.out = static_cast<double2*>(zbuf.p) + 2 * i + ch;
      pt.push_back(p);
    }
  std::vector<double> z(4 * std::max<size_t>(terms.size(), 1), 0.0);
  if (!pt.empty()) {
    DevBuf dpt;
    upload_vec(dpt, pt, stream);
    (k_pair_dot<<<(unsigned)pt.size(), kThreads, 0, stream>>>(static_cast<PairTask*>(dpt.p)), note_launch());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(z.data(), zbuf.p, 2 * terms.size() * sizeof(double2), cudaMemcpyDeviceToHost, stream));
  }
  CK(cudaStreamSynchronize(stream));
  double sr = 0.0, si = 0.0;
  for (size_t i = 0; i < terms.size(); ++i) {
    const std::complex<double> zp(z[4 * i], z[4 * i + 1]), zi(z[4 * i + 2], z[4 * i + 3]);
    const std::complex<double> v = zp / zi;
    if (values) { values[2 * i] = v.real(); values[2 * i + 1] = v.imag(); }
    const std::complex<double> c = std::complex<double>(terms[i].coeff[0], terms[i].coeff[1]) * v;
    sr += c.real();
    si += c.imag();
  }
  if (sum) { sum[0] = sr; sum[1] = si; }
}

int Job::edge_of(int la, int lb) const {
  auto ia = g.index_of.find(la), ib = g.index_of.find(lb);
  if (ia == g.index_of.end() || ib == g.index_of.end()) return -1;
  for (int e : g.legs[ia->second]) {
    if ((g.site_a[e] == ia->second && g.site_b[e] == ib->second) ||
        (g.site_b[e] == ia->second && g.site_a[e] == ib->second))
      return e;
  }
  return -1;
}

}  // namespace tnbp
