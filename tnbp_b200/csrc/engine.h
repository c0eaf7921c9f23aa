// Internal declarations of the device engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kernels.cuh"

namespace tnbp {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

extern thread_local std::string g_last_error;
extern std::atomic<unsigned long long> g_launches;
void check_cuda(cudaError_t e, const char* what, const char* file, int line);
#define CK(x) ::tnbp::check_cuda((x), #x, __FILE__, __LINE__)

// Stream-ordered device allocation owned by one object.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; bytes = o.bytes; stream = o.stream;
      o.p = nullptr; o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf();
  // Keep the buffer if it already holds nbytes; otherwise re-allocate
  // (stream-ordered).  Returns true if the address changed.
  bool ensure(size_t nbytes, cudaStream_t s) {
    if (p && bytes >= nbytes) return false;
    alloc(nbytes, s);
    return true;
  }
  void release();
  void alloc(size_t nbytes, cudaStream_t s);
};

// Lattice bookkeeping of graph.h: sorted site labels, incident edges per
// site in edge order (the leg order of every site tensor).
struct Graph {
  std::vector<std::pair<int, int>> edges;
  std::vector<int> labels;
  std::map<int, int> index_of;
  std::vector<std::vector<int>> legs;
  std::vector<int> site_a, site_b, leg_a, leg_b;
  Graph() = default;
  Graph(const int32_t* e, int64_t n);
  int out_msg(int s, int k) const;
  int in_msg(int s, int k) const;
};

struct LevelHost {
  std::vector<LegTask> tasks[2];  // per message-arena parity
};

// One wave of a sweep: whole half-trees ("units") of consecutive sites whose
// site tensors and intermediate slots fit a byte budget, so that a unit's
// slots are written and read back while they are still in L2.  A wave runs
// its levels in order, then its Gram tasks, then the finalization of its
// messages; the next wave reuses the same slot and partial buffers.
struct WaveHost {
  std::vector<LevelHost> levels;
  std::vector<int> grams;  // indices into SweepPlan::gram
  std::vector<int> lgs;    // indices into SweepPlan::lg
  std::vector<int> msgs;   // indices into SweepPlan::msg (one per target)
};

// One kernel launch of a sweep batch; its task arrays live in the batch's
// arena at the given byte offsets.
struct SweepLaunch {
  enum Kind { LEG_BULK, LEG_T64, LEG_TC, LEG_CORE, GRAM_TC, GRAM_T64, GRAM_CORE, LEG_GRAM, MSG, SUM, SITE };
  int kind;
  size_t tasks_off, begins_off;
  int ntask;
  long long nblocks;
  int max_din;
};

// Device task arrays of one sweep launch sequence; built from one job (the
// per-job path, captured once per parity as a CUDA graph) or from many jobs
// at once (the served path: every active job's sweep in the same launches).
struct SweepBatch {
  DevBuf arena, cond;
  std::vector<SweepLaunch> launches;
  int nkernels = 0;
  int uses = 0;  // launches of this sequence so far (eager or graph)
  cudaGraphExec_t graph = nullptr;
  SweepBatch() = default;
  SweepBatch(const SweepBatch&) = delete;
  SweepBatch& operator=(const SweepBatch&) = delete;
  SweepBatch(SweepBatch&& o) noexcept { *this = std::move(o); }
  SweepBatch& operator=(SweepBatch&& o) noexcept;
  ~SweepBatch() { reset_graph(); }
  void reset_graph();
  uint64_t bytes() const { return arena.bytes + cond.bytes; }
};

struct SweepPlan {
  bool valid = false;
  DevBuf partial, dist;
  std::vector<WaveHost> waves;
  std::vector<GramTask> gram;
  std::vector<long long> gram_blocks;  // blocks of each gram task (CUDA-core kernel)
  std::vector<LegGramTask> lg[2];      // fused last absorption + Gram, per parity
  std::vector<MsgTask> msg[2];         // one per target, per message-arena parity
  std::vector<SiteTask> site[2];       // sites swept whole on chip (k_site_sweep), per parity
  SweepBatch single[2];
  double flops = 0.0, bytes_alg = 0.0;
  SweepPlan() = default;
  SweepPlan(SweepPlan&&) = default;
  SweepPlan& operator=(SweepPlan&&) = default;
  ~SweepPlan();
  uint64_t bytes() const;
};

struct Job;
struct BatchEntry { Job* job; int parity; };
void build_batch(const std::vector<BatchEntry>& entries, SweepBatch& b, cudaStream_t stream);
int launch_batch(const SweepBatch& b, int prec, cudaStream_t stream);
void note_launch(int n = 1);
void keep_pool_memory();
constexpr double kC64TolFloor = 1e-7;
constexpr double kC64GrowthGate = 1e-5;
double effective_tol(int prec, double tol);
bool stop_on_growth(int prec, double prev, double c);
inline bool reduced_sweeps(int prec) { return prec != TNBP_C128; }
void prepare_kernels(int prec);
size_t wave_budget_bytes();
size_t scratch_cap_bytes();
size_t device_bytes_available();
size_t chain_cap_bytes();
bool autotune_enabled();
bool tcgen05_enabled();
bool bulk_leg_enabled();
bool leg_gram_enabled();
bool site_sweep_enabled();
int num_sms();
void check_tc_error(cudaStream_t stream);

// A TPO layer on the device: complex128 op tensors of shape
// (r_leg0..r_leg{g-1}, d, d') per site.
struct Tpo {
  std::vector<int> rank;          // per edge
  std::vector<int64_t> op_offset; // per site, complex elements
  std::vector<int> dout;          // per site
  DevBuf ops;
  ~Tpo();
};

struct TermSpec {
  int kind;          // 1 or 2
  int site_a;        // kind 1: site index
  int edge;          // kind 2: edge index
  int label_a;       // kind 2: label of the first operator's site
  double op[32];     // reference layout, interleaved complex
  double coeff[2];
};

struct ChainEntry;

// One environment request of Job::env_grams: keep_leg = -1 (one-site rho)
// or the bond leg left open; mats[k], when given, replaces the incoming BP
// message on leg k (a D_k x D_k matrix in storage precision).
struct EnvReq {
  int site;
  int keep_leg;
  std::vector<const void*> mats;
};

// A Pauli product on distinct sites measured on a tree cluster (see
// Job::measure_clusters).
struct ClusterTerm {
  std::vector<int> labels;  // site labels of the qubits (the lowest is the tree root)
  std::vector<char> letters;
  double coeff[2];
};

struct Job {
  Graph g;
  int prec;      // TNBP_C128, TNBP_C64 or TNBP_MIXED
  int sprec;     // storage precision: TNBP_C64 for TNBP_C64, else TNBP_C128
  size_t esz;    // bytes of a stored complex element
  size_t wsz;    // bytes of a complex element inside a BP sweep
  uint64_t budget;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double* host_scalar = nullptr;
  std::vector<int> pd, dim;
  std::vector<size_t> voff, moff;
  size_t v_elems = 0, m_elems = 0;
  DevBuf V, M[2];
  // TNBP_MIXED: complex64 copy of V read by the BP sweeps, refreshed before
  // the first sweep after V changed
  DevBuf V32;
  bool shadow_dirty = true;
  // Work buffers that only grow over the job's life, so that the Floquet
  // steps do not return and re-map gigabytes through the allocator: the
  // sweep's intermediate slots, the two chain buffers of truncation and
  // measurement, and the spare site-tensor buffer that absorption and
  // truncation write into before it is swapped with V.
  DevBuf ws_scratch, ws_chain[2], Vspare;
  int cur = 0;
  int last_par = 0;
  SweepPlan plan;
  uint64_t plan_serial = 0;  // unique per plan build (keys of the server's sweep graphs)
  size_t wave_budget = 0;    // wave byte budget of the next plan (0: one wave)
  size_t scratch_cap = 0;    // most sweep-slot bytes a plan may hold (0: from free device memory)
  bool tuning = false;       // the autotuner sets wave_budget itself
  long long sweeps_run = 0;
  float last_sweep_ms = 0.f;
  double total_sweep_ms = 0.0, total_sweep_flops = 0.0, total_sweep_bytes = 0.0;
  long long timed_sweeps = 0;

  Job(const int32_t* e, int64_t n, const int32_t* pdims, int precision, cudaStream_t s, uint64_t budget);
  ~Job();
  std::vector<int> site_shape(int s) const;
  bool site_whole(int s) const;  // swept whole on chip by k_site_sweep
  size_t site_elems(int s) const;
  void layout();
  void put_complex(DevBuf& dst, const double* src, size_t n, size_t elem_off);
  void get_complex(const DevBuf& src, double* dst, size_t n, size_t elem_off);
  uint64_t device_bytes() const;
  void check_budget() const;
  void* vptr(int s) const;
  void* sweep_vptr(int s) const;
  void sync_shadow();
  void* mptr(int arena, int m) const;
  void destroy_graphs();
  void build_plan();
  size_t scratch_limit() const;
  void run_sweep(int par);
  double read_cond();
  void bp_sweep();
  double bp_condition();
  void bp_run(double tol, int max_iter, int* iters, double* cond);
  std::string tune_key() const;
  void choose_wave_budget();
  void autotune_waves();
  void absorb_tpo(const Tpo& tpo);
  void run_chains(std::vector<ChainEntry>& chains);
  void truncate(int chi_max, double sv_min, int32_t* dims_out, double* err_out);
  void normalize_sites();
  void env_grams(const std::vector<EnvReq>& reqs, DevBuf& out, std::vector<size_t>& off);
  void measure_clusters(const std::vector<ClusterTerm>& terms, double* values, double* sum);
  void compute_envs(const std::vector<int>& sites1, const std::vector<std::pair<int, int>>& sidelegs,
                    DevBuf& out1, DevBuf& out2, std::vector<size_t>& off2);
  void measure_terms(const std::vector<TermSpec>& terms, double* values, double* sum);
  int edge_of(int la, int lb) const;
};

}  // namespace tnbp
