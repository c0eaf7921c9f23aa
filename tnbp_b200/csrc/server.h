// Continuous-batching request loop over device-resident estimator jobs.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <deque>
#include <functional>
#include <list>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"
#include "host_setup.h"

namespace tnbp {

// Device TPO layers of one circuit on one edge list, read-only and shared
// by every request built from the same circuit.
struct TpoSet {
  std::vector<std::pair<int, int>> edges;
  std::vector<std::unique_ptr<Tpo>> layers;
  std::vector<int> rank_max;  // per edge: largest TPO bond dimension of any layer
  uint64_t device_bytes = 0;
};

uint64_t footprint_estimate(const std::vector<std::pair<int, int>>& edges, const std::vector<double>& D, int prec,
                            uint64_t extra_bytes);

struct Request {
  enum Phase { QUEUED, ABSORB, BP, TRUNC, MEASURE, DONE };
  // KICKED_ISING: the one layer of tpos applied `steps` times; QASM: the
  // layers of tpos in order (steps = their number)
  enum Source { KICKED_ISING, QASM };
  Source source = KICKED_ISING;
  int64_t id = 0;
  int L = 0, chi = 0, steps = 0, maxit = 0;
  double theta_j = 0, theta_h = 0, tol = 0, sv_min = 0;
  std::vector<int32_t> kind, q0, q1;
  std::string letters;
  std::vector<double> coeff;
  Phase phase = QUEUED;
  std::unique_ptr<Job> job;
  std::shared_ptr<const TpoSet> tpos;
  int step = 0, bp_iters = 0;
  double prev_cond = 0;
  uint64_t footprint = 0;
  int prec = 0;               // precision of the request's job (the server's, or TNBP_C128 once escalated)
  bool escalated = false;     // restarted in complex128 after a BP loop that did not converge
  bool bp_converged = true;   // every BP loop of the (last) run reached its tolerance
  // BP loops of the (last) run that stopped at the iteration limit, the
  // largest final condition among them and the largest of their smallest
  // conditions (how close the closest of them came to converging)
  int unconv_loops = 0;
  double worst_final_cond = 0, worst_min_cond = 0;
  double loop_min_cond = 0;   // smallest condition of the current loop so far
  double result[2] = {0, 0};
  int error_code = 0;  // a request that failed keeps its error; others go on
  std::string error;
};

struct Server {
  int prec;
  uint64_t budget;
  // Reduced-precision server (TNBP_C64 / TNBP_MIXED): a request whose BP loop
  // ends at its iteration limit without reaching its tolerance is restarted
  // from |0...0> in complex128.  Where BP does not converge, the messages
  // after the iteration limit depend on every rounding of the earlier steps,
  // so only the complex128 run reproduces the plain path's value.
  bool escalate = false;
  // Escalate only when the non-converging loop's smallest condition is above
  // this (0: every non-converging loop).  A loop whose messages settled to a
  // small but non-zero change per sweep (a slow approach or a small limit
  // cycle) leaves them well determined, and rounding is not amplified; a
  // loop whose messages keep changing by O(1) per sweep is the
  // ill-conditioned case.
  double escalate_min_cond = 0;
  int max_active;
  cudaStream_t stream = nullptr;   // every job's own work and the server's first batch
  cudaStream_t stream2 = nullptr;  // the complex128 batch of escalated requests
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // page-locked read-back of each batch's conditions (one per batch of a step)
  struct PinnedConds {
    double* p = nullptr;
    size_t cap = 0;
  };
  PinnedConds hconds[2];
  int64_t next_id = 1;
  std::deque<int64_t> queue;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<int64_t> active;
  uint64_t in_use = 0;
  // Batched sweeps by membership: key = (plan serial, parity) of every job
  // in the batch.  A batch seen for the first time is launched kernel by
  // kernel; seen again (the same jobs, e.g. two steps later with the same
  // parities) it is captured as a CUDA graph and from then on relaunched as
  // one graph.  Least recently used entries are dropped beyond the cap.
  struct CachedSweep {
    SweepBatch batch;
    int uses = 0;
  };
  std::map<std::vector<uint64_t>, std::unique_ptr<CachedSweep>> sweeps;
  std::list<std::vector<uint64_t>> sweeps_lru;
  size_t sweeps_cap = 16;
  int64_t graph_launches = 0, eager_launches = 0;
  // TPO cache keyed by the circuit (and its TPO options), least recently
  // used evicted first; requests keep their set alive after eviction
  std::map<std::string, std::shared_ptr<const TpoSet>> tpo_cache;
  std::list<std::string> tpo_lru;
  size_t tpo_cache_cap = 32;
  int64_t cache_hits = 0, cache_misses = 0;

  Server(int precision, uint64_t budget_bytes, int max_active_jobs);
  ~Server();
  int64_t submit(std::unique_ptr<Request> r);
  std::shared_ptr<const TpoSet> tpo_set(const std::string& key,
                                        const std::function<void(tnbp_host::Edges&,
                                                                 std::vector<tnbp_host::Layer>&)>& build);
  void step(int* n_active, int* n_queued, int* n_done);
  struct GroupSweep {
    int gprec = 0;
    std::vector<Request*> reqs;
    CachedSweep* cs = nullptr;
    double* h = nullptr;
  };
  GroupSweep prepare_group(int gprec, const std::vector<Request*>& grp);
  void launch_group(GroupSweep& g, cudaStream_t s, PinnedConds& h);
  void finish_group(GroupSweep& g);
  void restart_c128(Request& r);
  uint64_t footprint(const Request& r) const;
  void start(Request& r);
  void finish(Request& r);
  void fail(Request& r, int code, const std::string& msg);
  void cancel(int64_t id);
};

}  // namespace tnbp
