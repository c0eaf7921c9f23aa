// Host-side phase timing.  With TNBP_TRACE=1 in the environment every
// TNBP_TRACE_SCOPE region adds its wall time to a per-name total, and the
// totals (calls, seconds) are printed to stderr when the process exits.
// Regions that end in a stream synchronization include the device time of
// the work they waited for.  With TNBP_NVTX=1 each region is also an NVTX
// range of the same name, so a profiler (ncu --nvtx, Nsight Systems) can
// filter and label kernels by engine phase.  Both are off by default; when
// off a scope costs one branch on a cached flag.
#pragma once
#include <chrono>

namespace tnbp {

bool trace_enabled();
bool nvtx_enabled();
void trace_add(const char* name, double seconds);
void nvtx_push(const char* name);
void nvtx_pop();

struct TraceScope {
  const char* name;
  std::chrono::steady_clock::time_point t0;
  bool on, nvtx;
  explicit TraceScope(const char* n) : name(n), on(trace_enabled()), nvtx(nvtx_enabled()) {
    if (on) t0 = std::chrono::steady_clock::now();
    if (nvtx) nvtx_push(name);
  }
  ~TraceScope() {
    if (nvtx) nvtx_pop();
    if (on) trace_add(name, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  }
};

}  // namespace tnbp

#define TNBP_TRACE_CAT2(a, b) a##b
#define TNBP_TRACE_CAT(a, b) TNBP_TRACE_CAT2(a, b)
#define TNBP_TRACE_SCOPE(name) ::tnbp::TraceScope TNBP_TRACE_CAT(tnbp_trace_, __LINE__)(name)
