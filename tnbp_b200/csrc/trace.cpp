#include "trace.h"

#include <nvtx3/nvToolsExt.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <utility>

namespace tnbp {
namespace {
struct Totals {
  std::mutex mu;
  std::map<std::string, std::pair<long long, double>> t;
  ~Totals() {
    if (t.empty()) return;
    std::fprintf(stderr, "tnbp trace (host wall time per region):\n");
    for (auto& kv : t)
      std::fprintf(stderr, "  %-28s %8lld calls %10.4f s\n", kv.first.c_str(), kv.second.first, kv.second.second);
  }
};
Totals& totals() {
  static Totals tt;
  return tt;
}
}  // namespace

bool trace_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_TRACE");
    return e && e[0] == '1';
  }();
  return on;
}

bool nvtx_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TNBP_NVTX");
    return e && e[0] == '1';
  }();
  return on;
}

void nvtx_push(const char* name) { nvtxRangePushA(name); }
void nvtx_pop() { nvtxRangePop(); }

void trace_add(const char* name, double seconds) {
  Totals& tt = totals();
  std::lock_guard<std::mutex> lk(tt.mu);
  auto& v = tt.t[name];
  v.first += 1;
  v.second += seconds;
}

}  // namespace tnbp
