// The engine's host code (tnbp_b200/csrc/host_setup.cpp, qasm_text.cpp, tps_io.cpp) under
// AddressSanitizer / UndefinedBehaviorSanitizer: every golden QASM program,
// observable and checkpoint, then seeded truncations and byte mutations of
// them.  Malformed input must end in a HostError (a status code at the C
// ABI), never in a crash or undefined behaviour.  tests/test_host_sanitizers.py
// compiles it with -fsanitize=address,undefined and runs it.
//
// usage: host_sanitize <qasm files...> -- <pauli files...> -- <checkpoint + its qasm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "host_setup.h"
#include "tps_io.h"

using namespace tnbp_host;

static std::string slurp(const std::string& p) {
  std::ifstream f(p, std::ios::binary);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

static int ok = 0, refused = 0;

template <class F>
static void guarded(F&& f) {
  try {
    f();
    ++ok;
  } catch (const HostError&) {
    ++refused;
  }
}

static void qasm_path(const std::string& src) {
  guarded([&] {
    const auto prog = parse_qasm(src);
    const auto edges = qasm_edges(prog);
    if (edges.empty()) return;
    auto layers = qasm_tpo(prog, edges);
    for (auto& l : layers) opt_tpo_svd(edges, l, 1e-8);
  });
}

static std::vector<std::string> variants(const std::string& s, std::mt19937_64& rng, int n) {
  std::vector<std::string> out;
  if (s.empty()) return out;
  for (int i = 0; i < n; ++i) {
    std::string v = s;
    switch (i % 3) {
      case 0: v.resize(rng() % s.size()); break;                       // truncation
      case 1: v[rng() % v.size()] = (char)(rng() % 256); break;        // one byte replaced
      default:                                                         // a span duplicated
        { const size_t a = rng() % v.size(), b = std::min(v.size(), a + 1 + rng() % 16);
          v.insert(a, v.substr(a, b - a)); }
    }
    out.push_back(v);
  }
  return out;
}

int main(int argc, char** argv) {
  std::vector<std::string> groups[3];
  int g = 0;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--") == 0) { ++g; continue; }
    if (g < 3) groups[g].push_back(argv[i]);
  }
  std::mt19937_64 rng(20261204);
  for (const auto& p : groups[0]) {
    const auto src = slurp(p);
    qasm_path(src);
    for (const auto& v : variants(src.size() > 20000 ? src.substr(0, 20000) : src, rng, 60)) qasm_path(v);
  }
  const auto lattice = square_lattice(4, 4);
  for (const auto& p : groups[1]) {
    const auto txt = slurp(p);
    for (const auto& t : std::vector<std::string>{txt}) {
      guarded([&] { int64_t d = 0; pauli_terms(t, lattice, &d); pauli_strings(t, lattice); });
    }
    for (const auto& v : variants(txt, rng, 60))
      guarded([&] { int64_t d = 0; pauli_terms(v, lattice, &d); pauli_strings(v, lattice); });
  }
  if (groups[2].size() == 2) {
    const auto bytes = slurp(groups[2][0]);
    const auto edges = qasm_edges(parse_qasm(slurp(groups[2][1])));
    const std::string tmp = "host_sanitize_ckpt.dat";
    auto check_file = [&](const std::string& b) {
      { std::ofstream f(tmp, std::ios::binary); f.write(b.data(), (std::streamsize)b.size()); }
      guarded([&] {
        const auto st = tps_read(tmp);
        std::vector<int> bd, pd;
        tps_check_whole(st, edges, bd, pd);
      });
    };
    check_file(bytes);
    for (const auto& v : variants(bytes, rng, 120)) check_file(v);
    std::remove(tmp.c_str());
  }
  std::printf("ok %d refused %d\n", ok, refused);
  return 0;
}
