// Host-side checks of include/tnbp_b200.hpp (no device needed): the
// reference's function names and argument meanings over the C ABI, and the
// exceptions its status codes become.  Prints one "ok <name>" line per check
// and exits non-zero on the first failure; tests/test_cpp_interface.py
// compiles and runs it.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "tnbp_b200.hpp"

namespace tb = tnbp_b200;

#define EXPECT(cond, name)                                      \
  do {                                                          \
    if (!(cond)) {                                              \
      std::printf("FAIL %s (%s:%d)\n", name, __FILE__, __LINE__); \
      return 1;                                                 \
    }                                                           \
    std::printf("ok %s\n", name);                               \
  } while (0)

template <class E, class F>
bool throws(F&& f) {
  try {
    f();
  } catch (const E&) {
    return true;
  } catch (...) {
    return false;
  }
  return false;
}

int main() {
  // bond_square_lattice / GetSiteIndexFromBond / GetSurroundingBondIndex / FindShortestPath / GreedyEdgeLayering
  const tb::Edges e = tb::bond_square_lattice(3, 2);
  EXPECT(e.size() == 7 && e[0] == std::make_pair(0, 1) && e[1] == std::make_pair(0, 3), "bond_square_lattice");
  EXPECT(tb::GetSiteIndexFromBond(e).size() == 6 && tb::GetSiteIndexFromBond(e)[5] == 5, "GetSiteIndexFromBond");
  const auto b4 = tb::GetSurroundingBondIndex(4, e);
  EXPECT(b4.size() == 3 && b4[0] == 3 && b4[1] == 5 && b4[2] == 6, "GetSurroundingBondIndex");
  const auto p = tb::FindShortestPath(e, 0, 5);
  EXPECT(p.size() == 4 && p.front() == 0 && p.back() == 5, "FindShortestPath");
  size_t nl = 0;
  for (const auto& l : tb::GreedyEdgeLayering(e)) nl += l.size();
  EXPECT(nl == e.size(), "GreedyEdgeLayering");

  // EdgesFromQasm / QasmToTPO / OptTPObySVD
  const std::string src =
      "OPENQASM 2.0;\ninclude \"qelib1.inc\";\nqreg q[3];\n"
      "cx q[0],q[1];\nrz(0.3) q[1];\ncx q[0],q[1];\ncz q[1],q[2];\nbarrier q;\nh q[0];\n";
  const tb::Edges qe = tb::EdgesFromQasm(src);
  EXPECT(qe.size() == 2 && qe[0] == std::make_pair(0, 1) && qe[1] == std::make_pair(1, 2), "EdgesFromQasm");
  auto tpo = tb::QasmToTPO(src, qe);
  EXPECT(tpo.size() == 2 && tpo[0].edge_rank[0] == 4 && tpo[0].edge_rank[1] == 2 && tpo[1].edge_rank[0] == 1,
         "QasmToTPO");
  const size_t before = tpo[0].op_data.size();
  tb::OptTPObySVD(qe, tpo[0], 1e-8);
  EXPECT(tpo[0].edge_rank[0] == 2 && tpo[0].edge_rank[1] == 2 && tpo[0].op_data.size() < before, "OptTPObySVD");
  const auto ki = tb::CircuitTPO(e, -0.25 * M_PI, 0.0, 0.4, 1.0);
  EXPECT(ki.edge_rank.size() == e.size() && ki.edge_rank[0] == 2, "CircuitTPO");

  // ClassifyOps on an observable text
  const auto terms = tb::ClassifyOps("1.0 0.0 IIZ\n0.5 IZZ\n2.0 ZIZ\n0.25 III\n", qe);
  EXPECT(terms.size() == 2 && terms.kind[0] == 1 && terms.kind[1] == 2 && terms.dropped == 2, "ClassifyOps");

  // status codes -> the reference's exceptions
  EXPECT(throws<tb::ParseError>([&] { tb::EdgesFromQasm("OPENQASM 2.0;\nqreg q[2];\ncx q[0] q[1];\n"); }),
         "ParseError on a QASM syntax error");
  EXPECT(throws<std::runtime_error>([&] { tb::ClassifyOps("1.0 IXQ\n", qe); }),
         "runtime_error on an invalid Pauli label");
  EXPECT(throws<std::runtime_error>([&] { tb::QasmToTPO("OPENQASM 2.0;\nqreg q[3];\nccx q[0],q[1],q[2];\n", qe); }),
         "runtime_error on an unsupported gate");
  EXPECT(throws<std::invalid_argument>([&] { tb::bond_square_lattice(0, 3); }), "invalid_argument on bad sizes");
  if (!tnbp_device_available()) {
    EXPECT(throws<std::runtime_error>([&] { tb::State s(e); }), "no device: State refuses (no CPU path)");
    EXPECT(throws<std::runtime_error>([&] { tb::Server s; }), "no device: Server refuses (no CPU path)");
  }
  return 0;
}
