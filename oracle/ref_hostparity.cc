// Host-parity probe: runs the reference's own lattice, graph, QASM and Pauli
// code (include/tnbp/lattice/square.h, include/tnbp/framework/graph.h,
// include/qasm/*, include/pauli/*, include/tnbp/parser/*) and prints the
// results as JSON for the bit-exact tests of the B200 host builders.
//
// TEST INFRASTRUCTURE ONLY, built into oracle/_ref/ by oracle/Makefile.
//
// usage: ref_hostparity lattice <Lx> <Ly>
//        ref_hostparity qasm <file.qasm> [<pauli.txt> [<Lx> <Ly>]]
//        ref_hostparity opttpo <file.qasm> <eps> [<Lx> <Ly>]
//        ref_hostparity tpocount <file.qasm> <n0,n1,...>
// (tpocount: QasmToTPO with manual gate-number layering, qasmtotpo.h:709-738)
// (opttpo: every TPO layer of QasmToTPO before and after the reference's
//  OptTPObySVD, include/tnbp/ptns/function/optsvdtpo.h, as shapes and
//  column-major element lists)
// (with Lx Ly the TPO and Pauli classification use bond_square_lattice)
#include <chrono>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>

#include "pauli/sparse_pauli.h"
#include "qasm/any.h"
#include "qasm/utility.h"
#include "tnbp/tnbp.h"

using Tensor = gqten::tensor<std::complex<double>>;

static void edges_json(const char* key, const std::vector<std::pair<int, int>>& e) {
  std::printf("\"%s\": [", key);
  for (size_t i = 0; i < e.size(); ++i) std::printf("%s[%d,%d]", i ? "," : "", e[i].first, e[i].second);
  std::printf("]");
}

static void graph_json(const std::vector<std::pair<int, int>>& edges) {
  edges_json("edges", edges);
  auto layers = tnbp::GreedyEdgeLayering(edges);
  std::printf(", \"layers\": [");
  for (size_t l = 0; l < layers.size(); ++l) {
    std::printf("%s[", l ? "," : "");
    for (size_t i = 0; i < layers[l].size(); ++i) std::printf("%s[%d,%d]", i ? "," : "", layers[l][i].first, layers[l][i].second);
    std::printf("]");
  }
  std::printf("]");
  auto sites = tnbp::GetSiteIndexFromBond(edges);
  std::printf(", \"sites\": [");
  for (size_t i = 0; i < sites.size(); ++i) std::printf("%s%d", i ? "," : "", sites[i]);
  std::printf("], \"bonds\": [");
  for (size_t i = 0; i < sites.size(); ++i) {
    auto b = tnbp::GetSurroundingBondIndex(sites[i], edges);
    std::printf("%s[", i ? "," : "");
    for (size_t k = 0; k < b.size(); ++k) std::printf("%s%d", k ? "," : "", b[k]);
    std::printf("]");
  }
  std::printf("], \"paths\": [");
  bool first = true;
  for (size_t i = 0; i < sites.size(); i += 3)
    for (size_t j = 0; j < sites.size(); j += 5) {
      auto p = tnbp::FindShortestPath(edges, sites[i], sites[j]);
      std::printf("%s[%d,%d,[", first ? "" : ",", sites[i], sites[j]);
      first = false;
      for (size_t k = 0; k < p.size(); ++k) std::printf("%s%d", k ? "," : "", p[k]);
      std::printf("]]");
    }
  std::printf("]");
}

static void tpo_json(const char* key, const std::vector<std::vector<Tensor>>& T) {
  std::printf("\"%s\": [", key);
  for (size_t l = 0; l < T.size(); ++l) {
    std::printf("%s[", l ? "," : "");
    for (size_t s = 0; s < T[l].size(); ++s) {
      auto sh = T[l][s].Shape();
      std::printf("%s[[", s ? "," : "");
      for (size_t k = 0; k < sh.size(); ++k) std::printf("%s%d", k ? "," : "", sh[k]);
      std::printf("],[");
      for (size_t k = 0; k < T[l][s].Size(); ++k)
        std::printf("%s%.17g,%.17g", k ? "," : "", T[l][s].GetElem(k).real(), T[l][s].GetElem(k).imag());
      std::printf("]]");
    }
    std::printf("]");
  }
  std::printf("]");
}

int main(int argc, char** argv) {
  if (argc < 3) { std::fprintf(stderr, "usage\n"); return 2; }
  const std::string mode = argv[1];
  std::printf("{");
  if (mode == "lattice") {
    auto edges = tnbp::bond_square_lattice(std::atoi(argv[2]), std::atoi(argv[3]));
    graph_json(edges);
  } else if (mode == "opttpo") {
    auto prog = qasm::parse_any(qasm::read_all_file(argv[2]));
    const double eps = std::atof(argv[3]);
    auto edges = argc > 5 ? tnbp::bond_square_lattice(std::atoi(argv[4]), std::atoi(argv[5]))
                          : tnbp::EdgesFromQasm(prog);
    edges_json("edges", edges);
    tci::gqten_handle ctx;
    auto T = tnbp::QasmToTPO<Tensor>(ctx, prog, edges);
    std::printf(", ");
    tpo_json("before", T);
    const auto t0 = std::chrono::steady_clock::now();
    for (auto& layer : T) tnbp::OptTPObySVD(ctx, edges, layer, eps);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf(", ");
    tpo_json("after", T);
    std::printf(", \"eps\": %.17g, \"opt_seconds\": %.6g", eps, secs);
  } else if (mode == "tpocount") {
    auto prog = qasm::parse_any(qasm::read_all_file(argv[2]));
    std::vector<int> counts;
    {
      std::stringstream ss(argv[3]);
      std::string tok;
      while (std::getline(ss, tok, ',')) counts.push_back(std::stoi(tok));
    }
    auto edges = tnbp::EdgesFromQasm(prog);
    edges_json("edges", edges);
    tci::gqten_handle ctx;
    auto T = tnbp::QasmToTPO<Tensor>(ctx, prog, edges, counts);
    std::printf(", ");
    tpo_json("layers", T);
  } else if (mode == "qasm") {
    auto prog = qasm::parse_any(qasm::read_all_file(argv[2]));
    std::printf("\"instructions\": [");
    for (size_t i = 0; i < prog.instructions.size(); ++i) {
      const auto& in = prog.instructions[i];
      std::printf("%s[%d,[", i ? "," : "", (int)in.op);
      for (size_t k = 0; k < in.qubits.size(); ++k) std::printf("%s%zu", k ? "," : "", in.qubits[k].index);
      std::printf("],[");
      for (size_t k = 0; k < in.params.size(); ++k) std::printf("%s%.17g", k ? "," : "", in.params[k]);
      std::printf("]]");
    }
    std::printf("], ");
    auto edges = argc > 5 ? tnbp::bond_square_lattice(std::atoi(argv[4]), std::atoi(argv[5]))
                          : tnbp::EdgesFromQasm(prog);
    graph_json(edges);
    tci::gqten_handle ctx;
    bool has_3q = false;
    // QasmToTPO throws on measure/reset/custom (qasmtotpo.h:139-142) and its
    // three-qubit branch indexes past its path vector (qasmtotpo.h:465-488),
    // so TPO shapes are only recorded for programs without those.
    for (auto& in : prog.instructions)
      has_3q |= (tnbp::OpQubitCount(in) == 3 && in.op != qasm::Op::BARRIER) || in.op == qasm::Op::MEASURE ||
                in.op == qasm::Op::RESET || in.op == qasm::Op::CUSTOM;
    if (!has_3q) {
      auto T = tnbp::QasmToTPO<Tensor>(ctx, prog, edges);
      std::printf(", \"tpo_shapes\": [");
      for (size_t l = 0; l < T.size(); ++l) {
        std::printf("%s[", l ? "," : "");
        for (size_t s = 0; s < T[l].size(); ++s) {
          auto sh = T[l][s].Shape();
          std::printf("%s[", s ? "," : "");
          for (size_t k = 0; k < sh.size(); ++k) std::printf("%s%d", k ? "," : "", sh[k]);
          std::printf("]");
        }
        std::printf("]");
      }
      std::printf("]");
    }
    if (argc > 3) {
      auto spo = pauli::load_sparse_pauli_op<std::complex<double>>(argv[3]);
      std::vector<Tensor> ops, one_t, two_t;
      std::vector<std::vector<int>> qs;
      std::vector<int> one;
      std::vector<std::pair<int, int>> two;
      tnbp::SparsePauliToTensorOp(ctx, spo, ops, qs);
      tnbp::ClassifyOps(ctx, edges, ops, qs, one_t, one, two_t, two);
      std::printf(", \"pauli_one\": [");
      for (size_t i = 0; i < one.size(); ++i) {
        std::printf("%s[%d,[", i ? "," : "", one[i]);
        for (size_t k = 0; k < one_t[i].Size(); ++k)
          std::printf("%s[%.17g,%.17g]", k ? "," : "", one_t[i].GetElem(k).real(), one_t[i].GetElem(k).imag());
        std::printf("]]");
      }
      std::printf("], \"pauli_two\": [");
      for (size_t i = 0; i < two.size(); ++i) {
        std::printf("%s[%d,%d,[", i ? "," : "", two[i].first, two[i].second);
        for (size_t k = 0; k < two_t[i].Size(); ++k)
          std::printf("%s[%.17g,%.17g]", k ? "," : "", two_t[i].GetElem(k).real(), two_t[i].GetElem(k).imag());
        std::printf("]]");
      }
      std::printf("], \"pauli_coeffs\": [");
      for (size_t i = 0; i < spo.size(); ++i)
        std::printf("%s[%.17g,%.17g]", i ? "," : "", spo[i].coeff.real(), spo[i].coeff.imag());
      std::printf("]");
    }
  }
  std::printf("}\n");
  return 0;
}
