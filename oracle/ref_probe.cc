// Golden-vector probe: the reference's own estimator loop
// (apps/estimator/main.cc:105-238) on the reference's unchanged headers,
// with every intermediate tensor written to a binary record file.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/ by oracle/Makefile
// against the CPU gqten stand-in in oracle/gqten_cpu).  The records are the
// fixtures the B200 kernels are checked against.
//
// usage: ref_probe <circuit.qasm> <pauli.txt> <out.bin> <max_bond_dim>
//                  <sv_min> <bp_tolerance> <max_bp_iterations> [<Lx> <Ly>]
// With Lx Ly the edge list is bond_square_lattice(Lx, Ly) (so 2-qubit gates
// between non-adjacent qubits get identity pass-through tensors), else
// EdgesFromQasm of the program (apps/estimator/main.cc:45-48).
//
// Record layout (little-endian): u32 name_len, name bytes, u32 rank,
// i32 shape[rank], u64 n, then n complex128 (re, im) values in column-major
// order.  Scalars are rank-0 records with n = 1.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "pauli/sparse_pauli.h"
#include "qasm/any.h"
#include "qasm/utility.h"
#include "tnbp/tnbp.h"

using Tensor = gqten::tensor<std::complex<double>>;
using Elem = std::complex<double>;

static std::ofstream g_out;

static void rec(const std::string& name, const std::vector<int32_t>& shape, const std::vector<Elem>& data) {
  uint32_t nl = (uint32_t)name.size(), r = (uint32_t)shape.size();
  uint64_t n = data.size();
  g_out.write((const char*)&nl, 4);
  g_out.write(name.data(), nl);
  g_out.write((const char*)&r, 4);
  if (r) g_out.write((const char*)shape.data(), 4 * r);
  g_out.write((const char*)&n, 8);
  g_out.write((const char*)data.data(), 16 * n);
}
static void rec_t(const std::string& name, const Tensor& t) {
  std::vector<Elem> d(t.Size());
  for (size_t i = 0; i < t.Size(); ++i) d[i] = t.GetElem(i);
  rec(name, t.Shape(), d);
}
static void rec_s(const std::string& name, Elem v) { rec(name, {}, {v}); }

int main(int argc, char** argv) {
  if (argc < 8) {
    std::fprintf(stderr, "usage: ref_probe qasm pauli out max_bond_dim sv_min bp_tol bp_max\n");
    return 2;
  }
  const std::string qasm_path = argv[1], pauli_path = argv[2];
  g_out.open(argv[3], std::ios::binary);
  const int max_bond_dim = std::atoi(argv[4]);
  const double sv_min = std::atof(argv[5]);
  const double bp_tol = std::atof(argv[6]);
  const int bp_max = std::atoi(argv[7]);

  MPI_Comm comm = MPI_COMM_WORLD;
  tci::gqten_handle ctx;
  tci::create_context(ctx);
  auto program = qasm::parse_any(qasm::read_all_file(qasm_path));
  auto edges = argc > 9 ? tnbp::bond_square_lattice(std::atoi(argv[8]), std::atoi(argv[9]))
                        : tnbp::EdgesFromQasm(program);
  auto layer_edges = tnbp::GreedyEdgeLayering(edges);
  {
    std::vector<Elem> e;
    for (auto& p : edges) { e.push_back(p.first); e.push_back(p.second); }
    rec("edges", {2, (int32_t)edges.size()}, e);
  }
  auto TPO = tnbp::QasmToTPO<Tensor>(ctx, program, edges);
  rec_s("n_layers", (double)TPO.size());
  for (size_t l = 0; l < TPO.size(); ++l)
    for (size_t s = 0; s < TPO[l].size(); ++s)
      rec_t("tpo/" + std::to_string(l) + "/" + std::to_string(s), TPO[l][s]);

  auto qubit = tnbp::GetSiteIndexFromBond(edges);
  std::vector<Tensor> V, E, F;
  std::vector<int> SiteIdx, EdgeIdx;
  std::map<int, int> Site_To_MpiRank;
  std::vector<int> pdim(qubit.size(), 2);
  tnbp::InitTensorProductState(ctx, edges, pdim, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm);

  for (size_t t = 0; t < TPO.size(); ++t) {
    const std::string P = "step/" + std::to_string(t) + "/";
    tnbp::AbsorbTPO(ctx, TPO[t], edges, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm);
    for (size_t s = 0; s < V.size(); ++s) rec_t(P + "absorb/V/" + std::to_string(s), V[s]);
    for (size_t m = 0; m < E.size(); ++m) rec_t(P + "absorb/E/" + std::to_string(m), E[m]);
    double cond = 0;
    size_t k = 0;
    for (; k < (size_t)bp_max; ++k) {
      for (size_t p = 0; p < layer_edges.size(); ++p)
        tnbp::BeliefPropagation(ctx, edges, V, SiteIdx, Site_To_MpiRank, layer_edges[p], E, EdgeIdx, comm, F);
      auto itE = E.begin();
      for (const auto& et : F) tci::copy(ctx, et, *itE++);
      if (k == 0)
        for (size_t m = 0; m < E.size(); ++m) rec_t(P + "sweep0/E/" + std::to_string(m), E[m]);
      tnbp::BeliefPropagationCondition(ctx, edges, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm, cond);
      rec_s(P + "cond/" + std::to_string(k), cond);
      if (cond < bp_tol) break;
    }
    rec_s(P + "bp_iters", (double)std::min<size_t>(k + 1, (size_t)bp_max));
    for (size_t m = 0; m < E.size(); ++m) rec_t(P + "bp/E/" + std::to_string(m), E[m]);
    std::vector<int32_t> dims;
    std::vector<double> errs;
    tnbp::Truncation(ctx, edges, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm, max_bond_dim, sv_min, 0.0, dims, errs);
    {
      std::vector<Elem> d, er;
      for (auto x : dims) d.push_back((double)x);
      for (auto x : errs) er.push_back(x);
      rec(P + "trunc/dims", {(int32_t)d.size()}, d);
      rec(P + "trunc/errs", {(int32_t)er.size()}, er);
    }
    for (size_t s = 0; s < V.size(); ++s) rec_t(P + "trunc/V/" + std::to_string(s), V[s]);
    for (size_t m = 0; m < E.size(); ++m) rec_t(P + "trunc/E/" + std::to_string(m), E[m]);
  }

  auto spo = pauli::load_sparse_pauli_op<Elem>(pauli_path);
  std::vector<Tensor> exOp, exOp_one, exOp_two;
  std::vector<std::vector<int>> exSite;
  std::vector<int> exSite_one;
  std::vector<std::pair<int, int>> exPair_two;
  tnbp::SparsePauliToTensorOp(ctx, spo, exOp, exSite);
  tnbp::ClassifyOps(ctx, edges, exOp, exSite, exOp_one, exSite_one, exOp_two, exPair_two);
  auto one = tnbp::Measure(ctx, edges, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm, exSite_one, exOp_one);
  {
    std::vector<Elem> s;
    for (int x : exSite_one) s.push_back((double)x);
    rec("meas1/sites", {(int32_t)s.size()}, s);
    rec("meas1/values", {(int32_t)one.size()}, one);
    for (size_t i = 0; i < exOp_one.size(); ++i) rec_t("meas1/op/" + std::to_string(i), exOp_one[i]);
  }
  // The reference sizes the two-site result by the edge count
  // (measure.h:123); keep the requested pairs within that size.
  if (exPair_two.size() > edges.size()) exPair_two.resize(edges.size());
  auto two = tnbp::Measure(ctx, edges, V, SiteIdx, Site_To_MpiRank, E, EdgeIdx, comm, exPair_two, exOp_two);
  two.resize(exPair_two.size());
  {
    std::vector<Elem> p;
    for (auto& q : exPair_two) { p.push_back((double)q.first); p.push_back((double)q.second); }
    rec("meas2/pairs", {2, (int32_t)exPair_two.size()}, p);
    rec("meas2/values", {(int32_t)two.size()}, two);
    for (size_t i = 0; i < exPair_two.size(); ++i) rec_t("meas2/op/" + std::to_string(i), exOp_two[i]);
  }
  g_out.close();
  return 0;
}
