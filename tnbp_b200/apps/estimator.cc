// tnbp_estimator: the estimator app's loop (apps/estimator/main.cc:18-245)
// written against the engine's C++ interface (include/tnbp_b200.hpp, the
// reference's function names over the C ABI of libtnbp_b200), the BP,
// truncation and measurement running on the B200.
//
// Command line as the reference app (apps/estimator/option.h:28-73):
//   --circuit FILE  --sparse_pauli FILE  --max_bond_dim N  --bp_tolerance X
//   --max_bp_iterations N  --sv_min X  --truncation_error X (accepted, unused
//   by the reference too)  --backend default  --do_opt_tpo N (nonzero:
//   OptTPObySVD on every layer)  --eps_opt_tpo X  --num_gates n0,n1,...
//   (manual gate-number layering instead of barriers)
// plus --precision c128|mixed|c64 (default c128, the drop-in), --sum
// (print sum_k c_k <P_k>, which the reference does not compute) and
// --measure_clusters (also measure the terms the reference drops --
// non-adjacent pairs, three or more qubits -- on their tree clusters, and
// print them with their file row).
// Printed lines follow the reference's wording for the per-layer BP
// condition, the per-edge truncation results and the per-term expectation
// values (one-site terms first, then two-site terms, each in file order);
// the reference's time stamps are left out.  Not supported here: the
// ibm_kobe backend's fixed edge list, which is outside the BP hot path.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "tnbp_b200.hpp"

namespace {

std::string read_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

struct Options {
  std::string backend = "default", circuit = "circuit.qasm", sparsepauli = "sparsepauliop.txt";
  int max_bp_iterations = 50, max_bond_dim = 100;
  double bp_tolerance = 1.0e-8, sv_min = 1.0e-8, truncation_error = 1.0e-8;
  bool do_opt_tpo = false;
  std::vector<int> num_gates;
  double eps_opt_tpo = 1.0e-8;
  int precision = TNBP_C128;
  bool print_sum = false;
  bool clusters = false;
};

Options parse(int argc, char** argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) throw std::invalid_argument("missing value after " + a);
      return argv[++i];
    };
    if (a == "--backend") o.backend = next();
    else if (a == "--circuit") o.circuit = next();
    else if (a == "--sparse_pauli") o.sparsepauli = next();
    else if (a == "--max_bp_iterations") o.max_bp_iterations = std::atoi(next().c_str());
    else if (a == "--bp_tolerance") o.bp_tolerance = std::atof(next().c_str());
    else if (a == "--max_bond_dim") o.max_bond_dim = std::atoi(next().c_str());
    else if (a == "--sv_min") o.sv_min = std::atof(next().c_str());
    else if (a == "--truncation_error") o.truncation_error = std::atof(next().c_str());
    else if (a == "--sum") o.print_sum = true;
    else if (a == "--measure_clusters") o.clusters = true;
    else if (a == "--do_opt_tpo") o.do_opt_tpo = std::atoi(next().c_str()) != 0;
    else if (a == "--eps_opt_tpo") o.eps_opt_tpo = std::atof(next().c_str());
    else if (a == "--precision") {
      const std::string p = next();
      if (p == "c128") o.precision = TNBP_C128;
      else if (p == "mixed") o.precision = TNBP_MIXED;
      else if (p == "c64") o.precision = TNBP_C64;
      else throw std::invalid_argument("--precision must be c128, mixed or c64");
    } else if (a == "--num_gates") {
      std::stringstream ss(next());
      std::string tok;
      while (std::getline(ss, tok, ',')) o.num_gates.push_back(std::stoi(tok));
    }
  }
  if (o.backend != "default") throw std::invalid_argument("only --backend default is supported");
  return o;
}

int run(const Options& o) {
  namespace tb = tnbp_b200;
  const std::string qasm = read_file(o.circuit);
  // edges (EdgesFromQasm), one TPO layer per barrier block (QasmToTPO)
  const tb::Edges edges = tb::EdgesFromQasm(qasm);
  std::cout << " edges:";
  for (const auto& e : edges) std::cout << " (" << e.first << "," << e.second << ")";
  std::cout << "\n";
  std::vector<tb::TpoLayer> TPO =
      o.num_gates.empty() ? tb::QasmToTPO(qasm, edges) : tb::QasmToTPO(qasm, edges, o.num_gates);
  if (o.do_opt_tpo)
    for (size_t l = 0; l < TPO.size(); ++l) {
      tb::OptTPObySVD(edges, TPO[l], o.eps_opt_tpo);
      std::cout << " optimization of tpo for layer " << l << " is performed\n";
    }

  tb::State W = tb::InitTensorProductState(edges, o.precision);
  std::vector<int> res_bond_dim;
  std::vector<double> res_trunc_err;
  std::cout.precision(16);
  for (size_t t = 0; t < TPO.size(); ++t) {
    tb::AbsorbTPO(W, TPO[t]);
    const auto [iters, cond] = tb::BeliefPropagationLoop(W, o.bp_tolerance, o.max_bp_iterations);
    std::cout << " error from belief propagation condition at step " << t << " = " << cond << " (" << iters
              << " sweeps)\n";
    tb::Truncation(W, o.max_bond_dim, o.sv_min, res_bond_dim, res_trunc_err);
    for (size_t e = 0; e < edges.size(); ++e)
      std::cout << " truncation error for edge (" << edges[e].first << "," << edges[e].second
                << ") = " << res_trunc_err[e] << " bond dim = " << res_bond_dim[e] << "\n";
  }

  // measurement: load_sparse_pauli_op + SparsePauliToTensorOp + ClassifyOps
  const std::string pauli = read_file(o.sparsepauli);
  const tb::PauliTerms terms = tb::ClassifyOps(pauli, edges);
  std::cout << " number of measrement operators = " << (int64_t)terms.size() + terms.dropped << "\n";
  std::vector<tb::cplx> per;
  const tb::cplx sum = tb::MeasurePauliSum(W, terms, &per);
  for (size_t k = 0; k < terms.size(); ++k)
    if (terms.kind[k] == 1)
      std::cout << " Expectation value of single site operator at site " << terms.q0[k] << " " << per[k].real()
                << "\n";
  for (size_t k = 0; k < terms.size(); ++k)
    if (terms.kind[k] == 2)
      std::cout << " Expectation value of two site operator at sites (" << terms.q0[k] << "," << terms.q1[k]
                << ") " << per[k].real() << "\n";
  if (o.print_sum) std::cout << " Sum of c_k <P_k> = " << sum.real() << " " << sum.imag() << "\n";
  if (o.clusters) {
    std::vector<tb::cplx> values;
    std::vector<int> kinds;
    const tb::cplx all = tb::MeasurePauliText(W, pauli, &values, &kinds);
    for (size_t r = 0; r < values.size(); ++r)
      if (kinds[r] == 3)
        std::cout << " Expectation value of cluster operator in row " << r << " " << values[r].real() << "\n";
    if (o.print_sum) std::cout << " Sum of c_k <P_k> over all terms = " << all.real() << " " << all.imag() << "\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(parse(argc, argv));
  } catch (const std::exception& e) {
    std::cerr << "tnbp_estimator: " << e.what() << "\n";
    return 1;
  }
}
