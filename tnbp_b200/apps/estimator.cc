// tnbp_estimator: the estimator app's loop (apps/estimator/main.cc:18-245)
// as C++ host code over the C ABI of libtnbp_b200 (include/tnbp_b200.h), the
// BP, truncation and measurement running on the B200.
//
// Command line as the reference app (apps/estimator/option.h:28-73):
//   --circuit FILE  --sparse_pauli FILE  --max_bond_dim N  --bp_tolerance X
//   --max_bp_iterations N  --sv_min X  --truncation_error X (accepted, unused
//   by the reference too)  --backend default  --do_opt_tpo N (nonzero:
//   OptTPObySVD on every layer)  --eps_opt_tpo X
// plus --precision c128|mixed|c64 (default c128, the drop-in), --sum
// (print sum_k c_k <P_k>, which the reference does not compute) and
// --measure_clusters (also measure the terms the reference drops --
// non-adjacent pairs, three or more qubits -- on their tree clusters, and
// print them with their file row).
// Printed lines follow the reference's wording for the per-layer BP
// condition, the per-edge truncation results and the per-term expectation
// values (one-site terms first, then two-site terms, each in file order);
// the reference's time stamps are left out.  Not supported here: the
// ibm_kobe backend's fixed edge list and --num_gates manual layering, which
// are outside the BP hot path.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "tnbp_b200.h"

namespace {

void check(int rc, const char* what) {
  if (rc != TNBP_OK) throw std::runtime_error(std::string(what) + ": " + tnbp_last_error());
}

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
      throw std::invalid_argument(a + " is not supported by tnbp_estimator");
    }
  }
  if (o.backend != "default") throw std::invalid_argument("only --backend default is supported");
  return o;
}

int run(const Options& o) {
  const std::string qasm = read_file(o.circuit);
  // edges (EdgesFromQasm) and the greedy layering the reference prints
  int64_t ne = 0;
  check(tnbp_qasm_edges(qasm.c_str(), nullptr, 0, &ne), "tnbp_qasm_edges");
  std::vector<int32_t> edges(2 * ne);
  check(tnbp_qasm_edges(qasm.c_str(), edges.data(), ne, &ne), "tnbp_qasm_edges");
  std::cout << " edges:";
  for (int64_t e = 0; e < ne; ++e) std::cout << " (" << edges[2 * e] << "," << edges[2 * e + 1] << ")";
  std::cout << "\n";

  // one TPO layer per barrier block (QasmToTPO)
  int32_t nlayers = 0;
  int64_t nelems = 0;
  check(tnbp_qasm_tpo(qasm.c_str(), edges.data(), ne, nullptr, nullptr, nullptr, 0, &nlayers, &nelems),
        "tnbp_qasm_tpo");
  int64_t ns = 0;
  {
    std::vector<char> seen;
    for (int32_t v : edges) {
      if ((size_t)v >= seen.size()) seen.resize(v + 1, 0);
      seen[v] = 1;
    }
    for (char c : seen) ns += c;
  }
  std::vector<int32_t> rank((size_t)nlayers * ne);
  std::vector<int64_t> off((size_t)nlayers * ns);
  std::vector<double> data(2 * (size_t)nelems);
  check(tnbp_qasm_tpo(qasm.c_str(), edges.data(), ne, rank.data(), off.data(), data.data(), nelems, &nlayers,
                      &nelems),
        "tnbp_qasm_tpo");

  // each layer on its own, its offsets re-based to its first element
  // (tnbp_qasm_tpo packs the layers one after another, site 0 first)
  std::vector<std::vector<int32_t>> lrank(nlayers);
  std::vector<std::vector<int64_t>> loff(nlayers);
  std::vector<std::vector<double>> ldata(nlayers);
  for (int32_t t = 0; t < nlayers; ++t) {
    const int64_t base = off[(size_t)t * ns];
    const int64_t end = t + 1 < nlayers ? off[(size_t)(t + 1) * ns] : nelems;
    lrank[t].assign(rank.begin() + (size_t)t * ne, rank.begin() + (size_t)(t + 1) * ne);
    for (int64_t k = 0; k < ns; ++k) loff[t].push_back(off[(size_t)t * ns + k] - base);
    ldata[t].assign(data.begin() + 2 * base, data.begin() + 2 * end);
  }
  if (o.do_opt_tpo) {
    for (int32_t t = 0; t < nlayers; ++t) {
      int64_t n = 0;
      check(tnbp_opt_tpo_svd(edges.data(), ne, o.eps_opt_tpo, lrank[t].data(), loff[t].data(), ldata[t].data(), &n),
            "tnbp_opt_tpo_svd");
      ldata[t].resize(2 * n);
      std::cout << " optimization of tpo for layer " << t << " is performed\n";
    }
  }

  tnbp_job* job = nullptr;
  check(tnbp_job_create(edges.data(), ne, nullptr, o.precision, nullptr, 0, &job), "tnbp_job_create");
  std::vector<int32_t> dims(ne);
  std::vector<double> errs(ne);
  std::cout.precision(16);
  for (int32_t t = 0; t < nlayers; ++t) {
    tnbp_tpo* tpo = nullptr;
    check(tnbp_tpo_create(job, lrank[t].data(), loff[t].data(), ldata[t].data(), &tpo), "tnbp_tpo_create");
    check(tnbp_absorb_tpo(job, tpo), "tnbp_absorb_tpo");
    check(tnbp_tpo_destroy(tpo), "tnbp_tpo_destroy");
    int32_t iters = 0;
    double cond = 0.0;
    check(tnbp_bp_run(job, o.bp_tolerance, o.max_bp_iterations, &iters, &cond), "tnbp_bp_run");
    std::cout << " error from belief propagation condition at step " << t << " = " << cond << " (" << iters
              << " sweeps)\n";
    check(tnbp_truncate(job, o.max_bond_dim, o.sv_min, dims.data(), errs.data()), "tnbp_truncate");
    for (int64_t e = 0; e < ne; ++e)
      std::cout << " truncation error for edge (" << edges[2 * e] << "," << edges[2 * e + 1] << ") = " << errs[e]
                << " bond dim = " << dims[e] << "\n";
  }

  // measurement: load_sparse_pauli_op + SparsePauliToTensorOp + ClassifyOps
  const std::string pauli = read_file(o.sparsepauli);
  int64_t nk = 0, nd = 0;
  check(tnbp_pauli_terms(pauli.c_str(), edges.data(), ne, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0,
                         &nk, &nd),
        "tnbp_pauli_terms");
  std::vector<int32_t> kind(nk + 1), q0(nk + 1), q1(nk + 1), row(nk + 1);
  std::vector<char> letters(2 * nk + 2);
  std::vector<double> coeff(2 * nk + 2), per(2 * nk + 2), sum(2);
  check(tnbp_pauli_terms(pauli.c_str(), edges.data(), ne, kind.data(), q0.data(), q1.data(), letters.data(),
                         coeff.data(), row.data(), nk, &nk, &nd),
        "tnbp_pauli_terms");
  std::cout << " number of measrement operators = " << nk + nd << "\n";
  if (nk > 0)
    check(tnbp_measure_pauli_sum(job, nk, kind.data(), q0.data(), q1.data(), letters.data(), coeff.data(),
                                 per.data(), sum.data()),
          "tnbp_measure_pauli_sum");
  for (int64_t k = 0; k < nk; ++k)
    if (kind[k] == 1)
      std::cout << " Expectation value of single site operator at site " << q0[k] << " " << per[2 * k] << "\n";
  for (int64_t k = 0; k < nk; ++k)
    if (kind[k] == 2)
      std::cout << " Expectation value of two site operator at sites (" << q0[k] << "," << q1[k] << ") "
                << per[2 * k] << "\n";
  if (o.print_sum) std::cout << " Sum of c_k <P_k> = " << sum[0] << " " << sum[1] << "\n";
  if (o.clusters) {
    int64_t nrows = 0;
    check(tnbp_measure_pauli_text(job, pauli.c_str(), 1, nullptr, nullptr, 0, &nrows, nullptr),
          "tnbp_measure_pauli_text");
    std::vector<double> vals(2 * nrows + 2), all(2);
    std::vector<int32_t> kinds(nrows + 1);
    check(tnbp_measure_pauli_text(job, pauli.c_str(), 1, vals.data(), kinds.data(), nrows, &nrows, all.data()),
          "tnbp_measure_pauli_text");
    for (int64_t r = 0; r < nrows; ++r)
      if (kinds[r] == 3)
        std::cout << " Expectation value of cluster operator in row " << r << " " << vals[2 * r] << "\n";
    if (o.print_sum) std::cout << " Sum of c_k <P_k> over all terms = " << all[0] << " " << all[1] << "\n";
  }
  check(tnbp_job_destroy(job), "tnbp_job_destroy");
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
