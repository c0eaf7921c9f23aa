// Host-side problem builders (lattice, QASM, Pauli, TPO); see host_setup.cpp.
#pragma once
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace tnbp_host {

struct HostError : std::runtime_error {
  int code;
  HostError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

using Edges = std::vector<std::pair<int, int>>;

// Same enumerator order as qasm::Op (include/qasm/ir.h:13-16).
enum class Op { U3, U2, U1, RX, RY, RZ, H, X, Y, Z, S, SDG, T, TDG, ID, CX, CZ, SWAP, RZZ, CCX, CSWAP,
                MEASURE, BARRIER, RESET, CUSTOM };
struct QArg { std::string reg; size_t index = 0; };
struct Instruction { Op op = Op::ID; std::vector<double> params; std::vector<QArg> qubits; };
struct Program { std::vector<Instruction> instructions; };

struct Layer {
  std::vector<int32_t> edge_rank;
  std::vector<int64_t> op_offset;
  std::vector<double> op_data;  // interleaved complex
};

struct PauliTerm {
  int kind = 0;  // 1 or 2
  int q0 = -1, q1 = -1;
  char l0 = 0, l1 = 0;
  double coeff_re = 0, coeff_im = 0;
  int64_t row = 0;
};

// Every row of a sparse-Pauli text: kind 0 identity, 1 one qubit, 2 a pair
// on an edge (the two kinds ClassifyOps keeps), 3 any other product.
struct PauliString {
  int kind = 0;
  std::vector<int> qubits;  // ascending
  std::string letters;      // one per qubit
  double coeff_re = 0, coeff_im = 0;
};

Edges square_lattice(int Lx, int Ly);
std::vector<int> greedy_layering(const Edges& e, int* nlayers);
std::vector<int> surrounding_bonds(const Edges& e, int site);
std::vector<int> site_labels(const Edges& e);
std::vector<int> shortest_path(const Edges& e, int src, int dst);
// One parsed line of a sparse-Pauli text: coefficient and the non-identity
// letters with their qubits (ascending; the rightmost letter is qubit 0).
struct PauliRow {
  double re = 0, im = 0;
  std::vector<std::pair<int, char>> ops;
};

Program parse_qasm(const std::string& src);          // qasm_text.cpp
int op_arity(Op op);                                 // qasm_text.cpp
std::vector<PauliRow> pauli_rows(const std::string& text);  // qasm_text.cpp
int qubit_count(const Instruction& in);
Edges qasm_edges(const Program& p);
std::vector<Layer> qasm_tpo(const Program& p, const Edges& edges);
std::vector<Layer> qasm_tpo_counts(const Program& p, const Edges& edges, const std::vector<int>& num_gates);
Layer kicked_ising_tpo(const Edges& edges, double Jz, double hz, double hx, double dt);
void opt_tpo_svd(const Edges& edges, Layer& layer, double eps);
std::vector<PauliTerm> pauli_terms(const std::string& text, const Edges& edges, int64_t* n_dropped);
std::vector<PauliString> pauli_strings(const std::string& text, const Edges& edges);
std::vector<std::complex<double>> pauli_list(char letter);

}  // namespace tnbp_host
