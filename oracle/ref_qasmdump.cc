// Differential probe of the QASM front end: parses every file named on the
// command line with the reference's own parser (qasm::parse_any,
// include/qasm/any.h) and prints one line per file:
//   ERR                                   the reference refused the text
//   OK;op,nq,q...,np,p...;op,...          each instruction: the qasm::Op
//                                         enumerator, its qubit indices and
//                                         its parameters as hex floats (%a)
// tests/test_qasm_differential.py compares these lines with the engine's
// parser on seeded mutations of the golden programs.
//
// TEST INFRASTRUCTURE ONLY, built into oracle/_ref/ by oracle/Makefile.
#include <cstdio>
#include <exception>
#include <fstream>
#include <sstream>
#include <string>

#include "qasm/any.h"

int main(int argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    std::ifstream f(argv[i], std::ios::binary);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string src = ss.str();
    std::string line = "OK";
    try {
      const auto prog = qasm::parse_any(src);
      for (const auto& in : prog.instructions) {
        line += ";" + std::to_string((int)in.op) + "," + std::to_string(in.qubits.size());
        for (const auto& q : in.qubits) line += "," + std::to_string(q.index);
        line += "," + std::to_string(in.params.size());
        char buf[64];
        for (double p : in.params) {
          std::snprintf(buf, sizeof buf, ",%a", p);
          line += buf;
        }
      }
    } catch (const std::exception&) {
      line = "ERR";
    }
    std::printf("%s\n", line.c_str());
  }
  return 0;
}
