// Text front end of the estimator path: OpenQASM 2 / 3-subset programs and
// sparse-Pauli observable files.
//
// QASM is read in two passes.  A tokenizer turns the whole source into a
// vector of tokens (identifiers, numeric literals, quoted strings, the arrow
// "->" and single-character symbols), dropping white space and // and /* */
// comments; each token keeps its line and column for error messages.  A
// statement reader then dispatches on the first token through a per-dialect
// keyword table; everything not in the table is a gate call.
//
// What the reference accepts is kept (include/qasm/any.h:8-21,
// include/qasm/v2/parser.h, include/qasm/v3/parser.h), because programs and
// fixtures are shared with it:
//   * keywords and gate names match case-insensitively; register names do not;
//   * expressions: + - (left-associative) over * / (left-associative) over a
//     unary sign over numbers, pi, tau and parentheses; a literal is converted
//     with strtod on its own characters, so parameters are the same doubles;
//     division by an exact zero is an error;
//   * a bare register argument stands for all of its qubits; OpenQASM 3 also
//     takes the half-open slice r[lo:hi];
//   * a gate with k x (its arity) qubit arguments becomes k instructions; a
//     gate of unknown name keeps all its arguments in one CUSTOM instruction;
//     barrier keeps all its qubits in one instruction; reset makes one per
//     qubit;
//   * measure: "measure q -> c;" in both dialects, "c[i] = measure q;",
//     "c = measure q;" (c of size 1) and "bit b = measure q;" in OpenQASM 3;
//   * OpenQASM 3 is chosen when the 32 characters from the first "OPENQASM"
//     contain a '3'; its header is then required.
// Malformed input of any kind ends in a HostError with code -5 (TNBP_EPARSE).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "host_setup.h"

namespace tnbp_host {

namespace {

constexpr int kParseError = -5;

enum class Tok { Ident, Number, String, Arrow, Symbol, End };

struct Token {
  Tok kind;
  std::string text;  // identifier / literal characters / the symbol
  size_t line, col;
};

bool ident_start(char c) { return std::isalpha((unsigned char)c) || c == '_'; }
bool ident_char(char c) { return std::isalnum((unsigned char)c) || c == '_' || c == '$'; }

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

[[noreturn]] void fail(size_t line, size_t col, const std::string& what) {
  throw HostError(kParseError, "QASM, line " + std::to_string(line) + " column " + std::to_string(col) + ": " + what);
}

// ----------------------------------------------------------- tokenizer
std::vector<Token> tokenize(const std::string& s) {
  std::vector<Token> out;
  size_t i = 0, line = 1, col = 1;
  const size_t n = s.size();
  auto advance = [&](size_t k) {
    for (size_t j = 0; j < k && i < n; ++j, ++i) {
      if (s[i] == '\n') { ++line; col = 1; } else { ++col; }
    }
  };
  while (i < n) {
    const char c = s[i];
    if (std::isspace((unsigned char)c)) { advance(1); continue; }
    if (c == '/' && i + 1 < n && s[i + 1] == '/') {
      while (i < n && s[i] != '\n') advance(1);
      continue;
    }
    if (c == '/' && i + 1 < n && s[i + 1] == '*') {
      advance(2);
      while (i < n && !(s[i] == '*' && i + 1 < n && s[i + 1] == '/')) advance(1);
      advance(2);  // an unterminated comment runs to the end of the text
      continue;
    }
    Token t{Tok::Symbol, std::string(1, c), line, col};
    if (ident_start(c)) {
      size_t j = i + 1;
      while (j < n && ident_char(s[j])) ++j;
      t.kind = Tok::Ident;
      t.text = s.substr(i, j - i);
      advance(j - i);
    } else if (std::isdigit((unsigned char)c) || c == '.') {
      // digits with at most one '.', then at most one exponent marker with
      // an optional sign (the literal form the reference's reader scans)
      size_t j = i;
      bool dot = false, exp = false;
      while (j < n) {
        const char d = s[j];
        if (std::isdigit((unsigned char)d)) {
          ++j;
        } else if (d == '.' && !dot) {
          dot = true;
          ++j;
        } else if ((d == 'e' || d == 'E') && !exp) {
          exp = true;
          ++j;
          if (j < n && (s[j] == '+' || s[j] == '-')) ++j;
        } else {
          break;
        }
      }
      t.kind = Tok::Number;
      t.text = s.substr(i, j - i);
      advance(j - i);
    } else if (c == '"') {
      size_t j = i + 1;
      while (j < n && s[j] != '"') ++j;
      t.kind = Tok::String;
      t.text = s.substr(i + 1, j - i - 1);
      advance(std::min(n, j + 1) - i);  // an unterminated string runs to the end
    } else if (c == '-' && i + 1 < n && s[i + 1] == '>') {
      t.kind = Tok::Arrow;
      t.text = "->";
      advance(2);
    } else {
      advance(1);
    }
    out.push_back(std::move(t));
  }
  out.push_back(Token{Tok::End, "", line, col});
  return out;
}

// ------------------------------------------------------------ gate table
struct GateSpec { const char* name; Op op; int arity; };
// Names of the reference's gate map (include/qasm/v2/parser.h mapGate),
// with the arity of gateArity; any other name is a CUSTOM instruction.
const GateSpec kGates[] = {
    {"u3", Op::U3, 1},   {"u", Op::U3, 1},    {"u2", Op::U2, 1},     {"u1", Op::U1, 1},   {"p", Op::U1, 1},
    {"rx", Op::RX, 1},   {"ry", Op::RY, 1},   {"rz", Op::RZ, 1},     {"h", Op::H, 1},     {"x", Op::X, 1},
    {"y", Op::Y, 1},     {"z", Op::Z, 1},     {"s", Op::S, 1},       {"sdg", Op::SDG, 1}, {"t", Op::T, 1},
    {"tdg", Op::TDG, 1}, {"id", Op::ID, 1},   {"cx", Op::CX, 2},     {"cnot", Op::CX, 2}, {"cz", Op::CZ, 2},
    {"swap", Op::SWAP, 2}, {"rzz", Op::RZZ, 2}, {"ccx", Op::CCX, 3}, {"toffoli", Op::CCX, 3},
    {"cswap", Op::CSWAP, 3},
};

const GateSpec* find_gate(const std::string& lname) {
  for (const auto& g : kGates)
    if (lname == g.name) return &g;
  return nullptr;
}

// ------------------------------------------------------ statement reader
class QasmReader {
 public:
  QasmReader(const std::string& src, bool v3) : toks_(tokenize(src)), v3_(v3) {}

  Program run() {
    if (is_keyword(0, "openqasm")) {
      ++pos_;
      // version: any run of numeric literals and dots ("2.0", "3"), or a string
      while (at(0).kind == Tok::Number || at(0).kind == Tok::String || sym(0, '.')) ++pos_;
      want(';');
    } else if (v3_) {
      err(at(0), "an OpenQASM 3 program must start with its OPENQASM header");
    }
    while (at(0).kind != Tok::End) statement();
    return std::move(prog_);
  }

 private:
  using Handler = void (QasmReader::*)();

  std::vector<Token> toks_;
  size_t pos_ = 0;
  bool v3_;
  Program prog_;
  std::unordered_map<std::string, size_t> qregs_, cregs_;

  const Token& at(size_t k) const { return toks_[std::min(pos_ + k, toks_.size() - 1)]; }
  bool sym(size_t k, char c) const { return at(k).kind == Tok::Symbol && at(k).text[0] == c; }
  bool is_keyword(size_t k, const char* kw) const { return at(k).kind == Tok::Ident && lower(at(k).text) == kw; }
  [[noreturn]] void err(const Token& t, const std::string& what) const { fail(t.line, t.col, what); }

  void want(char c) {
    if (!sym(0, c)) err(at(0), std::string("'") + c + "' was expected here");
    ++pos_;
  }
  std::string name() {
    if (at(0).kind != Tok::Ident) err(at(0), "a name was expected here");
    return toks_[pos_++].text;
  }

  // A non-negative integer written as a (possibly signed) literal, as in
  // register sizes and indices; the literal is truncated toward zero.
  size_t count() {
    const Token& t0 = at(0);
    double sign = 1.0;
    if (sym(0, '+') || sym(0, '-')) {
      sign = sym(0, '-') ? -1.0 : 1.0;
      ++pos_;
    }
    if (at(0).kind != Tok::Number) err(at(0), "a number was expected here");
    const double v = sign * std::strtod(toks_[pos_++].text.c_str(), nullptr);
    if (!(v > -1.0) || !(v < 1e15)) err(t0, "size or index out of range");
    return v < 0.0 ? 0 : (size_t)v;
  }

  // expression := term { (+|-) term }; term := unary { (*|/) unary };
  // unary := (+|-) unary | ( expression ) | number | pi | tau
  double expression() {
    double v = term();
    while (sym(0, '+') || sym(0, '-')) {
      const bool minus = sym(0, '-');
      ++pos_;
      const double r = term();
      v = minus ? v - r : v + r;
    }
    return v;
  }
  double term() {
    double v = unary();
    while (sym(0, '*') || sym(0, '/')) {
      const bool div = sym(0, '/');
      const Token& op = at(0);
      ++pos_;
      const double r = unary();
      if (div && r == 0.0) err(op, "division by zero in a gate parameter");
      v = div ? v / r : v * r;
    }
    return v;
  }
  double unary() {
    const Token& t = at(0);
    if (sym(0, '+') || sym(0, '-')) {
      ++pos_;
      const double v = unary();
      return t.text[0] == '-' ? -v : v;
    }
    if (sym(0, '(')) {
      ++pos_;
      const double v = expression();
      want(')');
      return v;
    }
    if (t.kind == Tok::Ident) {
      const std::string l = lower(t.text);
      ++pos_;
      if (l == "pi") return 3.14159265358979323846;
      if (l == "tau") return 6.28318530717958647692;
      err(t, "'" + t.text + "' is not a constant this reader knows");
    }
    if (t.kind != Tok::Number) err(t, "a number was expected here");
    ++pos_;
    return std::strtod(t.text.c_str(), nullptr);
  }

  size_t register_size(std::unordered_map<std::string, size_t>& regs, const Token& t, const char* what) {
    auto it = regs.find(t.text);
    if (it == regs.end()) err(t, std::string("no ") + what + " named '" + t.text + "'");
    return it->second;
  }

  // One quantum argument: reg, reg[i] or (OpenQASM 3) reg[lo:hi].
  void qubit_operand(std::vector<QArg>& out) {
    const Token& t = at(0);
    const std::string reg = name();
    const size_t size = register_size(qregs_, t, "quantum register");
    if (!sym(0, '[')) {
      for (size_t k = 0; k < size; ++k) out.push_back({reg, k});
      return;
    }
    ++pos_;
    const size_t lo = count();
    if (v3_ && sym(0, ':')) {
      ++pos_;
      const size_t hi = count();
      want(']');
      if (hi < lo || hi > size) err(t, "slice " + reg + "[" + std::to_string(lo) + ":" + std::to_string(hi) + "] is outside the register");
      for (size_t k = lo; k < hi; ++k) out.push_back({reg, k});
      return;
    }
    want(']');
    if (lo >= size) err(t, "qubit " + reg + "[" + std::to_string(lo) + "] is outside the register");
    out.push_back({reg, lo});
  }
  std::vector<QArg> qubit_list() {
    std::vector<QArg> out;
    qubit_operand(out);
    while (sym(0, ',')) {
      ++pos_;
      qubit_operand(out);
    }
    return out;
  }
  // One classical target: c[i], or (OpenQASM 3) c for a one-bit register.
  void bit_operand() {
    const Token& t = at(0);
    name();
    const size_t size = register_size(cregs_, t, "classical register");
    if (!sym(0, '[')) {
      if (!v3_) err(at(0), "'[' was expected here");
      if (size != 1) err(t, "classical register '" + t.text + "' needs an index");
      return;
    }
    ++pos_;
    const size_t idx = count();
    want(']');
    if (idx >= size) err(t, "bit " + t.text + "[" + std::to_string(idx) + "] is outside the register");
  }

  void emit(Op op, std::vector<QArg> q, const std::vector<double>& params) {
    Instruction in;
    in.op = op;
    in.qubits = std::move(q);
    in.params = params;
    prog_.instructions.push_back(std::move(in));
  }
  void measured_qubit(const Token& where, std::vector<QArg> q) {
    if (q.size() != 1) err(where, "measure takes exactly one qubit");
    emit(Op::MEASURE, std::move(q), {});
  }

  // ---- statements (the keyword has not been consumed) ----
  void st_include() {
    ++pos_;
    if (at(0).kind != Tok::String) err(at(0), "include needs a quoted file name");
    ++pos_;
    want(';');
  }
  void declare(std::unordered_map<std::string, size_t>& regs) {  // OpenQASM 2: qreg q[n]; creg c[n];
    ++pos_;
    const std::string nm = name();
    want('[');
    const size_t n = count();
    want(']');
    want(';');
    regs[nm] = n;
  }
  void st_qreg() { declare(qregs_); }
  void st_creg() { declare(cregs_); }
  void declare3(std::unordered_map<std::string, size_t>& regs) {  // OpenQASM 3: qubit[n] q; bit c;
    ++pos_;
    size_t n = 1;
    if (sym(0, '[')) {
      ++pos_;
      n = count();
      want(']');
    }
    const std::string nm = name();
    want(';');
    regs[nm] = n;
  }
  void st_qubit() { declare3(qregs_); }
  void st_barrier() {
    ++pos_;
    auto q = qubit_list();
    want(';');
    emit(Op::BARRIER, std::move(q), {});
  }
  void st_reset() {
    ++pos_;
    auto q = qubit_list();
    want(';');
    for (auto& a : q) emit(Op::RESET, {a}, {});
  }
  void st_measure() {  // measure q -> c;
    const Token& kw = at(0);
    ++pos_;
    std::vector<QArg> q;
    qubit_operand(q);
    if (at(0).kind != Tok::Arrow) err(at(0), "'->' was expected after the measured qubit");
    ++pos_;
    bit_operand();
    want(';');
    measured_qubit(kw, std::move(q));
  }
  // OpenQASM 3 "bit ...": "bit b = measure q;" declares b (one bit) and
  // measures into it; otherwise a declaration "bit[n] c;" / "bit c;".
  void st_bit() {
    if (at(1).kind == Tok::Ident && sym(2, '=')) {
      ++pos_;
      const std::string nm = name();
      if (!cregs_.count(nm)) cregs_[nm] = 1;
      measure_rhs();
      return;
    }
    if (sym(1, '[') && at(2).kind == Tok::Number && sym(3, ']') && sym(4, '='))
      err(at(0), "a declared bit array cannot receive a measurement here");
    declare3(cregs_);
  }
  void measure_rhs() {  // '=' measure q ;
    want('=');
    const Token& kw = at(0);
    if (!is_keyword(0, "measure")) err(kw, "only 'measure' can be assigned to a bit");
    ++pos_;
    std::vector<QArg> q;
    qubit_operand(q);
    want(';');
    measured_qubit(kw, std::move(q));
  }
  void gate_call() {
    const Token& t = at(0);
    const std::string gname = name();
    const std::string l = lower(gname);
    if (v3_ && (l == "ctrl" || l == "inv" || l == "pow")) err(t, "gate modifiers (ctrl, inv, pow) are not supported");
    std::vector<double> params;
    if (sym(0, '(')) {
      ++pos_;
      if (!sym(0, ')')) {
        params.push_back(expression());
        while (sym(0, ',')) {
          ++pos_;
          params.push_back(expression());
        }
      }
      want(')');
    }
    auto q = qubit_list();
    want(';');
    const GateSpec* g = find_gate(l);
    if (!g) {
      emit(Op::CUSTOM, std::move(q), params);
      return;
    }
    const size_t ar = (size_t)g->arity;
    if (q.size() % ar != 0)
      err(t, "'" + gname + "' acts on " + std::to_string(ar) + " qubit(s); got " + std::to_string(q.size()));
    for (size_t k = 0; k < q.size(); k += ar) emit(g->op, std::vector<QArg>(q.begin() + k, q.begin() + k + ar), params);
  }
  // OpenQASM 3: "c = measure q;" or "c[i] = measure q;"
  bool is_bit_assignment() const {
    if (at(0).kind != Tok::Ident) return false;
    if (sym(1, '=')) return true;
    return sym(1, '[') && at(2).kind == Tok::Number && sym(3, ']') && sym(4, '=');
  }
  void st_bit_assignment() {
    bit_operand();
    measure_rhs();
  }

  void statement() {
    static const std::vector<std::pair<const char*, Handler>> v2 = {
        {"include", &QasmReader::st_include}, {"qreg", &QasmReader::st_qreg},       {"creg", &QasmReader::st_creg},
        {"barrier", &QasmReader::st_barrier}, {"reset", &QasmReader::st_reset},     {"measure", &QasmReader::st_measure}};
    static const std::vector<std::pair<const char*, Handler>> v3 = {
        {"include", &QasmReader::st_include}, {"qubit", &QasmReader::st_qubit},     {"bit", &QasmReader::st_bit},
        {"barrier", &QasmReader::st_barrier}, {"reset", &QasmReader::st_reset},     {"measure", &QasmReader::st_measure}};
    if (at(0).kind == Tok::Ident) {
      const std::string l = lower(at(0).text);
      for (const auto& e : v3_ ? v3 : v2)
        if (l == e.first) {
          (this->*e.second)();
          return;
        }
      if (v3_ && is_bit_assignment()) {
        st_bit_assignment();
        return;
      }
    }
    gate_call();
  }
};

}  // namespace

int op_arity(Op op) {
  for (const auto& g : kGates)
    if (g.op == op) return g.arity;
  return 0;
}

namespace {

bool is_openqasm3(const std::string& src) {
  const size_t pos = src.find("OPENQASM");
  return pos != std::string::npos && src.substr(pos, 32).find('3') != std::string::npos;
}

}  // namespace

Program parse_qasm(const std::string& src) { return QasmReader(src, is_openqasm3(src)).run(); }

// ------------------------------------------------------- sparse Pauli
// A line of the observable text (load_sparse_pauli_op,
// include/pauli/sparse_pauli.h:52-97): "re im LABEL" or "re LABEL", blank
// lines and lines starting with '#' or '//' skipped; LABEL is I/X/Y/Z in
// either case, its rightmost letter on qubit 0.  Fields are split on white
// space; a coefficient is a decimal literal, converted with strtod, finite.

namespace {

bool decimal_literal(const std::string& f) {
  size_t i = 0, digits = 0;
  if (i < f.size() && (f[i] == '+' || f[i] == '-')) ++i;
  while (i < f.size() && std::isdigit((unsigned char)f[i])) { ++i; ++digits; }
  if (i < f.size() && f[i] == '.') {
    ++i;
    while (i < f.size() && std::isdigit((unsigned char)f[i])) { ++i; ++digits; }
  }
  if (digits == 0) return false;
  if (i < f.size() && (f[i] == 'e' || f[i] == 'E')) {
    ++i;
    if (i < f.size() && (f[i] == '+' || f[i] == '-')) ++i;
    size_t ed = 0;
    while (i < f.size() && std::isdigit((unsigned char)f[i])) { ++i; ++ed; }
    if (ed == 0) return false;
  }
  return i == f.size();
}

bool coefficient(const std::string& f, double* v) {
  if (!decimal_literal(f)) return false;
  *v = std::strtod(f.c_str(), nullptr);
  return true;
}

std::vector<std::string> fields_of(const std::string& line) {
  std::vector<std::string> f;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
    size_t j = i;
    while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
    if (j > i) f.push_back(line.substr(i, j - i));
    i = j;
  }
  return f;
}

}  // namespace

std::vector<PauliRow> pauli_rows(const std::string& text) {
  std::vector<PauliRow> rows;
  size_t lineno = 0, begin = 0;
  while (begin <= text.size()) {
    size_t end = text.find('\n', begin);
    if (end == std::string::npos) end = text.size();
    const std::string line = text.substr(begin, end - begin);
    const bool last = end >= text.size();
    begin = end + 1;
    ++lineno;
    const auto f = fields_of(line);
    if (!f.empty() && f[0].compare(0, 1, "#") != 0 && f[0].compare(0, 2, "//") != 0) {
      PauliRow r;
      const std::string* label = nullptr;
      if (f.size() >= 3 && coefficient(f[0], &r.re) && coefficient(f[1], &r.im)) {
        label = &f[2];
      } else if (f.size() >= 2 && coefficient(f[0], &r.re)) {
        r.im = 0.0;
        label = &f[1];
      }
      if (!label) throw HostError(kParseError, "observable line " + std::to_string(lineno) + " is not 're [im] LABEL'");
      if (!std::isfinite(r.re) || !std::isfinite(r.im))
        throw HostError(kParseError, "observable line " + std::to_string(lineno) + ": coefficient out of range");
      const size_t n = label->size();
      for (size_t q = 0; q < n; ++q) {
        const char u = (char)std::toupper((unsigned char)(*label)[n - 1 - q]);
        if (u != 'I' && u != 'X' && u != 'Y' && u != 'Z')
          throw HostError(kParseError, "observable line " + std::to_string(lineno) + ": letters other than I, X, Y, Z");
        if (u != 'I') r.ops.push_back({(int)q, u});
      }
      rows.push_back(std::move(r));
    }
    if (last) break;
  }
  return rows;
}

}  // namespace tnbp_host
