// Device checks of include/tnbp_b200.hpp: the estimator loop through the
// C++ interface (State) and the same program served (Server) give the same
// sum_k c_k <P_k>; a cancelled request throws; checkpoint round trip; a mixed
// server with an escalation threshold reports its request's run and BP
// statistics and stays within 1e-6.
// usage: hpp_device_checks <program.qasm> <observable.txt> <chi> <tol> <maxit> <sv_min> <scratch file>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>

#include "tnbp_b200.hpp"

namespace tb = tnbp_b200;

static std::string slurp(const char* p) {
  std::ifstream f(p);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

int main(int argc, char** argv) {
  if (argc < 8) return 2;
  const std::string qasm = slurp(argv[1]), pauli = slurp(argv[2]);
  const int chi = std::atoi(argv[3]), maxit = std::atoi(argv[5]);
  const double tol = std::atof(argv[4]), sv_min = std::atof(argv[6]);
  try {
    const tb::Edges edges = tb::EdgesFromQasm(qasm);
    const auto TPO = tb::QasmToTPO(qasm, edges);
    tb::State W = tb::InitTensorProductState(edges, TNBP_C128);
    std::vector<int> dims;
    std::vector<double> errs;
    for (const auto& layer : TPO) {
      tb::AbsorbTPO(W, layer);
      tb::BeliefPropagationLoop(W, tol, maxit);
      tb::Truncation(W, chi, sv_min, dims, errs);
    }
    const tb::cplx direct = tb::MeasurePauliSum(W, tb::ClassifyOps(pauli, edges));
    // checkpoint round trip through the C++ names
    tb::SaveTPS(W, argv[7]);
    tb::State W2(edges, TNBP_C128);
    tb::LoadTPS(W2, argv[7]);
    const tb::cplx reloaded = tb::MeasurePauliSum(W2, tb::ClassifyOps(pauli, edges));

    tb::Server srv(TNBP_C128, 0, 4);
    const int64_t a = srv.submit_qasm(qasm, pauli, chi, tol, maxit, sv_min);
    const int64_t b = srv.submit_qasm(qasm, pauli, chi, tol, maxit, sv_min);
    srv.cancel(b);
    tb::cplx served;
    int steps = 0;
    while (!srv.result(a, &served) && steps < 100000) { srv.step(); ++steps; }
    bool cancelled = false;
    try {
      tb::cplx x;
      srv.result(b, &x);
    } catch (const std::runtime_error&) {
      cancelled = true;
    }
    std::printf("direct %.17g %.17g served %.17g %.17g reloaded %.17g cancelled %d\n", direct.real(), direct.imag(),
                served.real(), served.imag(), reloaded.real(), (int)cancelled);
    // a mixed server with escalation and a threshold: the request's run
    // fields and BP statistics come back through the C++ interface
    tb::Server msrv(TNBP_MIXED, 0, 2);
    msrv.set_escalation(true);
    msrv.set_escalation_threshold(1e-2);
    bool bad_threshold = false;
    try {
      msrv.set_escalation_threshold(-1.0);
    } catch (const std::invalid_argument&) {
      bad_threshold = true;
    }
    const int64_t m = msrv.submit_qasm(qasm, pauli, chi, tol, maxit, sv_min);
    tb::cplx mixed;
    steps = 0;
    while (!msrv.result(m, &mixed) && steps < 100000) { msrv.step(); ++steps; }
    const auto inf = msrv.info(m);
    std::printf("mixed %.17g %.17g precision %d escalated %d converged %d loops %d min %.3g final %.3g bad %d\n",
                mixed.real(), mixed.imag(), inf.precision, (int)inf.escalated, (int)inf.bp_converged,
                inf.unconverged_loops, inf.worst_min_cond, inf.worst_final_cond, (int)bad_threshold);
    const bool info_ok = bad_threshold && inf.unconverged_loops >= 0 && inf.worst_final_cond >= inf.worst_min_cond &&
                         (inf.bp_converged == (inf.unconverged_loops == 0)) &&
                         (inf.escalated ? inf.precision == TNBP_C128 : inf.precision == TNBP_MIXED);
    const bool ok = std::abs(direct - served) <= 1e-10 && direct == reloaded && cancelled && info_ok &&
                    std::abs(mixed - direct) <= 1e-6;
    return ok ? 0 : 1;
  } catch (const std::exception& e) {
    std::printf("exception: %s\n", e.what());
    return 1;
  }
}
