// elliptic [-h] [-i] [-v] session
//
// The `elliptic` program (elliptic/drive.cpp:61-96, elliptic/helmholtz.cpp:
// 29-52) on the device: the session's Helmholtz / Poisson problem
// del^2 c - LAMBDA2 c = f, forcing from session.frc if present, else the
// USER-section `forcing` expression, else zero; the solution written to
// session.fld.  With a USER `exact` expression the max and L2 errors are
// printed (AuxField::errors).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../../include/semtex_b200.h"
#include "host/fieldfile.hpp"
#include "host/session.hpp"

namespace {

[[noreturn]] void fail(const std::string& what) {
  std::fprintf(stderr, "elliptic: %s\n", what.c_str());
  std::exit(EXIT_FAILURE);
}

void check(int rc, const char* what) {
  if (rc != STX_OK) fail(std::string(what) + ": " + stx_last_error());
}

const char* kUsage =
    "Usage: elliptic [options] session\n"
    "  options:\n"
    "  -h       ... print this message\n"
    "  -i       ... use iterative solver\n"
    "  -v[v...] ... increase verbosity level\n";

double token(const stx_context* ctx, const char* name) {
  double v = 0.0;
  check(stx_token(ctx, name, &v), name);
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  bool iterative = false;
  int verbose = 0;
  int a = 1;
  for (; a < argc && argv[a][0] == '-'; ++a) {
    if (!std::strcmp(argv[a], "-h")) {
      std::fputs(kUsage, stdout);
      return EXIT_SUCCESS;
    } else if (!std::strcmp(argv[a], "-i")) {
      iterative = true;
    } else if (argv[a][1] == 'v') {
      verbose += static_cast<int>(std::strlen(argv[a])) - 1;
    } else {
      std::fputs(kUsage, stderr);
      return EXIT_FAILURE;
    }
  }
  if (a != argc - 1) fail("no session definition file");
  const std::string session = argv[a];
  stx_context* ctx = nullptr;
  check(stx_context_create(session.c_str(), iterative ? "ITERATIVE=1" : nullptr, 0, nullptr, &ctx), "session");
  int np = 0, nz = 0, nel = 0, ps = 0;
  check(stx_context_geometry(ctx, &np, &nz, &nel, &ps), "geometry");
  char fields[64];
  check(stx_context_fields(ctx, fields, sizeof(fields)), "fields");
  const char c = fields[0];
  const size_t n = static_cast<size_t>(nz) * nel * np * np;
  const stx::Session S = stx::read_session(session, iterative ? "ITERATIVE=1" : "");
  std::vector<double> forcing(n, 0.0), solution(n, 0.0);
  if (std::ifstream(session + ".frc")) {  // elliptic/drive.cpp:258-341
    const stx::FieldFile F = stx::read_field(session + ".frc");
    if (F.data.empty() || F.data[0].size() != n) fail(session + ".frc does not match the session");
    forcing = F.data[0];
    if (verbose) std::printf("-- Forcing from %s.frc\n", session.c_str());
  } else {
    const std::string f = S.user_value("forcing");
    if (!f.empty()) check(stx_field_evaluate(ctx, f.c_str(), 0.0, forcing.data()), "forcing");
    if (verbose) std::printf("-- Forcing: %s\n", f.empty() ? "zero" : f.c_str());
  }
  stx_modal* sys = nullptr;
  check(stx_modal_create(ctx, c, token(ctx, "LAMBDA2"), token(ctx, "BETA"), 0, (nz + 1) / 2,
                         iterative ? STX_JACPCG : STX_DIRECT, &sys),
        "ModalMatrixSys");
  check(stx_elliptic_solve_host(sys, forcing.data(), solution.data()), "Field::solve");
  const std::string exact = S.user_value("exact");
  if (!exact.empty()) {
    std::vector<double> ex(n);
    check(stx_field_evaluate(ctx, exact.c_str(), 0.0, ex.data()), "exact");
    double linf = 0.0, l2 = 0.0;
    for (size_t i = 0; i < n; ++i) {
      const double d = std::fabs(solution[i] - ex[i]);
      linf = std::max(linf, d);
      l2 += d * d;
    }
    std::printf("Field '%c': norm_inf: %.4e, rms (nodal): %.4e\n", c, linf, std::sqrt(l2 / n));
  }
  stx::FieldFile out;
  const size_t slash = session.find_last_of('/');
  out.session = slash == std::string::npos ? session : session.substr(slash + 1);
  out.np = np;
  out.nz = nz;
  out.nel = nel;
  out.step = 1;  // Helmholtz() advances the step once before the dump
  out.time = 0.0;
  out.dt = token(ctx, "D_T");
  out.kinvis = token(ctx, "KINVIS");
  out.beta = token(ctx, "BETA");
  out.names = std::string(1, c);
  out.data.push_back(solution);
  stx::write_field(session + ".fld", out);
  stx_modal_destroy(sys);
  stx_context_destroy(ctx);
  return EXIT_SUCCESS;
}
