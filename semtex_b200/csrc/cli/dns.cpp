// dns [-h] [-i] [-S|-C|-N] [-chk] [-v] session
//
// The `dns` program (dns/drive.cpp:56-160) on the device: the session's
// fields start from session.rst if present, else zero (Domain::restart,
// src/domain.cpp:123-156); N_STEP velocity-correction steps of integrate()
// (dns/integrate.cpp:66-200) with the advection form of -S (skew-symmetric),
// default (alternating skew-symmetric), -C (convective) or -N (Stokes); -i
// solves the viscous steps iteratively (token ITERATIVE = 1).
// Field dumps follow Domain::dump (src/domain.cpp:158-215): every IO_FLD
// steps and at the end, to session.chk (previous one kept as .chk.bak) with
// the final dump to session.fld, or with -chk all appended to session.fld.
// Every IO_CFL steps the CFL estimate and divergence energy are printed
// (Analyser::estimateCFL / divergence, src/analysis.cpp:382-443); with
// AVERAGE > 0 running averages are updated every IO_HIS steps and written
// to session.avg with each dump (Statistics, src/statistics.cpp).  Every
// IO_HIS and IO_FLD steps and at the end the HISTORY points go to
// session.his (Analyser::analyse, src/analysis.cpp:275-304) and the forces
// on the "wall" group to session.flx (DNSAnalyser, dns/dnsanalysis.cpp:
// 44-127); every IO_MDL steps the modal energies go to session.mdl
// (Analyser::modalEnergy, src/analysis.cpp:329-375); with IO_WSS > 0 and a
// "wall" group, every IO_WSS and IO_FLD steps and at the end the wall
// tractions are appended to session.wss (a header like a field file's, then
// the normal, in-plane and out-of-plane tractions, N_Z planes each,
// dns/dnsanalysis.cpp:130-250).  Particles listed in session.par are tracked
// every step (FluidParticle, src/particle.cpp; new ones at the listed places
// every SPAWN steps) and written to session.trk with the history points.
// With N_PHASE > 0 the phase averages are updated every STEPS_P / N_PHASE
// steps in session.<phase>.phs (Statistics::phaseUpdate,
// src/statistics.cpp:587-611; checks of src/analysis.cpp:141-172).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "../../../include/semtex_b200.h"
#include "host/fieldfile.hpp"
#include "host/session.hpp"

namespace {

[[noreturn]] void fail(const std::string& what) {
  std::fprintf(stderr, "dns: %s\n", what.c_str());
  std::exit(EXIT_FAILURE);
}

void check(int rc, const char* what) {
  if (rc != STX_OK) fail(std::string(what) + ": " + stx_last_error());
}

const char* kUsage =
    "Usage: dns [options] session-file\n"
    "  [options]:\n"
    "  -h       ... print this message\n"
    "  -i       ... use iterative solver for viscous steps\n"
    "  -v[v...] ... increase verbosity level\n"
    "  -chk     ... turn off checkpoint field dumps [default: selected]\n"
    "  -S|C|N   ... regular skew-symm || convective || Stokes advection\n";

double token(const stx_context* ctx, const char* name) {
  double v = 0.0;
  check(stx_token(ctx, name, &v), name);
  return v;
}

// Massless fluid particles (FluidParticle, src/particle.cpp:37-281, and the
// Analyser's handling of them, src/analysis.cpp:63-104, 206-226, 252-272):
// located in the mesh when made, moved every step by an Adams-Bashforth
// predictor and Adams-Moulton corrector of order min(steps, N_TIME) on the
// velocities probed on the device, relocated from their element (else by a
// full search); a particle that leaves the mesh stops.  z wraps into one
// period in 3D.
struct Particles {
  struct P {
    int id = 0, elmt = -1, step = 0;
    double ctime = 0.0, x = 0.0, y = 0.0, z = 0.0, r = 0.0, s = 0.0;
    std::vector<double> u, v, w;  // velocity levels, newest first
  };
  std::vector<P> all;
  std::vector<std::array<double, 3>> initial;  // places new particles start from
  int ncom = 2, tord = 1, nf = 1;
  double dt = 0.0, lz = 0.0;

  void setup(const stx_context* ctx, int nfields) {
    ncom = nfields > 3 ? 3 : 2;
    nf = nfields;
    tord = static_cast<int>(std::lround(token(ctx, "N_TIME")));
    dt = token(ctx, "D_T");
    lz = 2.0 * M_PI / token(ctx, "BETA");
  }
  double wrap(double z) const { return z < 0.0 ? lz - std::fmod(std::fabs(z), lz) : std::fmod(z, lz); }
  // FluidParticle::FluidParticle: false when the place is not in the mesh
  bool make(const stx_context* ctx, int id, const std::array<double, 3>& p, double t) {
    P q;
    q.id = id;
    q.ctime = t;
    q.x = p[0];
    q.y = p[1];
    double rs[2];
    check(stx_mesh_locate(ctx, 1, p.data(), &q.elmt, rs), "particle");
    if (q.elmt < 0) return false;
    q.r = rs[0];
    q.s = rs[1];
    q.z = ncom == 2 ? 0.0 : wrap(p[2]);
    q.u.assign(tord, 0.0);
    q.v.assign(tord, 0.0);
    q.w.assign(tord, 0.0);
    all.push_back(q);
    return true;
  }
  // velocities of the listed particles at (elmt, r, s, z)
  void probe(stx_dns* dns, const std::vector<int>& ix, const std::vector<double>& zs, std::vector<double>& vel) {
    const int n = static_cast<int>(ix.size());
    std::vector<int> el(n);
    std::vector<double> rs(2 * n), out(static_cast<size_t>(n) * nf);
    for (int k = 0; k < n; ++k) {
      el[k] = all[ix[k]].elmt;
      rs[2 * k] = all[ix[k]].r;
      rs[2 * k + 1] = all[ix[k]].s;
    }
    check(stx_dns_probe(dns, n, el.data(), rs.data(), zs.data(), out.data()), "particle");
    vel.assign(static_cast<size_t>(n) * 3, 0.0);
    for (int k = 0; k < n; ++k)
      for (int c = 0; c < ncom; ++c) vel[3 * k + c] = out[static_cast<size_t>(k) * nf + c];
  }
  void relocate(const stx_context* ctx, const std::vector<int>& ix, const std::vector<double>& xy) {
    const int n = static_cast<int>(ix.size());
    std::vector<int> el(n);
    std::vector<double> rs(2 * n);
    for (int k = 0; k < n; ++k) {
      el[k] = all[ix[k]].elmt;
      rs[2 * k] = all[ix[k]].r;
      rs[2 * k + 1] = all[ix[k]].s;
    }
    check(stx_mesh_relocate(ctx, n, xy.data(), el.data(), rs.data()), "particle");
    for (int k = 0; k < n; ++k) {
      all[ix[k]].elmt = el[k];
      all[ix[k]].r = rs[2 * k];
      all[ix[k]].s = rs[2 * k + 1];
    }
  }
  // FluidParticle::integrate for every particle still in the mesh
  void integrate(const stx_context* ctx, stx_dns* dns) {
    static const double kAB[3][3] = {{1.0, 0.0, 0.0}, {1.5, -0.5, 0.0}, {23.0 / 12.0, -16.0 / 12.0, 5.0 / 12.0}};
    static const double kAM[3][4] = {
        {0.5, 0.5, 0.0, 0.0}, {5.0 / 12.0, 8.0 / 12.0, -1.0 / 12.0, 0.0},
        {9.0 / 24.0, 19.0 / 24.0, -5.0 / 24.0, 1.0 / 24.0}};  // Integration::AdamsMoulton orders 2..4
    std::vector<int> ix;
    for (size_t k = 0; k < all.size(); ++k)
      if (all[k].elmt >= 0) ix.push_back(static_cast<int>(k));
    if (ix.empty()) return;
    const int n = static_cast<int>(ix.size());
    std::vector<double> zs(n), vel, xy(2 * n), zp(n);
    for (int k = 0; k < n; ++k) zs[k] = all[ix[k]].z;
    probe(dns, ix, zs, vel);  // predictor: the velocities where the particles are
    for (int k = 0; k < n; ++k) {
      P& q = all[ix[k]];
      const int N = std::min(++q.step, tord);
      q.u[0] = vel[3 * k];
      q.v[0] = vel[3 * k + 1];
      q.w[0] = vel[3 * k + 2];
      double x = q.x, y = q.y, z = q.z;
      for (int i = 0; i < N; ++i) {
        const double c = dt * kAB[N - 1][i];
        x += c * q.u[i];
        y += c * q.v[i];
        if (ncom == 3) z += c * q.w[i];
      }
      xy[2 * k] = x;
      xy[2 * k + 1] = y;
      zp[k] = z;
    }
    relocate(ctx, ix, xy);
    std::vector<int> in;  // still in the mesh
    std::vector<double> zin;
    for (int k = 0; k < n; ++k)
      if (all[ix[k]].elmt >= 0) {
        in.push_back(ix[k]);
        zin.push_back(zp[k]);
      }
    if (in.empty()) return;
    probe(dns, in, zin, vel);  // corrector: the velocities at the predicted places
    std::vector<double> xy2(2 * in.size());
    for (size_t k = 0; k < in.size(); ++k) {
      P& q = all[in[k]];
      const int N = std::min(q.step, tord);
      const double* c = kAM[N - 1];
      q.x += dt * c[0] * vel[3 * k];
      q.y += dt * c[0] * vel[3 * k + 1];
      if (ncom == 3) q.z += dt * c[0] * vel[3 * k + 2];
      for (int i = 1; i < N + 1; ++i) {
        q.x += dt * c[i] * q.u[i - 1];
        q.y += dt * c[i] * q.v[i - 1];
        if (ncom == 3) q.z += dt * c[i] * q.w[i - 1];
      }
      xy2[2 * k] = q.x;
      xy2[2 * k + 1] = q.y;
    }
    relocate(ctx, in, xy2);
    for (int k : in) {
      P& q = all[k];
      if (q.elmt >= 0 && ncom == 3) q.z = wrap(q.z);
      // rollv: every level one older, the oldest slot reused for the next
      std::rotate(q.u.rbegin(), q.u.rbegin() + 1, q.u.rend());
      std::rotate(q.v.rbegin(), q.v.rbegin() + 1, q.v.rend());
      std::rotate(q.w.rbegin(), q.w.rbegin() + 1, q.w.rend());
    }
  }
};

}  // namespace

int main(int argc, char** argv) {
  int advection = 1, verbose = 0;
  bool no_chk = false, iterative = false;
  int a = 1;
  for (; a < argc && argv[a][0] == '-'; ++a) {
    const std::string o = argv[a];
    if (o == "-h") {
      std::fputs(kUsage, stdout);
      return EXIT_SUCCESS;
    } else if (o == "-S") {
      advection = 0;
    } else if (o == "-C") {
      advection = 2;
    } else if (o == "-N") {
      advection = 3;
    } else if (o == "-chk") {
      no_chk = true;
    } else if (o.find_first_not_of('i', 1) == std::string::npos) {  // -i[i...]: viscous steps only
      iterative = true;
    } else if (o[1] == 'v') {
      verbose += static_cast<int>(o.size()) - 1;
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
  char fbuf[64];
  check(stx_context_fields(ctx, fbuf, sizeof(fbuf)), "fields");
  const std::string fields = fbuf;
  const size_t n = static_cast<size_t>(nz) * nel * np * np;
  stx_dns* dns = nullptr;
  check(stx_dns_create(ctx, advection, &dns), "integrate");
  // -- Domain::restart
  double t0 = 0.0;
  stx::FieldFile rst;
  const bool have_rst = static_cast<bool>(std::ifstream(session + ".rst"));
  if (have_rst) {
    rst = stx::read_field(session + ".rst");
    t0 = rst.time;
  }
  check(stx_dns_restart(dns, t0), "restart");
  std::vector<double> zero(n, 0.0);
  for (char c : fields) {
    const size_t k = have_rst ? rst.names.find(c) : std::string::npos;
    if (k != std::string::npos && rst.data[k].size() != n) fail(session + ".rst does not match the session");
    check(stx_dns_set_field(dns, c, k != std::string::npos ? rst.data[k].data() : zero.data()), "restart");
  }
  std::printf("-- Initial condition       : %s\n", have_rst ? ("read from file " + session + ".rst").c_str()
                                                             : "set to zero");
  const int nstep = static_cast<int>(std::lround(token(ctx, "N_STEP")));
  const int io_fld = std::max(1, static_cast<int>(std::lround(token(ctx, "IO_FLD"))));
  const int io_cfl = static_cast<int>(std::lround(token(ctx, "IO_CFL")));
  const int io_his = std::max(1, static_cast<int>(std::lround(token(ctx, "IO_HIS"))));
  const bool averaging = token(ctx, "AVERAGE") > 0.0;
  std::string avg_names;
  if (averaging) {  // Statistics::initialise: from session.avg, else zero
    char nb[64];
    check(stx_dns_stats_info(dns, nb, sizeof(nb), nullptr, -1), "statistics");
    avg_names = nb;
    if (std::ifstream(session + ".avg")) {
      const stx::FieldFile A = stx::read_field(session + ".avg");
      if (A.names != avg_names) fail(session + ".avg holds other averages than AVERAGE asks for");
      for (size_t k = 0; k < avg_names.size(); ++k) {
        if (A.data[k].size() != n) fail(session + ".avg does not match the session");
        check(stx_dns_stats_set(dns, avg_names[k], A.data[k].data()), "statistics");
      }
      check(stx_dns_stats_info(dns, nullptr, 0, nullptr, A.step), "statistics");
    }
  }
  // -- phase averaging (Analyser::Analyser, src/analysis.cpp:141-172)
  const int n_phase = static_cast<int>(std::lround(token(ctx, "N_PHASE")));
  int steps_p = 0;
  if (n_phase > 0) {
    double v = 0.0;
    if (stx_token(ctx, "STEPS_P", &v) == STX_OK) steps_p = static_cast<int>(std::lround(v));
    if (!averaging) fail("if N_PHASE is set, AVERAGE > 0 also required");
    if (!steps_p) fail("phase averaging is on but STEPS_P not set");
    if (steps_p % n_phase) fail("STEPS_P / N_PHASE non-integer");
    if (nstep % n_phase) fail("N_STEP / N_PHASE non-integer");
    if (io_fld != steps_p / n_phase) fail("phase averaging: IO_FLD != STEPS_P / N_PHASE");
  }
  // -- Analyser::Analyser (src/analysis.cpp:106-184) and DNSAnalyser::
  //    DNSAnalyser (dns/dnsanalysis.cpp:30-52): history points located in
  //    the mesh (shifted and scaled as X_SHIFT, X_SCALE, ... ask), files
  const int io_mdl = static_cast<int>(std::lround(token(ctx, "IO_MDL")));
  std::vector<int> his_id, his_el;
  std::vector<double> his_rs, his_z;
  {
    const stx::Session S = stx::read_session(session);
    const double xs = token(ctx, "X_SHIFT"), ys = token(ctx, "Y_SHIFT");
    const double xc = token(ctx, "X_SCALE"), yc = token(ctx, "Y_SCALE");
    for (const auto& h : S.history) {
      const double xy[2] = {(h.x + xs) * xc, (h.y + ys) * yc};
      int el = -1;
      double rs[2];
      check(stx_mesh_locate(ctx, 1, xy, &el, rs), "history");
      if (el < 0) {
        std::fprintf(stderr, "Analyser::Analyser: History point at (%f, %f, %f) not in mesh\n", xy[0], xy[1], h.z);
        continue;
      }
      his_id.push_back(h.id);
      his_el.push_back(el);
      his_rs.insert(his_rs.end(), rs, rs + 2);
      his_z.push_back(h.z);
    }
  }
  // particles (Analyser::Analyser, src/analysis.cpp:63-104): session.par
  // lines "id time ctime x y z", placed as given (shifted and scaled)
  Particles parts;
  std::ofstream trk;
  const int spawn = static_cast<int>(std::lround(token(ctx, "SPAWN")));
  {
    std::ifstream pf(session + ".par");
    if (pf) {
      parts.setup(ctx, static_cast<int>(fields.size()));
      const double xs = token(ctx, "X_SHIFT"), ys = token(ctx, "Y_SHIFT");
      const double xc = token(ctx, "X_SCALE"), yc = token(ctx, "Y_SCALE");
      double t0 = 0.0;
      check(stx_dns_state(dns, nullptr, &t0), "state");
      trk.open(session + ".trk");
      if (!trk) fail("can't open particle track file");
      trk.setf(std::ios::scientific, std::ios::floatfield);
      trk.precision(6);
      int id, i = 0;
      double tm, ct;
      std::array<double, 3> p;
      while (pf >> id >> tm >> ct >> p[0] >> p[1] >> p[2]) {
        p[0] = (p[0] + xs) * xc;
        p[1] = (p[1] + ys) * yc;
        if (!parts.make(ctx, ++i, p, t0))
          std::fprintf(stderr, "Analyser::Analyser: Particle at (%f, %f, %f) not in mesh\n", p[0], p[1], p[2]);
        else if (spawn)
          parts.initial.push_back(p);
      }
    }
  }
  std::ofstream his, mdl;
  if (!his_id.empty()) {
    his.open(session + ".his");
    if (!his) fail("can't open history file");
    his.setf(std::ios::scientific, std::ios::floatfield);
    his.precision(6);
  }
  if (io_mdl) {
    mdl.open(session + ".mdl");
    if (!mdl) fail("can't open modal energy file");
    mdl << "#     Time Mode         Energy" << std::endl << "# ----------------------------" << std::endl;
  }
  std::ofstream flx(session + ".flx");
  if (!flx) fail("can't open flux file");
  flx << "# DNS state information file" << std::endl
      << "# Step Time [Fpre Fvis Ftot]-axis" << std::endl
      << "# -------------------------------" << std::endl;
  // wall tractions (DNSAnalyser::DNSAnalyser, dns/dnsanalysis.cpp:53-81)
  const int io_wss = static_cast<int>(std::lround(token(ctx, "IO_WSS")));
  int wss_line = 0;
  check(stx_dns_wall_traction(dns, &wss_line, nullptr), "wall traction");
  std::ofstream wss;
  std::vector<double> wss_val;
  if (io_wss > 0 && wss_line > 0) {
    wss.open(session + ".wss", std::ios::binary);
    if (!wss) fail("can't open WSS file");
    wss_val.resize(static_cast<size_t>(3) * nz * wss_line);
  }
  std::vector<double> his_val(his_id.size() * fields.size());
  std::vector<double> ek((nz + 1) / 2);
  const double dt = token(ctx, "D_T");
  const bool chkpoint = !no_chk && token(ctx, "CHKPOINT") != 0.0;
  stx::FieldFile out;
  const size_t slash = session.find_last_of('/');
  out.session = slash == std::string::npos ? session : session.substr(slash + 1);
  out.np = np;
  out.nz = nz;
  out.nel = nel;
  out.dt = dt;
  out.kinvis = token(ctx, "KINVIS");
  out.beta = token(ctx, "BETA");
  out.names = fields;
  out.data.assign(fields.size(), std::vector<double>(n));
  int step = 0;
  while (step < nstep) {
    int next = std::min(nstep, (step / io_fld + 1) * io_fld);
    if (io_cfl > 0) next = std::min(next, (step / io_cfl + 1) * io_cfl);
    next = std::min(next, (step / io_his + 1) * io_his);
    if (io_mdl > 0) next = std::min(next, (step / io_mdl + 1) * io_mdl);
    if (wss.is_open()) next = std::min(next, (step / io_wss + 1) * io_wss);
    if (trk.is_open()) next = step + 1;  // particles move every step
    if (verbose) {  // the step line of DNSAnalyser::analyse, one step at a time
      for (; step < next; ++step) {
        check(stx_dns_advance(dns, 1), "integrate");
        double t;
        check(stx_dns_state(dns, nullptr, &t), "state");
        std::printf("Step: %d  Time: %g\n", step + 1, t);
      }
    } else {
      check(stx_dns_advance(dns, next - step), "integrate");
      step = next;
    }
    double time;
    check(stx_dns_state(dns, nullptr, &time), "state");
    if (trk.is_open()) {  // Analyser::analyse: new particles, then every particle moves
      if (spawn && step % spawn == 0) {
        int i = 0;
        for (const auto& p : parts.initial) parts.make(ctx, ++i, p, time);
      }
      parts.integrate(ctx, dns);
    }
    if (io_cfl > 0 && step % io_cfl == 0) {
      double inv = 0.0, div = 0.0;
      check(stx_dns_cfl(dns, &inv), "CFL");
      check(stx_dns_divergence_energy(dns, &div), "divergence");
      const double dt_max = 0.9 * 0.7 / inv;
      std::printf("-- CFL: %g, dt (max): %g, dt (set): %g (%d%%)\n", inv * dt, dt_max, dt,
                  static_cast<int>(100.0 * dt / dt_max));
      std::printf("------- Divergence Energy: %g\n", div);
    }
    // -- phase averages (Statistics::phaseUpdate): the second set of
    //    averages on the device takes session.<phase>.phs (or zero), is
    //    updated and written back; the running averages stay untouched
    if (n_phase > 0 && step % (steps_p / n_phase) == 0) {
      const int iphase = (step % steps_p) / (steps_p / n_phase);
      const std::string fn = session + "." + std::to_string(iphase) + ".phs";
      check(stx_dns_stats_swap(dns), "statistics");
      int nphs = 0;
      if (std::ifstream(fn)) {
        const stx::FieldFile A = stx::read_field(fn);
        if (A.names != avg_names) fail(fn + " holds other averages than AVERAGE asks for");
        for (size_t k = 0; k < avg_names.size(); ++k) {
          if (A.data[k].size() != n) fail(fn + " does not match the session");
          check(stx_dns_stats_set(dns, avg_names[k], A.data[k].data()), "statistics");
        }
        nphs = A.step;
      } else {
        for (size_t k = 0; k < avg_names.size(); ++k)
          check(stx_dns_stats_set(dns, avg_names[k], zero.data()), "statistics");
      }
      check(stx_dns_stats_info(dns, nullptr, 0, nullptr, nphs), "statistics");
      check(stx_dns_stats_update(dns), "statistics");
      stx::FieldFile A = out;
      A.time = time;
      A.names = avg_names;
      A.data.assign(avg_names.size(), std::vector<double>(n));
      check(stx_dns_stats_info(dns, nullptr, 0, &A.step, -1), "statistics");
      for (size_t k = 0; k < avg_names.size(); ++k)
        check(stx_dns_stats_get(dns, avg_names[k], A.data[k].data()), "statistics");
      stx::write_field(fn, A);
      check(stx_dns_stats_swap(dns), "statistics");
    }
    // -- history points and wall forces at IO_HIS / IO_FLD steps and at
    //    the end (Analyser::analyse, DNSAnalyser::analyse)
    if (step % io_his == 0 || step % io_fld == 0 || step == nstep) {
      for (const auto& q : parts.all)
        if (q.elmt >= 0)
          trk << std::setw(6) << q.id << std::setw(14) << time << std::setw(14) << q.ctime << std::setw(14) << q.x
              << std::setw(14) << q.y << std::setw(14) << q.z << std::endl;
      if (!his_id.empty()) {
        const int nf = static_cast<int>(fields.size());
        check(stx_dns_probe(dns, static_cast<int>(his_id.size()), his_el.data(), his_rs.data(), his_z.data(),
                            his_val.data()),
              "history");
        for (size_t i = 0; i < his_id.size(); ++i) {
          his << std::setw(4) << his_id[i] << std::setprecision(8) << std::setw(15) << time << std::setprecision(6);
          for (int j = 0; j < nf - 1; ++j) his << std::setw(14) << his_val[i * nf + j];
          his << std::setprecision(11) << std::setw(19) << his_val[i * nf + nf - 1] << std::setprecision(6)
              << std::endl;
        }
      }
      double pf[3], vf[3];
      check(stx_dns_wall_forces(dns, pf, vf), "wall forces");
      char line[256];
      std::snprintf(line, sizeof(line),
                    "%6d %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g %#10.6g", step,
                    time, pf[0], vf[0], pf[0] + vf[0], pf[1], vf[1], pf[1] + vf[1], pf[2], vf[2], pf[2] + vf[2]);
      flx << line << std::endl;
    }
    if (averaging && step % io_his == 0) check(stx_dns_stats_update(dns), "statistics");
    if (wss.is_open() && (step % io_wss == 0 || step % io_fld == 0 || step == nstep)) {
      check(stx_dns_wall_traction(dns, &wss_line, wss_val.data()), "wall traction");
      char created[64];
      const std::time_t now = std::time(nullptr);
      std::strftime(created, sizeof(created), "%a %b %d %H:%M:%S %Y", std::localtime(&now));
      const bool little = [] {
        const unsigned one = 1;
        return *reinterpret_cast<const unsigned char*>(&one) == 1;
      }();
      const std::string fmt = std::string("binary IEEE ") + (little ? "little-endian" : "big-endian");
      char h[1024];
      int n = 0;
      n += std::snprintf(h + n, sizeof(h) - n, "%-25s Session\n", out.session.c_str());
      n += std::snprintf(h + n, sizeof(h) - n, "%-25s Created\n", created);
      n += std::snprintf(h + n, sizeof(h) - n, "%-5d1    %-5d %-10dNr, Ns, Nz, Elements\n", np, nz, wss_line / np);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25d Step\n", step);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25.6g Time\n", time);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25.6g Time step\n", dt);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25.6g Kinvis\n", out.kinvis);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25.6g Beta\n", out.beta);
      n += std::snprintf(h + n, sizeof(h) - n, "%-25s Fields written\n", "nts");
      n += std::snprintf(h + n, sizeof(h) - n, "%-25s Format\n", fmt.c_str());
      wss.write(h, n);
      wss.write(reinterpret_cast<const char*>(wss_val.data()),
                static_cast<std::streamsize>(sizeof(double) * wss_val.size()));
      wss.flush();
      if (!wss) fail("unable to write WSS output");
    }
    if (io_mdl > 0 && step % io_mdl == 0) {  // Analyser::modalEnergy
      check(stx_dns_modal_energy(dns, ek.data()), "modal energy");
      for (size_t m = 0; m < ek.size(); ++m)
        mdl << std::setw(10) << time << std::setw(5) << m << std::setw(15) << ek[m] << std::endl;
    }
    const bool periodic = step % io_fld == 0, initial = step == io_fld, final = step == nstep;
    if (periodic || final) {
      for (size_t k = 0; k < fields.size(); ++k)
        check(stx_dns_get_field(dns, fields[k], out.data[k].data()), "dump");
      out.step = step;
      out.time = time;
      if (chkpoint) {
        if (final) {
          stx::write_field(session + ".fld", out);
        } else {
          if (!initial) std::rename((session + ".chk").c_str(), (session + ".chk.bak").c_str());
          stx::write_field(session + ".chk", out);
        }
      } else {
        stx::write_field(session + ".fld", out, !initial);
      }
      if (averaging) {  // Statistics::dump: the averages, step = number of updates
        stx::FieldFile A = out;
        A.names = avg_names;
        A.data.assign(avg_names.size(), std::vector<double>(n));
        int navg = 0;
        check(stx_dns_stats_info(dns, nullptr, 0, &navg, -1), "statistics");
        A.step = navg;
        for (size_t k = 0; k < avg_names.size(); ++k)
          check(stx_dns_stats_get(dns, avg_names[k], A.data[k].data()), "statistics");
        stx::write_field(session + ".avg", A);
      }
    }
  }
  int status = 0;
  check(stx_dns_status(dns, &status), "status");
  if (status) fail("a bounded wait on the device expired: the fields are not valid");
  stx_dns_destroy(dns);
  stx_context_destroy(ctx);
  return EXIT_SUCCESS;
}
