// DNS velocity-correction time stepping on the device (C ABI stx_dns_*).
//
// Host restatement of integrate() (dns/integrate.cpp:66-200): the same
// multi-level storage Us / Uf rolled by pointer (rollm, src/sem.h:108-122),
// the same sub-steps in the same order, every field operation a device
// kernel.  Cartesian coordinates; body forcing from the <FORCE> section
// (FieldForce, dns/fieldforce.cpp) except white noise; velocity BCs essential or
// natural (time-dependent values re-evaluated each step); pressure BCs
// essential, natural or high-order (<H>, BCmgr::maintainFourier /
// evaluateCNBCp, src/bcmgr.cpp:1036-1331, computed on the device each step).
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <memory>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/semtex_b200.h"
#include "host/fieldfile.hpp"
#include "kernels/dns_kernels.cuh"
#include "kernels/outflow.cuh"
#include "kernels/force.cuh"
#include "kernels/helmholtz.cuh"
#include "dns_internal.hpp"
#include "stx_internal.hpp"

using namespace stx;

namespace stx {

const double kSS[4][4] = {{0, 0, 0, 0}, {1.0, -1.0, 0, 0}, {1.5, -2.0, 0.5, 0}, {11.0 / 6.0, -3.0, 1.5, -1.0 / 3.0}};
const double kEX[4][3] = {{0, 0, 0}, {1.0, 0, 0}, {2.0, -1.0, 0}, {3.0, -3.0, 1.0}};

}  // namespace stx

namespace {

struct DnsError : std::runtime_error {
  int code;
  DnsError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw DnsError(STX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void ckstx(int rc) {
  if (rc != STX_OK) throw DnsError(rc, stx_last_error());
}

bool depends_on_t(const std::string& expr) {
  for (size_t i = 0; i < expr.size(); ++i)
    if (expr[i] == 't' && (i == 0 || !(std::isalnum(static_cast<unsigned char>(expr[i - 1])) || expr[i - 1] == '_')) &&
        (i + 1 == expr.size() || !(std::isalnum(static_cast<unsigned char>(expr[i + 1])) || expr[i + 1] == '_')))
      return true;
  return false;
}

template <class F>
int dns_guarded(F&& f) {
  try {
    f();
    set_last_error("");
    return STX_OK;
  } catch (const DnsError& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return STX_ESESSION;
  }
}

}  // namespace


namespace {

void transform(stx_dns* d, double* f, int sign) {
  ck(z_transform(f, d->ctx->M.nz, d->ctx->M.plane_size, sign, d->ctx->d_twiddle, nullptr, d->ctx->stream,
                 d->ctx->dg.pdl != 0),
     "transform");
}

void copy(stx_dns* d, double* dst, const double* src) {
  // a copy-engine copy (measured faster than a copy kernel launched
  // programmatically dependent)
  ck(cudaMemcpyAsync(dst, src, sizeof(double) * d->fsize, cudaMemcpyDeviceToDevice, d->ctx->stream), "copy");
}

// AuxField::transform32 INVERSE: Fourier f (N_Z planes) zero-padded to nz32
// planes, inverse transform of length nz32, into out.
void inverse32(stx_dns* d, const double* f, double* out) {
  stx_context* ctx = d->ctx;
  const size_t ps = ctx->M.plane_size, nz = ctx->M.nz;
  ck(cudaMemcpyAsync(out, f, sizeof(double) * nz * ps, cudaMemcpyDeviceToDevice, ctx->stream), "pad");
  ck(cudaMemsetAsync(out + nz * ps, 0, sizeof(double) * (d->nz32 - nz) * ps, ctx->stream), "pad");
  ck(z_transform(out, d->nz32, ctx->M.plane_size, STX_INVERSE, d->twiddle32, nullptr, ctx->stream), "transform32");
}

// AuxField::transform32 FORWARD: transform of length nz32 in place, the first
// N_Z planes copied to out (or left in place when out is null).
void forward32(stx_dns* d, double* io, double* out) {
  stx_context* ctx = d->ctx;
  const size_t ps = ctx->M.plane_size, nz = ctx->M.nz;
  ck(z_transform(io, d->nz32, ctx->M.plane_size, STX_FORWARD, d->twiddle32, nullptr, ctx->stream), "transform32");
  if (out) ck(cudaMemcpyAsync(out, io, sizeof(double) * nz * ps, cudaMemcpyDeviceToDevice, ctx->stream), "truncate");
}

// -- body forcing (dns/fieldforce.cpp) ------------------------------------

constexpr double kEpsDp = 6.0e-14;  // EPSDP, veclib/cveclib.h:58

ExprOp* upload_program(stx_dns* d, const ExprProgram& P) {
  auto* p = static_cast<ExprOp*>(d->arena.alloc(sizeof(ExprOp) * std::max<size_t>(P.ops.size(), 1)));
  if (!P.ops.empty())
    ck(cudaMemcpy(p, P.ops.data(), sizeof(ExprOp) * P.ops.size(), cudaMemcpyHostToDevice), "program upload");
  return p;
}

// A forcing field: the expression at every node of the forcing grid (the
// reference's AuxField = "expr"), evaluated on the device.
double* force_field(stx_dns* d, const std::string& expr) {
  auto& F = d->force;
  const Mesh& M = d->ctx->M;
  const size_t n = static_cast<size_t>(F.nzl) * M.plane_size;
  auto* f = static_cast<double*>(d->arena.alloc(sizeof(double) * n));
  ck(cudaMemset(f, 0, sizeof(double) * n), "memset");
  const ExprProgram P = d->ctx->S.tokens.compile(expr);
  ExprOp* ops = upload_program(d, P);
  ck(eval_program_field(ops, static_cast<int>(P.ops.size()), f, F.nzl, M.plane_size, M.nplane, F.x, F.y, F.dz,
                        d->ctx->S.tokens.value("t"), d->ctx->stream),
     "force field");
  ck(cudaStreamSynchronize(d->ctx->stream), "force field");
  return f;
}

// Velocity-component forcing fields read from a field file (VirtualForce::
// readSteadyFromFile, dns/fieldforce.cpp:217-233, readField, src/misc.cpp:
// 182-222): fields named u, v, w; one named in no dump stays zero.
void force_from_file(stx_dns* d, std::string fname, double** out) {
  const size_t a = fname.find_first_not_of(" \t"), b = fname.find_last_not_of(" \t");
  fname = a == std::string::npos ? "" : fname.substr(a, b - a + 1);
  auto& F = d->force;
  const Mesh& M = d->ctx->M;
  if (d->nz32) throw DnsError(STX_EUNSUPPORTED, "forcing from a file with DEALIAS: the file holds N_Z planes");
  FieldFile ff;
  try {
    ff = read_field(fname);
  } catch (const std::exception& e) {
    throw DnsError(STX_ESESSION, std::string("can't open '") + fname + "' file: " + e.what());
  }
  if (ff.np != M.np || ff.nz != M.nz || ff.nel != M.nel)
    throw DnsError(STX_ESESSION, "forcing file '" + fname + "': sizes differ from the session");
  const size_t n = static_cast<size_t>(F.nzl) * M.plane_size;
  for (int i = 0; i < d->ncom; ++i) {
    out[i] = static_cast<double*>(d->arena.alloc(sizeof(double) * n));
    ck(cudaMemset(out[i], 0, sizeof(double) * n), "memset");
    const size_t k = ff.names.find(static_cast<char>('u' + i));
    if (k == std::string::npos) continue;
    ck(cudaMemcpy2D(out[i], sizeof(double) * M.plane_size, ff.data[k].data(), sizeof(double) * M.nplane,
                    sizeof(double) * M.nplane, M.nz, cudaMemcpyHostToDevice),
       "forcing upload");
  }
}

// FieldForce::FieldForce and the class constructors (dns/fieldforce.cpp:
// 31-73, 240-822): which terms the FORCE section switches on.
void force_setup(stx_dns* d) {
  const Session& S = d->ctx->S;
  const TokenTable& T = S.tokens;
  auto& F = d->force;
  if (!S.has_force) return;
  F.on = true;
  const Mesh& M = d->ctx->M;
  F.nzl = d->nz32 ? d->nz32 : M.nz;
  F.dz = 2.0 * M_PI / d->beta / F.nzl;
  F.x = static_cast<double*>(d->arena.alloc(sizeof(double) * M.nplane));
  F.y = static_cast<double*>(d->arena.alloc(sizeof(double) * M.nplane));
  ck(cudaMemcpy(F.x, M.x.data(), sizeof(double) * M.nplane, cudaMemcpyHostToDevice), "x");
  ck(cudaMemcpy(F.y, M.y.data(), sizeof(double) * M.nplane, cudaMemcpyHostToDevice), "y");
  const char xyz[3] = {'X', 'Y', 'Z'};
  auto str = [&](const std::string& tok, std::string& v) { return S.force_value(tok, v); };
  auto num = [&](const std::string& tok, double& v) {
    std::string s;
    if (!str(tok, s)) return false;
    v = T.eval(s);
    return true;
  };
  auto tok = [&](const char* stem, int i) { return std::string(stem) + xyz[i]; };
  std::string s;
  // ConstForce (:240-270)
  for (int i = 0; i < d->ncom; ++i) num(tok("CONST_", i), F.cst[i]);
  // WhiteNoiseForce (:347-384): a random stream of the reference's own
  for (int i = 0; i < d->ncom; ++i) {
    double eps = 0.0;
    if (num(tok("WHITE_EPS_", i), eps) && std::fabs(eps) > kEpsDp)
      throw DnsError(STX_EUNSUPPORTED, "WHITE_EPS_* (white-noise forcing) is not supported");
  }
  // SteadyForce (:273-332)
  if (str("STEADY_FILE", s)) {
    force_from_file(d, s, F.steady);
  } else {
    for (int i = 0; i < d->ncom; ++i)
      if (str(tok("STEADY_", i), s)) F.steady[i] = force_field(d, s);
  }
  // ModulatedForce (:387-446)
  bool alpha_found = false;
  for (int i = 0; i < d->ncom; ++i) {
    F.alpha[i] = "0";
    if (str(tok("MOD_ALPHA_", i), F.alpha[i])) alpha_found = true;
  }
  if (alpha_found) {
    if (str("MOD_A_FILE", s)) {
      force_from_file(d, s, F.moda);
    } else {
      for (int i = 0; i < d->ncom; ++i)
        if (str(tok("MOD_A_", i), s)) F.moda[i] = force_field(d, s);
    }
    for (int i = 0; i < d->ncom; ++i) F.tdep = F.tdep || (F.moda[i] && depends_on_t(F.alpha[i]));
  }
  // SpatioTemporalForce (:463-496)
  for (int i = 0; i < d->ncom; ++i)
    if (str(tok("SPATIOTEMP_ALPHA_", i), s)) {
      const ExprProgram P = T.compile(s);
      F.st[i] = upload_program(d, P);
      F.nst[i] = static_cast<int>(P.ops.size());
      F.tdep = true;
    }
  // SpongeForce (:516-560).  A mask re-evaluated every SPONGE_UPDATE steps is
  // also evaluated here, so that it holds values before its first update.
  if (str("SPONGE_M", s)) {
    F.mask = force_field(d, s);
    std::string u;
    if (str("SPONGE_UPDATE", u)) {
      F.sponge_update = static_cast<int>(std::lround(T.eval(u)));
      const ExprProgram P = T.compile(s);
      F.mask_prog = upload_program(d, P);
      F.nmask = static_cast<int>(P.ops.size());
      F.tdep = F.tdep || F.sponge_update != 0;
    }
    const char* ref[3] = {"SPONGE_U", "SPONGE_V", "SPONGE_W"};
    for (int i = 0; i < d->ncom; ++i) {
      std::string r = "0";
      str(ref[i], r);
      F.uref[i] = force_field(d, r);
    }
  }
  // DragForce (:581-611)
  if (str("DRAG_M", s)) F.drag = force_field(d, s);
  // CoriolisForce (:631-723): in 2-D only the z components are read
  {
    std::string u;
    const int unsteady = str("CORIOLIS_UNSTEADY", u) ? static_cast<int>(std::lround(T.eval(u))) : 0;
    bool enabled = false;
    for (int i = 0; i < 3; ++i) {
      F.omega[i] = "0";
      F.domega[i] = "0";
      if (d->ncom == 3 || i == 2) {
        if (str(tok("CORIOLIS_OMEGA_", i), F.omega[i])) enabled = true;
        if (unsteady) str(tok("CORIOLIS_DOMEGA_", i) + "_DT", F.domega[i]);
      }
    }
    if (enabled) {
      F.coriolis = unsteady ? 2 : 1;
      if (!unsteady)
        for (int i = 0; i < 3; ++i) F.m2o[i] = -2.0 * T.eval(F.omega[i]);
      F.tdep = F.tdep || unsteady;
    }
  }
  // SFDForce (:759-789)
  {
    double delta = 0.0, chi = 0.0;
    const bool hd = num("SFD_DELTA", delta), hc = num("SFD_CHI", chi);
    if (hd || hc) {
      if (!(hd && hc)) throw DnsError(STX_ESESSION, "SFD_DELTA and SFD_CHI must be paired.");
      F.chi = chi;
      F.rate = d->dt / delta;
      const size_t n = static_cast<size_t>(F.nzl) * M.plane_size;
      for (int i = 0; i < d->ncom; ++i) {
        F.qbar[i] = static_cast<double*>(d->arena.alloc(sizeof(double) * n));
        ck(cudaMemset(F.qbar[i], 0, sizeof(double) * n), "memset");
      }
    }
  }
  for (int i = 0; i < d->ncom; ++i)
    F.physical = F.physical || F.steady[i] || F.moda[i] || F.st[i] || F.qbar[i];
  F.physical = F.physical || F.mask || F.drag || F.coriolis;
}

// FieldForce::addPhysical (dns/fieldforce.cpp:75-107) for component i: the
// force added to N, physical values on the forcing grid; Up the physical
// velocities on the same grid.
void force_physical(stx_dns* d, int i, double* N, const std::vector<double*>& Up) {
  auto& F = d->force;
  if (!F.physical) return;
  const Mesh& M = d->ctx->M;
  const TokenTable& T = d->ctx->S.tokens;
  cudaStream_t st = d->ctx->stream;
  std::map<std::string, double> vars{{"t", d->time}};
  ForceArgs a{};
  a.N = N;
  for (int c = 0; c < d->ncom; ++c) a.U[c] = Up[c];
  a.ncom = d->ncom;
  a.com = i;
  a.nzl = F.nzl;
  a.plane_size = M.plane_size;
  a.nplane = M.nplane;
  a.dz = F.dz;
  a.t = F.tdep ? d->time : 0.0;
  a.x = F.x;
  a.y = F.y;
  if (F.mask) {
    if (i == 0 && F.sponge_update && d->step % F.sponge_update == 0)
      ck(eval_program_field(F.mask_prog, F.nmask, F.mask, F.nzl, M.plane_size, M.nplane, F.x, F.y, F.dz, d->time,
                            st),
         "sponge mask");
    a.mask = F.mask;
    a.uref = F.uref[i];
  }
  if (F.coriolis) {
    if (F.coriolis == 2 && i == 0)
      for (int c = d->ncom == 2 ? 2 : 0; c < 3; ++c) {
        F.o[c] = T.eval(F.omega[c], &vars);
        F.mo[c] = -F.o[c];
        F.m2o[c] = -2.0 * F.o[c];
        F.dodt[c] = -T.eval(F.domega[c], &vars);
      }
    a.coriolis = F.coriolis;
    for (int c = 0; c < 3; ++c) {
      a.m2o[c] = F.m2o[c];
      a.o[c] = F.o[c];
      a.mo[c] = F.mo[c];
      a.dodt[c] = F.dodt[c];
    }
  }
  a.steady = F.steady[i];
  if (F.moda[i]) {
    a.alpha = T.eval(F.alpha[i], &vars);
    if (std::fabs(a.alpha) > kEpsDp) a.moda = F.moda[i];
  }
  a.st = F.st[i];
  a.nst = F.nst[i];
  a.drag = F.drag;
  if (F.qbar[i]) {
    a.qbar = F.qbar[i];
    a.chi = F.chi;
    a.rate = F.rate;
    a.sfd_init = F.sfd_started ? 0 : 1;
    if (i == d->ncom - 1) F.sfd_started = true;
  }
  ck(dns_force_physical(a, st), "force");
}

// FieldForce::addFourier (dns/fieldforce.cpp:110-137): ConstForce on mode 0.
void force_fourier(stx_dns* d, int i, double* N) {
  const auto& F = d->force;
  if (F.on && std::fabs(F.cst[i]) > kEpsDp)
    ck(dns_force_const(N, d->ctx->M.nplane, F.cst[i], d->ctx->stream), "const force");
}

// The same nonlinear terms with every product on the 3/2-padded z grid.
void nonlinear32(stx_dns* d, int form) {
  stx_context* ctx = d->ctx;
  DevGeom g32 = ctx->dg;
  g32.nz = d->nz32;
  cudaStream_t st = ctx->stream;
  for (int i = 0; i < d->ncom; ++i) {
    copy(d, d->Us[0][i], d->u[i]);
    inverse32(d, d->u[i], d->Up32[i]);
  }
  const DevNumbering& Nm = ctx->fields.at(d->names[0]).dn;
  for (int i = 0; i < d->ncom; ++i) {
    double* N = d->Uf[0][i];
    if (form < 0) {
      if (d->force.physical) {  // the force alone, on the padded grid
        ck(cudaMemsetAsync(d->A32, 0, sizeof(double) * d->nz32 * ctx->M.plane_size, st), "zero");
        force_physical(d, i, d->A32, d->Up32);
        forward32(d, d->A32, N);
      } else {
        ck(cudaMemsetAsync(N, 0, sizeof(double) * d->fsize, st), "zero");
      }
    } else {
      NonlinearArgs a{};
      a.U0 = d->Up32[0];
      a.U1 = d->Up32[1];
      a.U2 = d->Up32[2];
      a.Ui = d->Up32[i];
      a.N = d->A32;
      a.form = form;
      if (form != 2) {  // u_j grad: w * IFFT32(dz U_i)
        ck(dns_grad_z(ctx->dg, d->Us[0][i], d->tmp0, d->beta, st), "gradz");
        inverse32(d, d->tmp0, d->B32);
        a.Tc = d->B32;
      }
      if (form != 1) {  // div(uu): IFFT32(dz FFT32(u_i w))
        ck(dns_product(g32, d->Up32[i], d->Up32[2], d->C32, st), "product");
        forward32(d, d->C32, nullptr);
        ck(dns_grad_z(ctx->dg, d->C32, d->tmp1, d->beta, st), "gradz");
        inverse32(d, d->tmp1, d->C32);
        a.Tk = d->C32;
      }
      ck(dns_nonlinear(g32, a, st), "nonlinear");
      force_physical(d, i, d->A32, d->Up32);
      forward32(d, d->A32, N);
    }
    force_fourier(d, i, N);
    ck(dns_smooth(ctx->dg, Nm, N, d->dsswork, st), "smooth");
  }
}

void rollm_levels(std::vector<double*>& v);

// Nonlinear terms N(u) into Uf[0], copy of u into Us[0] (dns/nonlinear.cpp).
int next_form(const stx_dns* d) {
  switch (d->form) {
    case 0: return 0;
    case 1: return d->toggle ? 1 : 2;
    case 2: return 1;
    default: return -1;
  }
}

void nonlinear(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  const bool z3 = d->ndim == 3;
  const int form = next_form(d);  // 0 skew, 1 convective, 2 conservative, -1 Stokes
  if (d->nz32) {
    nonlinear32(d, form);
    if (d->form == 1) d->toggle = 1 - d->toggle;
    return;
  }
  for (int i = 0; i < d->ncom; ++i) {
    copy(d, d->Us[0][i], d->u[i]);
    copy(d, d->Up[i], d->u[i]);
    transform(d, d->Up[i], STX_INVERSE);
  }
  if (d->oe.no) {  // BCmgr::maintainPhysical (src/bcmgr.cpp:998-1034): edge velocities of this step
    rollm_levels(d->o_uvw);
    ck(outflow_gather(g, d->oe, d->Up[0], d->Up[1], d->ncom > 2 ? d->Up[2] : nullptr, d->o_uvw[0], st),
       "outflow edge velocities");
  }
  const DevNumbering& Nm = ctx->fields.at(d->names[0]).dn;
  for (int i = 0; i < d->ncom; ++i) {
    double* N = d->Uf[0][i];
    if (form < 0) {
      ck(cudaMemsetAsync(N, 0, sizeof(double) * d->fsize, st), "zero");
    } else {
      NonlinearArgs a{};
      a.U0 = d->Up[0];
      a.U1 = d->Up[1];
      a.U2 = z3 ? d->Up[2] : nullptr;
      a.Ui = d->Up[i];
      a.N = N;
      a.form = form;
      if (z3 && form != 2) {  // u_j grad: w * IFFT(dz U_i)
        ck(dns_grad_z(g, d->Us[0][i], d->tmp0, d->beta, st), "gradz");
        transform(d, d->tmp0, STX_INVERSE);
        a.Tc = d->tmp0;
      }
      if (z3 && form != 1) {  // div(uu): IFFT(dz FFT(u_i w))
        ck(dns_product(g, d->Up[i], d->Up[2], d->tmp2, st), "product");
        transform(d, d->tmp2, STX_FORWARD);
        ck(dns_grad_z(g, d->tmp2, d->tmp1, d->beta, st), "gradz");  // not in place
        transform(d, d->tmp1, STX_INVERSE);
        a.Tk = d->tmp1;
      }
      ck(dns_nonlinear(g, a, st), "nonlinear");
    }
    force_physical(d, i, N, d->Up);
    transform(d, N, STX_FORWARD);
    force_fourier(d, i, N);
    ck(dns_smooth(g, Nm, N, d->dsswork, st), "smooth");
  }
  if (d->form == 1) d->toggle = 1 - d->toggle;
}

// rollv (src/sem.h:98-106): the last level moves to the front.
void rollm_levels(std::vector<double*>& v) {
  if (v.size() < 2) return;
  std::rotate(v.rbegin(), v.rbegin() + 1, v.rend());
}

template <class T>
void rollm(std::vector<std::vector<T>>& u) {
  if (u.size() < 2) return;
  std::vector<T> last = u.back();
  for (size_t i = u.size() - 1; i; --i) u[i] = u[i - 1];
  u[0] = last;
}

void solve(stx_dns* d, int idx, double* forcing, stx_modal* sys) {
  std::vector<int> it(d->ctx->M.nz);
  int rc = stx_field_solve(sys, forcing, d->u[idx], d->tol, d->step_max, it.data());
  if (rc == STX_ENOCONV) rc = STX_OK;  // the reference warns and carries on
  ckstx(rc);
  if (sys->method == STX_JACPCG) d->last_iters = it;
}

// BCmgr::maintainFourier + Pressure->evaluateBoundaries (dns/integrate.cpp:
// 153-156) for the high-order pressure edges, from Us[0] and Uf[0].
void hopbc(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const int Je = std::min(d->step - 1, d->nord), Jx = std::min(d->step, d->nord);
  rollm_levels(d->hop_lvl);
  HopbcArgs a{};
  a.U = d->Us[0][0];
  a.V = d->Us[0][1];
  a.W = d->ndim == 3 ? d->Us[0][2] : nullptr;
  a.Nx = d->Uf[0][0];
  a.Ny = d->Uf[0][1];
  a.nh = d->nh;
  a.elmt = d->h_elmt;
  a.side = d->h_side;
  a.line = d->h_line;
  a.nx = d->h_nx;
  a.ny = d->h_ny;
  for (int q = 0; q < Je; ++q) a.un_old[q] = d->un_lvl[q];
  a.un_new = d->un_lvl[d->nord - 1];
  a.hop_new = d->hop_lvl[0];
  for (int q = 0; q + 1 < Jx; ++q) a.hop_old[q] = d->hop_lvl[q + 1];
  const FieldDev& P = ctx->fields.at(d->names[d->ncom]);
  a.lines = P.d_lines;
  a.nline = P.nline;
  a.Je = Je;
  for (int q = 0; q <= Je; ++q) a.alpha[q] = kSS[Je][q];
  a.invdt = 1.0 / d->dt;
  a.nu = d->nu;
  a.beta = d->beta;
  a.Jx = Jx;
  for (int q = 0; q < Jx; ++q) a.ex[q] = kEX[Jx][q];
  ck(dns_hopbc(ctx->dg, a, ctx->stream), "hopbc");
  rollm_levels(d->un_lvl);
}

// Computed outflow BCs: BCmgr::maintainFourier's gradient terms (newest
// level from Us[0]) and the essential pressure of the outflow edges
// (evaluateCEBCp), written into the pressure's BC lines.
void outflow_pressure(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  rollm_levels(d->o_divu);
  rollm_levels(d->o_gradu);
  ck(outflow_fourier(g, d->oe, d->Us[0][0], d->Us[0][1], d->ncom > 2 ? d->Us[0][2] : nullptr, d->nu, d->beta,
                     d->o_divu[0], d->o_gradu[0], st),
     "outflow gradients");
  const int Jx = std::min(d->step, d->nord);
  ck(outflow_energy(g, d->oe, d->o_uvw.data(), kEX[Jx], Jx, d->o_iuzd, d->o_fb, st), "outflow energy");
  if (g.nz > 2)
    ck(z_transform(d->o_fb, g.nz, d->oe.ostride, STX_FORWARD, ctx->d_twiddle, nullptr, st), "outflow transform");
  else if (g.nz == 2)
    ck(cudaMemsetAsync(d->o_fb + d->oe.ostride, 0, sizeof(double) * d->oe.ostride, st), "outflow nyquist");
  const FieldDev& P = ctx->fields.at(d->names[d->ncom]);
  ck(outflow_plines(g, d->oe, d->o_gradu.data(), kEX[Jx], Jx, d->o_fb, P.d_lines, P.nline, st), "outflow p");
}

// Natural u, v values of the outflow edges from the new pressure
// (evaluateCNBCu), written into their BC lines.
void outflow_velocity(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const int Jx = std::min(d->step, d->nord);
  for (int i = 0; i < 2 && i < d->ncom; ++i) {
    FieldDev& F = ctx->fields.at(d->names[i]);
    ck(outflow_ulines(ctx->dg, d->oe, d->o_divu.data(), kEX[Jx], Jx, d->o_fb, d->u[d->ncom], d->nu, i, F.d_lines,
                      F.nline, ctx->stream),
       "outflow velocity");
  }
}

void advance_one(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  nonlinear(d);
  d->step += 1;
  d->time += d->dt;
  const char pc = d->names[d->ncom];
  if (d->tdep[d->ncom]) ckstx(stx_field_bc_evaluate(ctx, pc, d->time));
  if (d->nh) hopbc(d);
  if (d->oe.no) outflow_pressure(d);
  // -- waveProp (dns/integrate.cpp:204-239)
  const int Je = std::min(d->step, d->nord);
  for (int i = 0; i < d->ncom; ++i) {
    CombineArgs a{};
    a.n = 0;
    for (int q = 0; q < Je; ++q) {
      a.c[a.n] = -kSS[Je][q + 1];
      a.p[a.n++] = d->Us[q][i];
      a.c[a.n] = kEX[Je][q] * d->dt;
      a.p[a.n++] = d->Uf[q][i];
    }
    a.out = d->u[i];
    ck(dns_combine(g, a, st), "waveProp");
  }
  for (int i = 0; i < d->ncom; ++i) std::swap(d->u[i], d->Us[0][i]);
  rollm(d->Uf);
  // -- setPForce: div u^ / dt (dns/integrate.cpp:242-257)
  ck(dns_divergence(g, d->Us[0][0], d->Us[0][1], d->ndim == 3 ? d->Us[0][2] : nullptr, d->Uf[0][0], d->dt,
                    d->beta, st),
     "setPForce");
  solve(d, d->ncom, d->Uf[0][0], d->psys);
  // -- project (dns/integrate.cpp:260-289)
  const double alpha = -1.0 / (d->dt * d->nu), bcoef = 1.0 / d->nu;
  for (int i = 0; i < d->ncom; ++i) {
    std::swap(d->Us[0][i], d->Uf[0][i]);
    ck(dns_project(g, d->Uf[0][i], d->u[d->ncom], i < d->ndim ? i : -1, alpha, bcoef, d->beta, st), "project");
  }
  for (int i = 0; i < d->ncom; ++i) copy(d, d->Us[0][i], d->u[i]);
  rollm(d->Us);
  // -- velocity BCs, viscous substep (dns/integrate.cpp:177-193, 328-356)
  for (int i = 0; i < d->ncom; ++i)
    if (d->tdep[i]) ckstx(stx_field_bc_evaluate(ctx, d->names[i], d->time));
  if (d->oe.no) outflow_velocity(d);
  // direct systems sharing their matrices: one skeleton solve for all
  // components (every matrix tile read once)
  bool shared = d->step >= d->nord && d->ncom <= 3 && !d->iterative;
  for (int i = 1; i < d->ncom; ++i) shared = shared && d->vsys[i]->store == d->vsys[0]->store;
  if (shared) {
    const double* F[3];
    double* U[3];
    for (int i = 0; i < d->ncom; ++i) {
      F[i] = d->Uf[0][i];
      U[i] = d->u[i];
    }
    ckstx(stx_field_solve_multi(d->vsys.data(), d->ncom, F, U));
    return;
  }
  for (int i = 0; i < d->ncom; ++i) {
    stx_modal* sys = d->vsys[i];
    if (d->step < d->nord) {
      const auto key = std::make_pair(d->names[i], Je);
      auto itp = d->pcg.find(key);
      if (itp == d->pcg.end()) {
        stx_modal* m = nullptr;
        const double lam = kSS[Je][0] / (d->dt * d->nu);
        ckstx(stx_modal_create(ctx, d->names[i], lam, d->beta, 0, (ctx->M.nz + 1) / 2, STX_JACPCG, &m));
        itp = d->pcg.emplace(key, m).first;
      }
      sys = itp->second;
    }
    solve(d, i, d->Uf[0][i], sys);
  }
}

}  // namespace

namespace stx {

void dns_advance_one(stx_dns* d) { advance_one(d); }

int dns_next_form(const stx_dns* d) { return next_form(d); }

int dns_error_code(const std::exception& e) {
  if (const auto* de = dynamic_cast<const DnsError*>(&e)) return de->code;
  return STX_ESESSION;
}

}  // namespace stx

namespace {

constexpr int kMaxCycle = 42;

// Buffers whose roles rotate from step to step (by pointer), in a fixed order.
std::vector<double*> pointer_state(const stx_dns* d) {
  std::vector<double*> k(d->u.begin(), d->u.end());
  for (const auto& v : d->Us) k.insert(k.end(), v.begin(), v.end());
  for (const auto& v : d->Uf) k.insert(k.end(), v.begin(), v.end());
  k.insert(k.end(), d->un_lvl.begin(), d->un_lvl.end());
  k.insert(k.end(), d->hop_lvl.begin(), d->hop_lvl.end());
  k.insert(k.end(), d->o_uvw.begin(), d->o_uvw.end());
  k.insert(k.end(), d->o_divu.begin(), d->o_divu.end());
  k.insert(k.end(), d->o_gradu.begin(), d->o_gradu.end());
  return k;
}

// A step is steady (its kernels and coefficients repeat) once the start-up
// orders are past, no BC is re-evaluated on the host, no forcing term
// changes with time and the velocity solves are direct (a Jacobi-PCG solve
// reads its iteration counts back).
bool steady(const stx_dns* d) {
  if (d->step < d->nord || d->force.tdep || d->iterative) return false;
  for (char t : d->tdep)
    if (t) return false;
  return true;
}

void drop_graph(stx_dns* d) {
  if (d->gexec) cudaGraphExecDestroy(d->gexec);
  d->gexec = nullptr;
  d->gperiod = 0;
  d->gkey.clear();
}

// Capture the steps from the current pointer state back to it (at most
// kMaxCycle: the velocity storage of N_TIME = 3 rotates through a 7-cycle,
// the alternating form through 2 and the pressure BC levels through 3).
// The host state moves on during the capture without the work running; on
// success the graph is launched once to run those steps, on failure the
// host state is put back and false returned.
bool capture_steps(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const auto u = d->u;
  const auto Us = d->Us, Uf = d->Uf;
  const auto un = d->un_lvl, hop = d->hop_lvl;
  const auto ouvw = d->o_uvw, odiv = d->o_divu, ogr = d->o_gradu;
  const int step = d->step, toggle = d->toggle;
  const double time = d->time;
  const std::vector<double*> key = pointer_state(d);
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
  int period = 0;
  bool ok = true;
  try {
    do {
      advance_one(d);
      ++period;
    } while (period < kMaxCycle && !(pointer_state(d) == key && d->toggle == toggle));
  } catch (const std::exception&) {
    ok = false;
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  ok = ok && e == cudaSuccess && graph && pointer_state(d) == key && d->toggle == toggle;
  cudaGraphExec_t exec = nullptr;
  if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // clear a capture error, the steps run directly instead
  if (!ok) {
    d->u = u;
    d->Us = Us;
    d->Uf = Uf;
    d->un_lvl = un;
    d->hop_lvl = hop;
    d->o_uvw = ouvw;
    d->o_divu = odiv;
    d->o_gradu = ogr;
    d->step = step;
    d->toggle = toggle;
    d->time = time;
    return false;
  }
  d->gexec = exec;
  d->gperiod = period;
  d->gkey = key;
  d->gtoggle = toggle;
  ck(cudaGraphLaunch(d->gexec, ctx->stream), "graph launch");
  ++d->graph_launches;
  return true;
}

}  // namespace

extern "C" {

int stx_dns_create(stx_context* ctx, int advection, stx_dns** out) {
  return dns_guarded([&] {
    if (!ctx || !out) throw DnsError(STX_EINVAL, "null argument");
    if (advection < 0 || advection > 3) throw DnsError(STX_EINVAL, "advection must be 0..3");
    *out = nullptr;
    auto d = new stx_dns();
    std::unique_ptr<stx_dns> guard(d);
    d->ctx = ctx;
    const Session& S = ctx->S;
    d->names = S.fields;
    if (d->names.size() < 3) throw DnsError(STX_ESESSION, "dns needs velocity fields and pressure");
    d->ncom = static_cast<int>(d->names.size()) - 1;
    d->ndim = ctx->M.nz > 1 ? 3 : 2;
    if (d->ndim == 3 && d->ncom != 3) throw DnsError(STX_ESESSION, "3D needs fields u v w p");
    d->nord = S.tokens.ivalue("N_TIME");
    if (d->nord < 1 || d->nord > 3) throw DnsError(STX_ESESSION, "N_TIME must be 1..3");
    d->dt = S.tokens.value("D_T");
    d->nu = S.tokens.value("KINVIS");
    d->beta = S.tokens.value("BETA");
    d->tol = S.tokens.value("TOL_REL");
    d->step_max = S.tokens.ivalue("STEP_MAX");
    d->form = advection;
    d->use_graph = !S.tokens.has("STX_DNS_GRAPH") || S.tokens.ivalue("STX_DNS_GRAPH") != 0;
    cudaSetDevice(ctx->device);
    const DevGeom& g = ctx->dg;
    d->fsize = static_cast<size_t>(g.nz) * g.plane_size;
    const int nfield = (d->ncom + 1) + 2 * d->nord * d->ncom + d->ncom + 3;
    double* base = static_cast<double*>(d->arena.alloc(sizeof(double) * d->fsize * nfield));
    ck(cudaMemset(base, 0, sizeof(double) * d->fsize * nfield), "memset");
    int k = 0;
    for (int i = 0; i <= d->ncom; ++i) d->u.push_back(base + d->fsize * k++);
    d->Us.assign(d->nord, {});
    d->Uf.assign(d->nord, {});
    for (int q = 0; q < d->nord; ++q)
      for (int i = 0; i < d->ncom; ++i) {
        d->Us[q].push_back(base + d->fsize * k++);
        d->Uf[q].push_back(base + d->fsize * k++);
      }
    for (int i = 0; i < d->ncom; ++i) d->Up.push_back(base + d->fsize * k++);
    d->tmp0 = base + d->fsize * k++;
    d->tmp1 = base + d->fsize * k++;
    d->tmp2 = base + d->fsize * k++;
    d->part = static_cast<double*>(
        d->arena.alloc(sizeof(double) * dns_analysis_blocks() * std::max((g.nz + 1) / 2, 3)));
    size_t ws = 0;
    for (char c : d->names) ws = std::max(ws, dns_smooth_workspace_doubles(g, ctx->fields.at(c).dn));
    d->dsswork = static_cast<double*>(d->arena.alloc(sizeof(double) * ws));
    for (char c : d->names) {
      bool td = false;
      for (const auto& E : ctx->fields.at(c).N.edges) td = td || depends_on_t(E.expr);
      d->tdep.push_back(td);
    }
    // -- running averages (Statistics::Statistics)
    d->avg_level = S.tokens.has("AVERAGE") ? S.tokens.ivalue("AVERAGE") : 0;
    if (d->avg_level < 0 || d->avg_level > 3) throw DnsError(STX_EINVAL, "AVERAGE token out of [0,3]");
    if (d->avg_level > 0) {
      std::string names = d->names;
      if (d->avg_level > 1)
        for (int i = 0; i < d->ncom * (d->ncom + 1) / 2; ++i) names.push_back(static_cast<char>('A' + i));
      if (d->avg_level > 2) {
        // energy-equation correlations (Statistics::Statistics,
        // src/statistics.cpp:128-175): q, d; p u_i (m n o); q u_i (r s t);
        // S_ij u_j (a b c); S_ij (G H I, J K L)
        names += d->ncom == 3 ? "qdmnortsabcGHIJKL" : "qdmnrsabGHI";
        // work fields: p and q in physical space, then the strain-rate
        // components and a gradient
        d->avg_work = static_cast<double*>(d->arena.alloc(sizeof(double) * d->fsize * 7));
      }
      std::sort(names.begin(), names.end());
      d->avg_names = names;
      double* ab = static_cast<double*>(d->arena.alloc(sizeof(double) * d->fsize * names.size()));
      ck(cudaMemset(ab, 0, sizeof(double) * d->fsize * names.size()), "memset");
      for (size_t k = 0; k < names.size(); ++k) d->avg_buf.push_back(ab + d->fsize * k);
    }
    // -- 3/2-rule products: padded buffers and the length-nz32 twiddles
    if (S.tokens.has("DEALIAS") && S.tokens.ivalue("DEALIAS") > 0 && g.nz > 2) {
      d->nz32 = 3 * g.nz / 2;
      const size_t n32 = static_cast<size_t>(d->nz32) * g.plane_size;
      double* pb = static_cast<double*>(d->arena.alloc(sizeof(double) * n32 * (d->ncom + 3)));
      for (int i = 0; i < d->ncom; ++i) d->Up32.push_back(pb + n32 * i);
      d->A32 = pb + n32 * d->ncom;
      d->B32 = d->A32 + n32;
      d->C32 = d->B32 + n32;
      std::vector<double> tw(2 * d->nz32);
      for (int m = 0; m < d->nz32; ++m) {
        tw[m] = std::cos(2.0 * M_PI * m / d->nz32);
        tw[d->nz32 + m] = std::sin(2.0 * M_PI * m / d->nz32);
      }
      d->twiddle32 = static_cast<double*>(d->arena.alloc(sizeof(double) * tw.size()));
      ck(cudaMemcpy(d->twiddle32, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice), "twiddle");
    }
    // -- body forcing (FieldForce::FieldForce)
    force_setup(d);
    // -- high-order pressure BC edges and storage (BCmgr::buildComputedBCs,
    //    src/bcmgr.cpp:937-996)
    {
      const FieldDev& P = ctx->fields.at(d->names[d->ncom]);
      std::vector<int> el, sd, ln;
      std::vector<double> nx, ny;
      for (size_t b = 0; b < P.N.edges.size(); ++b) {
        const BoundaryEdge& E = P.N.edges[b];
        if (E.kind != 'H') continue;
        el.push_back(E.elmt);
        sd.push_back(E.side);
        ln.push_back(static_cast<int>(b));
        nx.insert(nx.end(), E.nx.begin(), E.nx.end());
        ny.insert(ny.end(), E.ny.begin(), E.ny.end());
      }
      d->nh = static_cast<int>(el.size());
      if (d->nh) {
        auto up = [&](const auto& v) {
          using T = typename std::decay_t<decltype(v)>::value_type;
          T* p = static_cast<T*>(d->arena.alloc(sizeof(T) * v.size()));
          ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
          return p;
        };
        d->h_elmt = up(el);
        d->h_side = up(sd);
        d->h_line = up(ln);
        d->h_nx = up(nx);
        d->h_ny = up(ny);
        d->hsize = static_cast<size_t>(g.nz) * d->nh * g.np;
        double* hb = static_cast<double*>(d->arena.alloc(sizeof(double) * d->hsize * 2 * d->nord));
        ck(cudaMemset(hb, 0, sizeof(double) * d->hsize * 2 * d->nord), "memset");
        for (int q = 0; q < d->nord; ++q) {
          d->un_lvl.push_back(hb + d->hsize * q);
          d->hop_lvl.push_back(hb + d->hsize * (d->nord + q));
        }
      }
    }
    // -- edges of the boundary group "wall" (the group string compared as
    //    Edge::normTraction does, src/edge.cpp:259-289), for the forces and
    //    tractions, in the order of the SURFACES section (BCmgr::buildsurf,
    //    src/bcmgr.cpp:827-870: the order of the tractions in session.wss)
    {
      const FieldDev& U = ctx->fields.at(d->names[0]);
      std::map<std::pair<int, int>, const BoundaryEdge*> by_side;
      for (const BoundaryEdge& E : U.N.edges) by_side[{E.elmt, E.side}] = &E;
      std::vector<int> el, nd;
      std::vector<double> nx, ny, area;
      std::vector<int> idx(g.np);
      for (const Surface& sf : S.surfaces) {
        if (sf.kind != 'B') continue;
        const auto gi = S.groups.find(sf.group);
        const auto be = by_side.find({sf.elmt, sf.side});
        if (gi == S.groups.end() || gi->second != "wall" || be == by_side.end()) continue;
        const BoundaryEdge& E = *be->second;
        el.push_back(E.elmt);
        ctx->M.side_nodes(E.side, idx.data());
        nd.insert(nd.end(), idx.begin(), idx.end());
        nx.insert(nx.end(), E.nx.begin(), E.nx.end());
        ny.insert(ny.end(), E.ny.begin(), E.ny.end());
        area.insert(area.end(), E.area.begin(), E.area.end());
      }
      d->nwall = static_cast<int>(el.size());
      if (d->nwall) {
        auto up = [&](const auto& v) {
          using T = typename std::decay_t<decltype(v)>::value_type;
          T* p = static_cast<T*>(d->arena.alloc(sizeof(T) * v.size()));
          ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
          return p;
        };
        d->w_elmt = up(el);
        d->w_node = up(nd);
        d->w_nx = up(nx);
        d->w_ny = up(ny);
        d->w_area = up(area);
        d->w_out = static_cast<double*>(d->arena.alloc(sizeof(double) * 5 * d->nwall));
        // tractions: nz planes of the three components' wall lines, padded
        // to an even length (DNSAnalyser::DNSAnalyser, dns/dnsanalysis.cpp:55-72)
        const int nline = g.np * d->nwall;
        d->w_npad = 3 * nline + (3 * nline) % 2;
        d->w_buf = static_cast<double*>(d->arena.alloc(sizeof(double) * d->w_npad * g.nz));
      }
    }
    // -- computed outflow edges and storage (BCmgr::buildComputedBCs,
    //    src/bcmgr.cpp:937-996): the pressure's 'O' edges, which u and v
    //    carry at the same positions of their BC lines
    {
      const FieldDev& P = ctx->fields.at(d->names[d->ncom]);
      std::vector<int> el, sd, ln;
      std::vector<double> nx, ny;
      for (size_t b = 0; b < P.N.edges.size(); ++b) {
        const BoundaryEdge& E = P.N.edges[b];
        if (E.kind != 'O') continue;
        for (int i = 0; i < 2; ++i) {
          const auto& V = ctx->fields.at(d->names[i]).N.edges;
          if (b >= V.size() || V[b].elmt != E.elmt || V[b].side != E.side)
            throw DnsError(STX_EUNSUPPORTED, "outflow edges differ between the velocity and pressure BC lines");
        }
        el.push_back(E.elmt);
        sd.push_back(E.side);
        ln.push_back(static_cast<int>(b));
        nx.insert(nx.end(), E.nx.begin(), E.nx.end());
        ny.insert(ny.end(), E.ny.begin(), E.ny.end());
      }
      if (!el.empty()) {
        if (d->nz32) throw DnsError(STX_EUNSUPPORTED, "computed outflow BCs with DEALIAS");
        auto up = [&](const auto& v) {
          using T = typename std::decay_t<decltype(v)>::value_type;
          T* p = static_cast<T*>(d->arena.alloc(sizeof(T) * v.size()));
          ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
          return p;
        };
        OutflowEdges& O = d->oe;
        O.no = static_cast<int>(el.size());
        O.ostride = (O.no * g.np + 1) / 2 * 2;
        O.elmt = up(el);
        O.side = up(sd);
        O.line = up(ln);
        O.nx = up(nx);
        O.ny = up(ny);
        const size_t lvl = static_cast<size_t>(g.nz) * O.ostride;
        const size_t total = lvl * (3 * d->nord + 2 * d->nord + 1);
        double* ob = static_cast<double*>(d->arena.alloc(sizeof(double) * total));
        ck(cudaMemset(ob, 0, sizeof(double) * total), "memset");
        for (int q = 0; q < d->nord; ++q) {
          d->o_uvw.push_back(ob + 3 * lvl * q);
          d->o_divu.push_back(ob + 3 * lvl * d->nord + lvl * q);
          d->o_gradu.push_back(ob + 4 * lvl * d->nord + lvl * q);
        }
        d->o_fb = ob + 5 * lvl * d->nord;
        const TokenTable& T = S.tokens;
        d->o_iuzd = 1.0 / (T.has("U0Delta") ? T.value("U0Delta") : 0.0);
      }
    }
    // -- preSolve (dns/integrate.cpp:292-325): ITERATIVE = 1 selects
    //    Jacobi-PCG velocity systems; the pressure system is always direct.
    //    Token STX_DNS_MIXED = 1 gives the steady velocity systems the
    //    mixed-precision form (FP32 skeleton inverses, FP64 refinement); the
    //    pressure system stays FP64 (its mode 0 is singular)
    const double lam = kSS[d->nord][0] / (d->dt * d->nu);
    const int nmodes = (ctx->M.nz + 1) / 2;
    d->iterative = S.tokens.ivalue("ITERATIVE") != 0;
    d->mixed = !d->iterative && S.tokens.has("STX_DNS_MIXED") && S.tokens.ivalue("STX_DNS_MIXED") != 0;
    for (int i = 0; i < d->ncom; ++i) {
      stx_modal* m = nullptr;
      ckstx(stx_modal_create(ctx, d->names[i], lam, d->beta, 0, nmodes,
                             d->iterative ? STX_JACPCG : d->mixed ? STX_MIXED : STX_DIRECT, &m));
      d->vsys.push_back(m);
    }
    ckstx(stx_modal_create(ctx, d->names[d->ncom], 0.0, d->beta, 0, nmodes, STX_DIRECT, &d->psys));
    *out = guard.release();
  });
}

int stx_dns_destroy(stx_dns* d) {
  return dns_guarded([&] {
    if (!d) return;
    cudaSetDevice(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
    drop_graph(d);
    for (auto* m : d->vsys) stx_modal_destroy(m);
    if (d->psys) stx_modal_destroy(d->psys);
    for (auto& kv : d->pcg) stx_modal_destroy(kv.second);
    if (d->probe_buf) cudaFree(d->probe_buf);
    delete d;
  });
}

int stx_dns_restart(stx_dns* d, double t0) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    cudaSetDevice(d->ctx->device);
    for (int q = 0; q < d->nord; ++q)
      for (int i = 0; i < d->ncom; ++i) {
        ck(cudaMemsetAsync(d->Us[q][i], 0, sizeof(double) * d->fsize, d->ctx->stream), "zero");
        ck(cudaMemsetAsync(d->Uf[q][i], 0, sizeof(double) * d->fsize, d->ctx->stream), "zero");
      }
    for (double* p : d->un_lvl) ck(cudaMemsetAsync(p, 0, sizeof(double) * d->hsize, d->ctx->stream), "zero");
    for (double* p : d->hop_lvl) ck(cudaMemsetAsync(p, 0, sizeof(double) * d->hsize, d->ctx->stream), "zero");
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    drop_graph(d);
    d->eager_steady = 0;
    d->step = 0;
    d->time = t0;
    d->force.sfd_started = false;  // SFD's filtered field restarts from u
    for (char c : d->names) ckstx(stx_field_bc_evaluate(d->ctx, c, t0));
  });
}

int stx_dns_set_field(stx_dns* d, char field, const double* h_phys) {
  return dns_guarded([&] {
    if (!d || !h_phys) throw DnsError(STX_EINVAL, "null argument");
    const size_t idx = d->names.find(field);
    if (idx == std::string::npos) throw DnsError(STX_EINVAL, std::string("no field ") + field);
    const Mesh& M = d->ctx->M;
    cudaSetDevice(d->ctx->device);
    double* f = d->u[idx];
    ck(cudaMemsetAsync(f, 0, sizeof(double) * d->fsize, d->ctx->stream), "zero");
    ck(cudaMemcpy2DAsync(f, sizeof(double) * M.plane_size, h_phys, sizeof(double) * M.nplane,
                         sizeof(double) * M.nplane, M.nz, cudaMemcpyHostToDevice, d->ctx->stream),
       "upload");
    transform(d, f, STX_FORWARD);
    if (M.nz > 1) ck(cudaMemsetAsync(f + M.plane_size, 0, sizeof(double) * M.plane_size, d->ctx->stream), "nyq");
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_get_field(stx_dns* d, char field, double* h_phys) {
  return dns_guarded([&] {
    if (!d || !h_phys) throw DnsError(STX_EINVAL, "null argument");
    const size_t idx = d->names.find(field);
    if (idx == std::string::npos) throw DnsError(STX_EINVAL, std::string("no field ") + field);
    const Mesh& M = d->ctx->M;
    cudaSetDevice(d->ctx->device);
    copy(d, d->tmp0, d->u[idx]);
    if (M.nz > 1) ck(cudaMemsetAsync(d->tmp0 + M.plane_size, 0, sizeof(double) * M.plane_size, d->ctx->stream), "nyq");
    transform(d, d->tmp0, STX_INVERSE);
    ck(cudaMemcpy2DAsync(h_phys, sizeof(double) * M.nplane, d->tmp0, sizeof(double) * M.plane_size,
                         sizeof(double) * M.nplane, M.nz, cudaMemcpyDeviceToHost, d->ctx->stream),
       "download");
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}


int stx_dns_advance(stx_dns* d, int nsteps) {
  return dns_guarded([&] {
    if (!d || nsteps < 0) throw DnsError(STX_EINVAL, "bad argument");
    cudaSetDevice(d->ctx->device);
    int left = nsteps;
    while (left > 0) {
      const bool st = steady(d);
      if (d->use_graph && st && d->eager_steady > 0) {
        if (d->gexec && pointer_state(d) == d->gkey && d->toggle == d->gtoggle && left >= d->gperiod) {
          ck(cudaGraphLaunch(d->gexec, d->ctx->stream), "graph launch");
          ++d->graph_launches;
          d->step += d->gperiod;
          for (int k = 0; k < d->gperiod; ++k) d->time += d->dt;
          left -= d->gperiod;
          continue;
        }
        if (!d->gexec && left >= kMaxCycle) {  // never run past nsteps
          if (capture_steps(d)) {
            left -= d->gperiod;
            continue;
          }
          d->use_graph = false;  // not capturable here: run every step directly
        }
      }
      advance_one(d);
      if (st) ++d->eager_steady;
      --left;
    }
    ck(cudaGetLastError(), "advance");
  });
}

int stx_dns_state(const stx_dns* d, int* step, double* time) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    if (step) *step = d->step;
    if (time) *time = d->time;
  });
}

namespace {

// Q4-weighted energies of every mode of Fourier field f, summed in order.
std::vector<double> mode_energies(stx_dns* d, const double* f) {
  stx_context* ctx = d->ctx;
  const int nb = dns_analysis_blocks(), nm = (ctx->M.nz + 1) / 2;
  double* part = d->part;
  ck(dns_mode_energy_partials(ctx->dg, f, part, ctx->stream), "mode energy");
  std::vector<double> h(static_cast<size_t>(nb) * nm), out(nm, 0.0);
  ck(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream), "download");
  ck(cudaStreamSynchronize(ctx->stream), "sync");
  for (int m = 0; m < nm; ++m)
    for (int b = 0; b < nb; ++b) out[m] += h[static_cast<size_t>(m) * nb + b];
  return out;
}

double mesh_area(const stx_context* ctx) {
  double a = 0.0;
  for (double q : ctx->M.Q4) a += q;
  return a;
}

}  // namespace

int stx_dns_modal_energy(stx_dns* d, double* h_ek) {
  return dns_guarded([&] {
    if (!d || !h_ek) throw DnsError(STX_EINVAL, "null argument");
    cudaSetDevice(d->ctx->device);
    const int nm = (d->ctx->M.nz + 1) / 2;
    const double area = mesh_area(d->ctx);
    for (int m = 0; m < nm; ++m) h_ek[m] = 0.0;
    for (int i = 0; i < d->ndim; ++i) {
      const std::vector<double> e = mode_energies(d, d->u[i]);
      for (int m = 0; m < nm; ++m) h_ek[m] += e[m] / (2.0 * area);
    }
  });
}

int stx_dns_divergence_energy(stx_dns* d, double* value) {
  return dns_guarded([&] {
    if (!d || !value) throw DnsError(STX_EINVAL, "null argument");
    stx_context* ctx = d->ctx;
    cudaSetDevice(ctx->device);
    ck(dns_divergence(ctx->dg, d->u[0], d->u[1], d->ndim == 3 ? d->u[2] : nullptr, d->tmp1, 1.0, d->beta,
                      ctx->stream),
       "divergence");
    const std::vector<double> e = mode_energies(d, d->tmp1);
    const double area = mesh_area(ctx);
    double L2 = 0.0;
    for (double v : e) L2 += v / (2.0 * area);
    *value = L2 / (2.0 * M_PI / d->beta);
  });
}

int stx_dns_cfl(stx_dns* d, double* inv_dt) {
  return dns_guarded([&] {
    if (!d || !inv_dt) throw DnsError(STX_EINVAL, "null argument");
    stx_context* ctx = d->ctx;
    cudaSetDevice(ctx->device);
    const int nb = dns_analysis_blocks();
    const double dxy = ctx->M.q.z[1] - ctx->M.q.z[0];
    const int ndir = d->ncom == 3 ? 3 : 2;
    std::vector<double> h(static_cast<size_t>(nb) * ndir);
    for (int dir = 0; dir < ndir; ++dir)
      ck(dns_cfl_partials(ctx->dg, d->u[dir], dir, dxy, d->part + static_cast<size_t>(nb) * dir, ctx->stream),
         "cfl");
    ck(cudaMemcpyAsync(h.data(), d->part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream),
       "download");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    double c = 0.0;
    for (int dir = 0; dir < ndir; ++dir) {
      double m = 0.0;
      for (int b = 0; b < nb; ++b) m = std::max(m, h[static_cast<size_t>(nb) * dir + b]);
      if (dir == 2) m /= 2.0 * M_PI / d->beta / ctx->M.nz;
      c = std::max(c, m);
    }
    *inv_dt = c;
  });
}

int stx_dns_probe(stx_dns* d, int npts, const int* elmt, const double* rs, const double* z, double* out) {
  return dns_guarded([&] {
    if (!d || npts < 0 || (npts > 0 && (!elmt || !rs || !out))) throw DnsError(STX_EINVAL, "null argument");
    if (npts == 0) return;
    stx_context* ctx = d->ctx;
    const Mesh& M = ctx->M;
    cudaSetDevice(ctx->device);
    const int np = M.np, nf = static_cast<int>(d->names.size());
    // 2D (fewer than 3 planes): plane 0 alone (src/auxfield.cpp:1668-1669)
    const int nzc = M.nz < 3 ? 1 : M.nz;
    const int stride = 2 * np + nzc;
    std::vector<double> w(static_cast<size_t>(npts) * stride);
    for (int p = 0; p < npts; ++p) {
      if (elmt[p] < 0 || elmt[p] >= M.nel) throw DnsError(STX_EINVAL, "history point element out of range");
      double* wp = w.data() + static_cast<size_t>(p) * stride;
      gll_interpolants(M.q, rs[2 * p + 1], wp, nullptr);
      gll_interpolants(M.q, rs[2 * p], wp + np, nullptr);
      double* c = wp + 2 * np;
      c[0] = 1.0;
      if (nzc > 1) {
        // the Fourier series at z of the packed half spectrum, non-zero
        // modes doubled (src/auxfield.cpp:1681-1695)
        const double bz = (z ? z[p] : 0.0) * d->beta;
        c[1] = std::cos((M.nz / 2) * bz);
        for (int k = 1; k < M.nz / 2; ++k) {
          c[2 * k] = 2.0 * std::cos(k * bz);
          c[2 * k + 1] = -2.0 * std::sin(k * bz);
        }
      }
    }
    const size_t wbytes = sizeof(double) * w.size(), ebytes = (sizeof(int) * npts + 15) / 16 * 16;
    const size_t obytes = sizeof(double) * static_cast<size_t>(npts) * nf;
    const size_t need = wbytes + ebytes + obytes;
    if (need > d->probe_bytes) {
      ck(cudaStreamSynchronize(ctx->stream), "sync");
      if (d->probe_buf) cudaFree(d->probe_buf);
      d->probe_buf = nullptr;
      d->probe_bytes = 0;
      ck(cudaMalloc(&d->probe_buf, need), "history point scratch");
      d->probe_bytes = need;
    }
    char* base = static_cast<char*>(d->probe_buf);
    ProbeArgs a{};
    a.npts = npts;
    a.nf = nf;
    a.nzc = nzc;
    a.w = reinterpret_cast<double*>(base);
    a.elmt = reinterpret_cast<int*>(base + wbytes);
    a.out = reinterpret_cast<double*>(base + wbytes + ebytes);
    for (int f = 0; f < nf; ++f) a.f[f] = d->u[f];
    ck(cudaMemcpyAsync(base, w.data(), wbytes, cudaMemcpyHostToDevice, ctx->stream), "upload");
    ck(cudaMemcpyAsync(base + wbytes, elmt, sizeof(int) * npts, cudaMemcpyHostToDevice, ctx->stream), "upload");
    ck(dns_probe(ctx->dg, a, ctx->stream), "probe");
    ck(cudaMemcpyAsync(out, a.out, obytes, cudaMemcpyDeviceToHost, ctx->stream), "download");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
  });
}

int stx_dns_wall_forces(stx_dns* d, double* pressure, double* viscous) {
  return dns_guarded([&] {
    if (!d || !pressure || !viscous) throw DnsError(STX_EINVAL, "null argument");
    stx_context* ctx = d->ctx;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < 3; ++i) pressure[i] = viscous[i] = 0.0;
    if (!d->nwall) return;
    // DNSAnalyser::analyse (dns/dnsanalysis.cpp:97-113) takes field DIM as
    // the pressure and field 2 as w in 3D only: with N_Z = 1 and fields
    // "uvwp" the third field (w) stands in the pressure's place there too
    WallArgs a{};
    a.nw = d->nwall;
    a.elmt = d->w_elmt;
    a.node = d->w_node;
    a.nx = d->w_nx;
    a.ny = d->w_ny;
    a.area = d->w_area;
    a.p = d->u[d->ndim];
    a.u = d->u[0];
    a.v = d->u[1];
    a.w = d->ndim == 3 ? d->u[2] : nullptr;
    a.out = d->w_out;
    std::vector<double> h(static_cast<size_t>(5) * d->nwall);
    ck(dns_wall_forces(ctx->dg, a, ctx->stream), "wall forces");
    ck(cudaMemcpyAsync(h.data(), d->w_out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream),
       "download");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    const double mu = ctx->S.tokens.value("RHO") * d->nu;
    for (int b = 0; b < d->nwall; ++b) {  // per edge, in order (Field::normTraction / tangTraction)
      const double* e = h.data() + 5 * b;
      pressure[0] += e[0];
      pressure[1] += e[1];
      viscous[0] -= mu * e[2];
      viscous[1] -= mu * e[3];
      if (d->ndim == 3) viscous[2] -= mu * e[4];
    }
  });
}

int stx_dns_wall_traction(stx_dns* d, int* nline, double* h_out) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    stx_context* ctx = d->ctx;
    const Mesh& M = ctx->M;
    const int nl = M.np * d->nwall;
    if (nline) *nline = nl;
    if (!h_out || !d->nwall) return;
    cudaSetDevice(ctx->device);
    TractionArgs a{};
    a.nw = d->nwall;
    a.nline = nl;
    a.npad = d->w_npad;
    a.nz = M.nz;
    a.elmt = d->w_elmt;
    a.node = d->w_node;
    a.nx = d->w_nx;
    a.ny = d->w_ny;
    // Field::traction's fields (dns/dnsanalysis.cpp:145-150): the pressure,
    // u, v, and w when the session has three velocity components
    a.p = d->u[d->ncom];
    a.u = d->u[0];
    a.v = d->u[1];
    a.w = d->ncom == 3 ? d->u[2] : nullptr;
    a.mu = ctx->S.tokens.value("RHO") * d->nu;
    a.beta = d->beta;
    a.out = d->w_buf;
    ck(cudaMemsetAsync(d->w_buf, 0, sizeof(double) * d->w_npad * M.nz, ctx->stream), "zero");
    ck(dns_wall_traction(ctx->dg, a, ctx->stream), "wall traction");
    // to physical space along z (Femlib::DFTr inverse, as Field::bTransform)
    ck(z_transform(d->w_buf, M.nz, d->w_npad, STX_INVERSE, ctx->d_twiddle, nullptr, ctx->stream), "transform");
    for (int c = 0; c < 3; ++c)
      ck(cudaMemcpy2DAsync(h_out + static_cast<size_t>(c) * M.nz * nl, sizeof(double) * nl, d->w_buf + c * nl,
                           sizeof(double) * d->w_npad, sizeof(double) * nl, M.nz, cudaMemcpyDeviceToHost,
                           ctx->stream),
         "download");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
  });
}

int stx_dns_status(stx_dns* d, int* status) {
  return dns_guarded([&] {
    if (!d || !status) throw DnsError(STX_EINVAL, "null argument");
    *status = 0;
    std::vector<stx_modal*> all(d->vsys.begin(), d->vsys.end());
    all.push_back(d->psys);
    for (auto& kv : d->pcg) all.push_back(kv.second);
    for (stx_modal* m : all) {
      int v = 0;
      ckstx(stx_modal_status(m, &v));
      if (v && !*status) *status = v;
    }
  });
}

namespace {

void combine2(stx_dns* d, double* out, double a, const double* x, double b, const double* y) {
  CombineArgs c{};
  c.n = 0;
  c.c[c.n] = a;
  c.p[c.n++] = x;
  if (y) {
    c.c[c.n] = b;
    c.p[c.n++] = y;
  }
  c.out = out;
  ck(dns_combine(d->ctx->dg, c, d->ctx->stream), "combine");
}

double* avg_buffer(stx_dns* d, char name) {
  const size_t k = d->avg_names.find(name);
  if (k == std::string::npos) throw DnsError(STX_EINVAL, std::string("no average ") + name);
  return d->avg_buf[k];
}

// The energy-equation correlations of AVERAGE 3 (Statistics::update,
// src/statistics.cpp:247-391, Cartesian): with the velocities in physical
// space in Up, add p u_i, q = |u|^2 / 2, q u_i, the rate-of-strain tensor
// S_ij = (du_i/dx_j + du_j/dx_i) / 2 (gradients of the Fourier fields,
// then to physical space), S_ij u_j and S_ij S_ij to the averages.
void stats_energy(stx_dns* d) {
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  const int nv = d->ncom;
  double* W[7];
  for (int k = 0; k < 7; ++k) W[k] = d->avg_work + d->fsize * k;
  auto add_product = [&](char name, const double* a, const double* b) {
    ck(dns_product(g, a, b, d->tmp0, st), "product");
    double* avg = avg_buffer(d, name);
    combine2(d, avg, 1.0, avg, 1.0, d->tmp0);
  };
  auto add_field = [&](char name, const double* f) {
    double* avg = avg_buffer(d, name);
    combine2(d, avg, 1.0, avg, 1.0, f);
  };
  // -- pressure--velocity terms
  double* P = W[0];
  copy(d, P, d->u[d->ncom]);
  transform(d, P, STX_INVERSE);
  const char pu[3] = {'m', 'n', 'o'}, qu[3] = {'r', 's', 't'};
  for (int i = 0; i < nv; ++i) add_product(pu[i], P, d->Up[i]);
  // -- q and q u_i
  double* Q = W[1];
  ck(dns_product(g, d->Up[0], d->Up[0], Q, st), "product");
  for (int i = 1; i < nv; ++i) {
    ck(dns_product(g, d->Up[i], d->Up[i], d->tmp0, st), "product");
    combine2(d, Q, 1.0, Q, 1.0, d->tmp0);
  }
  combine2(d, Q, 0.5, Q, 0.0, nullptr);
  add_field('q', Q);
  for (int i = 0; i < nv; ++i) add_product(qu[i], d->Up[i], Q);
  // -- rate of strain: off-diagonal k = i + j - 1 (xy, xz, yz), diagonal
  double* Sd[3] = {W[0], W[1], W[2]};
  double* So[3] = {W[3], W[4], W[5]};
  double* T = W[6];
  auto grad = [&](int i, int j, double* out) {
    if (j < 2) ck(dns_grad_xy(g, d->u[i], out, j, st), "gradient");
    else ck(dns_grad_z(g, d->u[i], out, d->beta, st), "gradient");
  };
  for (int i = 0; i < nv; ++i)
    for (int j = 0; j < nv; ++j) {
      if (j == i) continue;
      const int k = i + j - 1;
      if (j > i) {
        grad(i, j, So[k]);
      } else {
        grad(i, j, T);
        combine2(d, So[k], 1.0, So[k], 1.0, T);
      }
    }
  const int noff = nv * (nv - 1) / 2;
  for (int k = 0; k < noff; ++k) combine2(d, So[k], 0.5, So[k], 0.0, nullptr);
  for (int i = 0; i < nv; ++i) grad(i, i, Sd[i]);
  for (int i = 0; i < nv; ++i) transform(d, Sd[i], STX_INVERSE);
  for (int k = 0; k < noff; ++k) transform(d, So[k], STX_INVERSE);
  add_field('G', Sd[0]);
  add_field('H', So[0]);
  add_field('I', Sd[1]);
  if (nv == 3) {
    add_field('J', So[1]);
    add_field('K', So[2]);
    add_field('L', Sd[2]);
  }
  // -- S_ij u_j
  add_product('a', Sd[0], d->Up[0]);
  add_product('a', So[0], d->Up[1]);
  if (nv == 3) add_product('a', So[1], d->Up[2]);
  add_product('b', So[0], d->Up[0]);
  add_product('b', Sd[1], d->Up[1]);
  if (nv == 3) add_product('b', So[2], d->Up[2]);
  if (nv == 3) {
    add_product('c', So[1], d->Up[0]);
    add_product('c', So[2], d->Up[1]);
    add_product('c', Sd[2], d->Up[2]);
  }
  // -- S_ij S_ij, the off-diagonal terms twice (scaled by sqrt 2)
  for (int k = 0; k < noff; ++k) combine2(d, So[k], std::sqrt(2.0), So[k], 0.0, nullptr);
  add_product('d', Sd[0], Sd[0]);
  add_product('d', So[0], So[0]);
  add_product('d', Sd[1], Sd[1]);
  if (nv == 3) {
    add_product('d', So[1], So[1]);
    add_product('d', So[2], So[2]);
    add_product('d', Sd[2], Sd[2]);
  }
}

}  // namespace

int stx_dns_stats_update(stx_dns* d) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    if (!d->avg_level) throw DnsError(STX_EINVAL, "no averaging (token AVERAGE)");
    stx_context* ctx = d->ctx;
    cudaSetDevice(ctx->device);
    const double n = d->navg;
    // Statistics::update (src/statistics.cpp:206-405): weight the old
    // averages, add the raw fields and the velocity products, smooth,
    // normalise.
    for (double* b : d->avg_buf) combine2(d, b, n, b, 0.0, nullptr);
    for (size_t i = 0; i < d->names.size(); ++i) {
      double* b = avg_buffer(d, d->names[i]);
      combine2(d, b, 1.0, b, 1.0, d->u[i]);
    }
    if (d->avg_level > 1) {
      for (int i = 0; i < d->ncom; ++i) {
        copy(d, d->Up[i], d->u[i]);
        transform(d, d->Up[i], STX_INVERSE);
      }
      const int pi[6] = {0, 0, 1, 0, 1, 2}, pj[6] = {0, 1, 1, 2, 2, 2};
      for (int k = 0; k < d->ncom * (d->ncom + 1) / 2; ++k) {
        ck(dns_product(ctx->dg, d->Up[pi[k]], d->Up[pj[k]], d->tmp0, ctx->stream), "product");
        double* b = avg_buffer(d, static_cast<char>('A' + k));
        combine2(d, b, 1.0, b, 1.0, d->tmp0);
      }
    }
    if (d->avg_level > 2) stats_energy(d);
    const DevNumbering& Nm = ctx->fields.at(d->names[0]).dn;
    for (double* b : d->avg_buf) {
      ck(dns_smooth(ctx->dg, Nm, b, d->dsswork, ctx->stream), "smooth");
      combine2(d, b, 1.0 / (n + 1.0), b, 0.0, nullptr);
    }
    ++d->navg;
    ck(cudaGetLastError(), "stats");
  });
}

int stx_dns_stats_swap(stx_dns* d) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    if (!d->avg_level) throw DnsError(STX_EINVAL, "no averaging (token AVERAGE)");
    if (d->avg_alt.empty()) {
      const size_t nb = d->avg_buf.size();
      double* ab = static_cast<double*>(d->arena.alloc(sizeof(double) * d->fsize * nb));
      cudaSetDevice(d->ctx->device);
      ck(cudaMemset(ab, 0, sizeof(double) * d->fsize * nb), "memset");
      for (size_t k = 0; k < nb; ++k) d->avg_alt.push_back(ab + d->fsize * k);
      d->navg_alt = 0;
    }
    std::swap(d->avg_buf, d->avg_alt);
    std::swap(d->navg, d->navg_alt);
  });
}

int stx_dns_stats_info(stx_dns* d, char* names, int len, int* navg, int set_navg) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    if (set_navg >= 0) d->navg = set_navg;
    if (navg) *navg = d->navg;
    if (names) {
      if (len < static_cast<int>(d->avg_names.size()) + 1) throw DnsError(STX_EINVAL, "name buffer too short");
      std::memcpy(names, d->avg_names.c_str(), d->avg_names.size() + 1);
    }
  });
}

int stx_dns_stats_get(stx_dns* d, char name, double* h_phys) {
  return dns_guarded([&] {
    if (!d || !h_phys) throw DnsError(STX_EINVAL, "null argument");
    const Mesh& M = d->ctx->M;
    cudaSetDevice(d->ctx->device);
    double* b = avg_buffer(d, name);
    copy(d, d->tmp0, b);
    if (d->names.find(name) != std::string::npos) {  // raw averages are held in Fourier space
      if (M.nz > 1)
        ck(cudaMemsetAsync(d->tmp0 + M.plane_size, 0, sizeof(double) * M.plane_size, d->ctx->stream), "nyq");
      transform(d, d->tmp0, STX_INVERSE);
    }
    ck(cudaMemcpy2DAsync(h_phys, sizeof(double) * M.nplane, d->tmp0, sizeof(double) * M.plane_size,
                         sizeof(double) * M.nplane, M.nz, cudaMemcpyDeviceToHost, d->ctx->stream),
       "download");
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_stats_set(stx_dns* d, char name, const double* h_phys) {
  return dns_guarded([&] {
    if (!d || !h_phys) throw DnsError(STX_EINVAL, "null argument");
    const Mesh& M = d->ctx->M;
    cudaSetDevice(d->ctx->device);
    double* b = avg_buffer(d, name);
    ck(cudaMemsetAsync(b, 0, sizeof(double) * d->fsize, d->ctx->stream), "zero");
    ck(cudaMemcpy2DAsync(b, sizeof(double) * M.plane_size, h_phys, sizeof(double) * M.nplane,
                         sizeof(double) * M.nplane, M.nz, cudaMemcpyHostToDevice, d->ctx->stream),
       "upload");
    if (d->names.find(name) != std::string::npos) {  // Statistics::initialise: raw data to Fourier space
      transform(d, b, STX_FORWARD);
      if (M.nz > 1) ck(cudaMemsetAsync(b + M.plane_size, 0, sizeof(double) * M.plane_size, d->ctx->stream), "nyq");
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_graph_info(const stx_dns* d, int* period, long long* launches) {
  return dns_guarded([&] {
    if (!d) throw DnsError(STX_EINVAL, "null argument");
    if (period) *period = d->gperiod;
    if (launches) *launches = d->graph_launches;
  });
}

namespace {

// Full-state checkpoint: a header of kCkptHeader doubles, then the device
// blocks of ckpt_blocks in order.
constexpr double kCkptMagic = 1398035523.0;  // "STXC" read as a little-endian int
constexpr int kCkptHeader = 16;

std::vector<std::pair<double*, size_t>> ckpt_blocks(stx_dns* d) {
  std::vector<std::pair<double*, size_t>> b;
  for (int i = 0; i <= d->ncom; ++i) b.emplace_back(d->u[i], d->fsize);
  for (int q = 0; q < d->nord; ++q)
    for (int i = 0; i < d->ncom; ++i) {
      b.emplace_back(d->Us[q][i], d->fsize);
      b.emplace_back(d->Uf[q][i], d->fsize);
    }
  for (size_t q = 0; q < d->un_lvl.size(); ++q) {
    b.emplace_back(d->un_lvl[q], d->hsize);
    b.emplace_back(d->hop_lvl[q], d->hsize);
  }
  const size_t ol = static_cast<size_t>(d->ctx->M.nz) * d->oe.ostride;
  for (double* a : d->o_uvw) b.emplace_back(a, 3 * ol);
  for (double* a : d->o_divu) b.emplace_back(a, ol);
  for (double* a : d->o_gradu) b.emplace_back(a, ol);
  const size_t nf = static_cast<size_t>(d->force.nzl) * d->ctx->M.plane_size;
  for (int i = 0; i < 3; ++i)
    if (d->force.qbar[i]) b.emplace_back(d->force.qbar[i], nf);
  if (d->force.mask) b.emplace_back(d->force.mask, nf);
  for (double* a : d->avg_buf) b.emplace_back(a, d->fsize);
  return b;
}

void ckpt_header(stx_dns* d, double* h, size_t nblock) {
  for (int k = 0; k < kCkptHeader; ++k) h[k] = 0.0;
  h[0] = kCkptMagic;
  h[1] = 1.0;  // format version
  h[2] = d->step;
  h[3] = d->time;
  h[4] = d->toggle;
  h[5] = d->ncom;
  h[6] = d->nord;
  h[7] = static_cast<double>(d->fsize);
  h[8] = static_cast<double>(d->hsize);
  h[9] = static_cast<double>(nblock);
  h[10] = d->navg;
  h[11] = d->force.sfd_started ? 1.0 : 0.0;
}

}  // namespace

}  // extern "C"

namespace stx {

std::vector<std::pair<double*, size_t>> dns_state_blocks(stx_dns* d) { return ckpt_blocks(d); }

DnsHostState dns_host_state(const stx_dns* d) {
  DnsHostState s;
  s.step = d->step;
  s.toggle = d->toggle;
  s.navg = d->navg;
  s.time = d->time;
  s.sfd_started = d->force.sfd_started;
  return s;
}

void dns_set_host_state(stx_dns* d, const DnsHostState& s) {
  drop_graph(d);
  d->eager_steady = 0;
  d->step = s.step;
  d->time = s.time;
  d->toggle = s.toggle;
  d->navg = s.navg;
  d->force.sfd_started = s.sfd_started;
  for (char c : d->names) ckstx(stx_field_bc_evaluate(d->ctx, c, d->time));
}

}  // namespace stx

extern "C" {

int stx_dns_checkpoint_size(stx_dns* d, unsigned long long* bytes) {
  return dns_guarded([&] {
    if (!d || !bytes) throw DnsError(STX_EINVAL, "null argument");
    size_t n = kCkptHeader;
    for (const auto& b : ckpt_blocks(d)) n += b.second;
    *bytes = sizeof(double) * n;
  });
}

int stx_dns_checkpoint_save(stx_dns* d, void* h_buf, unsigned long long bytes) {
  return dns_guarded([&] {
    if (!d || !h_buf) throw DnsError(STX_EINVAL, "null argument");
    const auto blocks = ckpt_blocks(d);
    size_t n = kCkptHeader;
    for (const auto& b : blocks) n += b.second;
    if (bytes < sizeof(double) * n) throw DnsError(STX_EINVAL, "checkpoint buffer too small");
    cudaSetDevice(d->ctx->device);
    double* h = static_cast<double*>(h_buf);
    ckpt_header(d, h, blocks.size());
    size_t off = kCkptHeader;
    for (const auto& b : blocks) {
      ck(cudaMemcpyAsync(h + off, b.first, sizeof(double) * b.second, cudaMemcpyDeviceToHost, d->ctx->stream),
         "checkpoint d2h");
      off += b.second;
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_checkpoint_load(stx_dns* d, const void* h_buf, unsigned long long bytes) {
  return dns_guarded([&] {
    if (!d || !h_buf) throw DnsError(STX_EINVAL, "null argument");
    const auto blocks = ckpt_blocks(d);
    size_t n = kCkptHeader;
    for (const auto& b : blocks) n += b.second;
    const double* h = static_cast<const double*>(h_buf);
    if (bytes < sizeof(double) * kCkptHeader || h[0] != kCkptMagic || h[1] != 1.0)
      throw DnsError(STX_EINVAL, "not a DNS checkpoint");
    double want[kCkptHeader];
    ckpt_header(d, want, blocks.size());
    for (int k : {5, 6, 7, 8, 9})
      if (h[k] != want[k]) throw DnsError(STX_EINVAL, "checkpoint of a different session or layout");
    if (bytes < sizeof(double) * n) throw DnsError(STX_EINVAL, "checkpoint buffer too small");
    cudaSetDevice(d->ctx->device);
    size_t off = kCkptHeader;
    for (const auto& b : blocks) {
      ck(cudaMemcpyAsync(b.first, h + off, sizeof(double) * b.second, cudaMemcpyHostToDevice, d->ctx->stream),
         "checkpoint h2d");
      off += b.second;
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    drop_graph(d);
    d->eager_steady = 0;
    d->step = static_cast<int>(h[2]);
    d->time = h[3];
    d->toggle = static_cast<int>(h[4]);
    d->navg = static_cast<int>(h[10]);
    d->force.sfd_started = h[11] != 0.0;
    for (char c : d->names) ckstx(stx_field_bc_evaluate(d->ctx, c, d->time));
  });
}

int stx_dns_system(stx_dns* d, char field, stx_modal** sys) {
  return dns_guarded([&] {
    if (!d || !sys) throw DnsError(STX_EINVAL, "null argument");
    const size_t idx = d->names.find(field);
    if (idx == std::string::npos) throw DnsError(STX_EINVAL, std::string("no field ") + field);
    if (static_cast<int>(idx) == d->ncom) *sys = d->psys;
    else *sys = d->vsys.at(idx);
  });
}

int stx_dns_field_ptr(stx_dns* d, char field, double** d_ptr) {
  return dns_guarded([&] {
    if (!d || !d_ptr) throw DnsError(STX_EINVAL, "null argument");
    const size_t idx = d->names.find(field);
    if (idx == std::string::npos) throw DnsError(STX_EINVAL, std::string("no field ") + field);
    *d_ptr = d->u[idx];
  });
}

}  // extern "C"
