// Discrete adjoint and tangent-linear model of the DNS time step (C ABI
// stx_dns_adjoint_*).
//
// A recorded run keeps full-state checkpoints on the device every K steps
// (the same blocks as stx_dns_checkpoint_*: velocity, the multistep storage
// Us / Uf of dns/integrate.cpp:99-136, the high-order pressure BC levels of
// src/bcmgr.cpp:951-993).  The backward sweep goes over the segments last
// to first: a segment is recomputed from its checkpoint, keeping the
// velocity u^n before each step, and its steps are then transposed in
// reverse order.  The transpose of step s (u^n -> u^s, n = s - 1) undoes
// integrate()'s sub-steps (dns/integrate.cpp:138-200) last to first:
//
//   viscous solves    F_i = Q4 solve0(ub_i / Q4)   (the systems are
//                     symmetric; the BC values are data, so the adjoint
//                     solve has zero BCs)
//   project           Uhat_i = alpha F_i,  pb += b D_i^T F_i
//   pressure solve    Fp = Q4 solve0(pb / Q4); the pressure BC lines get
//                     -w (the same solve at the edge knots)
//   setPForce         Uhat += D^T Fp / dt
//   waveProp          the history levels get the SS / EX weights
//   pressure BCs      the transpose of the high-order BC terms (curl curl,
//                     d(u.n)/dt, n.N, extrapolation)
//   nonlinear terms   DSS^T = Q4 DSS Q4^-1, the z transforms' transposes
//                     (forward: G D^-1 / N; inverse: N D F, D = 1 for the
//                     zeroth and Nyquist planes, 2 otherwise), and the
//                     transposed linearised advection at u^n.
//
// The tangent-linear model applies the linearised step forward along the
// same recorded trajectory (the nonlinear term's derivative as two calls of
// the forward kernel, the linear sub-steps with zero BC data).  Both use
// DIRECT systems: where the forward run solved by Jacobi-PCG (start-up
// orders, ITERATIVE = 1) the adjoint solves exactly, which the forward
// matches to its tolerance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/semtex_b200.h"
#include "dns_internal.hpp"
#include "kernels/adjoint_kernels.cuh"
#include "kernels/dns_kernels.cuh"
#include "kernels/helmholtz.cuh"
#include "stx_internal.hpp"

using namespace stx;

namespace {

struct AdjError : std::runtime_error {
  int code;
  AdjError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw AdjError(STX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void ckstx(int rc) {
  if (rc != STX_OK) throw AdjError(rc, stx_last_error());
}

template <class F>
int adj_guarded(F&& f) {
  try {
    f();
    set_last_error("");
    return STX_OK;
  } catch (const AdjError& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return dns_error_code(e);
  }
}

struct DevBuf {
  double* p = nullptr;
  DevBuf() = default;
  explicit DevBuf(size_t n) {
    if (n) ck(cudaMalloc(&p, sizeof(double) * n), "adjoint allocation");
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p) { o.p = nullptr; }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

struct stx_dns_adjoint {
  stx_dns* d = nullptr;
  int every = 10;
  // recorded run
  int s0 = -1, s1 = -1;
  size_t state_doubles = 0;
  std::vector<DevBuf> ckpt;  // state at s0 + j * every, and at s1 last (ckpt_host.size() in use)
  std::vector<DnsHostState> ckpt_host;
  // level rings (level l at l mod (nord + 1)): adjoint (or tangent) of the
  // velocity and nonlinear terms of level l, of its pressure-BC level and u.n
  DeviceArena arena;
  int nring = 0;
  std::vector<std::vector<double*>> Au, AN;
  std::vector<double*> AH, AUn;
  std::vector<double*> Uh, Fb, Up, A, dUp;  // [ncom] work fields
  double *pb = nullptr, *sp = nullptr, *T1 = nullptr, *Pb = nullptr, *Tc = nullptr, *Tcb = nullptr,
         *Bz = nullptr, *X = nullptr, *Y = nullptr;
  double* zero_lines = nullptr;  // [nz][max nline], zero
  double* dlines = nullptr;      // tangent pressure BC lines [nz][nline of p]
  std::vector<double*> seg;      // [every][ncom] recorded u^n of a segment
  std::vector<int> seg_form;
  std::vector<double*> ucur;     // [ncom] u^n of the step being transposed
  // steady transposed steps (all orders at N_TIME) replayed as CUDA graphs,
  // one per (level ring position, nonlinear form); a class runs directly
  // once (work buffers, systems, launch attributes settle), is captured the
  // second time
  bool use_graph = true;
  std::map<int, cudaGraphExec_t> rgraph;
  std::set<int> rseen;
  std::map<int, stx_modal*> vel_sys;  // DIRECT velocity systems by order (start-up, ITERATIVE)
  std::vector<stx_modal*> own_sys;
};

namespace {

size_t nline_max(const stx_dns* d) {
  size_t n = 0;
  for (char c : d->names) n = std::max(n, static_cast<size_t>(d->ctx->fields.at(c).nline));
  return n;
}

void zero(stx_dns* d, double* p, size_t n) {
  ck(cudaMemsetAsync(p, 0, sizeof(double) * n, d->ctx->stream), "zero");
}

void zero_nyquist(stx_dns* d, double* f) {
  if (d->ctx->M.nz > 1)
    ck(cudaMemsetAsync(f + d->ctx->M.plane_size, 0, sizeof(double) * d->ctx->M.plane_size, d->ctx->stream),
       "zero nyquist");
}

void copyf(stx_dns* d, double* dst, const double* src) {
  ck(cudaMemcpyAsync(dst, src, sizeof(double) * d->fsize, cudaMemcpyDeviceToDevice, d->ctx->stream), "copy");
}

void axpy(stx_dns* d, double* y, double c, const double* x) {  // y += c x
  CombineArgs a{};
  a.n = 2;
  a.c[0] = 1.0;
  a.p[0] = y;
  a.c[1] = c;
  a.p[1] = x;
  a.out = y;
  ck(dns_combine(d->ctx->dg, a, d->ctx->stream), "axpy");
}

void scale(stx_dns* d, double* y, double c, const double* x) {  // y = c x
  CombineArgs a{};
  a.n = 1;
  a.c[0] = c;
  a.p[0] = x;
  a.out = y;
  ck(dns_combine(d->ctx->dg, a, d->ctx->stream), "scale");
}

void ztrans(stx_dns* d, double* f, int sign) {
  ck(z_transform(f, d->ctx->M.nz, d->ctx->M.plane_size, sign, d->ctx->d_twiddle, nullptr, d->ctx->stream),
     "transform");
}

// f <- F^T f = G D^-1 f / N  (the transpose of the forward transform).
// N_Z = 2 is the reference's degenerate pair (forward: plane 1 zeroed;
// inverse: plane 1 = plane 0), whose forward transform is its own transpose.
void forward_t(stx_dns* d, double* f) {
  const int nz = d->ctx->M.nz;
  if (nz < 2) return;
  if (nz == 2) {
    ztrans(d, f, STX_FORWARD);
    return;
  }
  ck(adj_plane_weights(d->ctx->dg, f, 1.0 / nz, 1.0 / nz, 0.5 / nz, d->ctx->stream), "weights");
  ztrans(d, f, STX_INVERSE);
}

// f <- G^T f = N D F f  (the transpose of the inverse transform)
void inverse_t(stx_dns* d, double* f) {
  const int nz = d->ctx->M.nz;
  if (nz < 2) return;
  if (nz == 2) {
    ck(adj_fold_nz2(d->ctx->dg, f, d->ctx->stream), "fold");
    return;
  }
  ztrans(d, f, STX_FORWARD);
  ck(adj_plane_weights(d->ctx->dg, f, nz, nz, 2.0 * nz, d->ctx->stream), "weights");
}

stx_modal* velocity_system(stx_dns_adjoint* a, int i, int order) {
  stx_dns* d = a->d;
  if (order == d->nord && d->vsys[i]->method != STX_JACPCG) return d->vsys[i];
  const auto key = order * 8 + i;
  auto it = a->vel_sys.find(key);
  if (it != a->vel_sys.end()) return it->second;
  stx_modal* m = nullptr;
  const double lam = kSS[order][0] / (d->dt * d->nu);
  ckstx(stx_modal_create(d->ctx, d->names[i], lam, d->beta, 0, (d->ctx->M.nz + 1) / 2, STX_DIRECT, &m));
  a->own_sys.push_back(m);
  a->vel_sys.emplace(key, m);
  return m;
}

// out = Q4 solve0(in / Q4): the transpose of a solve's forcing -> solution
// map (T1 is scratch; the solve leaves the Nyquist plane, zeroed here).
void solve_t(stx_dns_adjoint* a, stx_modal* sys, const double* in, double* out) {
  stx_dns* d = a->d;
  const DevGeom& g = d->ctx->dg;
  ck(adj_mass(g, in, a->T1, 1, d->ctx->stream), "mass");
  ckstx(field_solve_with_lines(sys, a->T1, out, a->zero_lines));
  zero_nyquist(d, out);
  ck(adj_mass(g, out, out, 0, d->ctx->stream), "mass");
}

int ring(const stx_dns_adjoint* a, int level) { return ((level % a->nring) + a->nring) % a->nring; }

double* au(stx_dns_adjoint* a, int level, int c) { return a->Au[ring(a, level)][c]; }
double* an(stx_dns_adjoint* a, int level, int c) { return a->AN[ring(a, level)][c]; }
double* ah(stx_dns_adjoint* a, int level) { return a->AH[ring(a, level)]; }
double* aun(stx_dns_adjoint* a, int level) { return a->AUn[ring(a, level)]; }

void clear_rings(stx_dns_adjoint* a) {
  stx_dns* d = a->d;
  for (int r = 0; r < a->nring; ++r) {
    for (int c = 0; c < d->ncom; ++c) {
      zero(d, a->Au[r][c], d->fsize);
      zero(d, a->AN[r][c], d->fsize);
    }
    if (d->nh) {
      zero(d, a->AH[r], d->hsize);
      zero(d, a->AUn[r], d->hsize);
    }
  }
}

// Weights of the convective and conservative parts of a nonlinear form.
void form_weights(int form, double& cw, double& cb) {
  cw = form == 0 ? 0.5 : (form == 1 ? 1.0 : 0.0);
  cb = form == 0 ? 0.5 : (form == 2 ? 1.0 : 0.0);
}

// Physical velocity of level u (Fourier components) into Up.
void physical(stx_dns_adjoint* a, const double* const* u, std::vector<double*>& out) {
  stx_dns* d = a->d;
  for (int c = 0; c < d->ncom; ++c) {
    copyf(d, out[c], u[c]);
    ztrans(d, out[c], STX_INVERSE);
  }
}

// -- the transpose of step s (u^n -> u^s), n = s - 1 ------------------------
void reverse_step(stx_dns_adjoint* a, int s, const double* const* un, int form) {
  stx_dns* d = a->d;
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  const int n = s - 1, ncom = d->ncom;
  const bool z3 = d->ndim == 3;
  const int Je = std::min(s, d->nord);
  // viscous solves
  for (int i = 0; i < ncom; ++i) {
    solve_t(a, velocity_system(a, i, Je), au(a, s, i), a->Fb[i]);
    zero(d, au(a, s, i), d->fsize);
  }
  // project: F_i = alpha Uhat_i + b dp/dx_i
  const double alpha = -1.0 / (d->dt * d->nu), bcoef = 1.0 / d->nu;
  zero(d, a->pb, d->fsize);
  for (int i = 0; i < ncom; ++i) {
    scale(d, a->Uh[i], alpha, a->Fb[i]);
    const int dir = i < d->ndim ? i : -1;
    if (dir == 0 || dir == 1) ck(adj_grad_t(g, a->Fb[i], a->pb, dir, bcoef, st), "project^T");
    if (dir == 2) ck(adj_grad_z_acc(g, a->Fb[i], a->pb, -bcoef, d->beta, st), "project^T");
  }
  // pressure solve (sp kept for the BC lines)
  ck(adj_mass(g, a->pb, a->T1, 1, st), "mass");
  ckstx(field_solve_with_lines(d->psys, a->T1, a->sp, a->zero_lines));
  zero_nyquist(d, a->sp);
  ck(adj_mass(g, a->sp, a->X, 0, st), "mass");  // X = adjoint of the pressure forcing
  // setPForce: Fp = (dUhat0/dx + dUhat1/dy + dUhat2/dz) / dt
  ck(adj_grad_t(g, a->X, a->Uh[0], 0, 1.0 / d->dt, st), "setPForce^T");
  ck(adj_grad_t(g, a->X, a->Uh[1], 1, 1.0 / d->dt, st), "setPForce^T");
  if (z3) ck(adj_grad_z_acc(g, a->X, a->Uh[2], -1.0 / d->dt, d->beta, st), "setPForce^T");
  // waveProp
  for (int q = 0; q < Je; ++q)
    for (int c = 0; c < ncom; ++c) {
      axpy(d, au(a, n - q, c), -kSS[Je][q + 1], a->Uh[c]);
      axpy(d, an(a, n - q, c), kEX[Je][q] * d->dt, a->Uh[c]);
    }
  // high-order pressure BCs of this step
  if (d->nh) {
    const FieldDev& P = ctx->fields.at(d->names[ncom]);
    HopbcAdjArgs h{};
    h.sp = a->sp;
    h.edge_area = P.dn.edge_area;
    h.nh = d->nh;
    h.elmt = d->h_elmt;
    h.side = d->h_side;
    h.line = d->h_line;
    h.nx = d->h_nx;
    h.ny = d->h_ny;
    const int Jh = std::min(s - 1, d->nord), Jx = std::min(s, d->nord);
    h.hop_adj = ah(a, n);
    h.un_adj = aun(a, n);
    for (int q = 0; q + 1 < Jx; ++q) h.hop_old_adj[q] = ah(a, n - 1 - q);
    for (int q = 0; q < Jh; ++q) h.un_old_adj[q] = aun(a, n - 1 - q);
    h.Au = au(a, n, 0);
    h.Av = au(a, n, 1);
    h.Aw = z3 ? au(a, n, 2) : nullptr;
    h.ANx = an(a, n, 0);
    h.ANy = an(a, n, 1);
    h.Je = Jh;
    for (int q = 0; q <= Jh; ++q) h.alpha[q] = kSS[Jh][q];
    h.invdt = 1.0 / d->dt;
    h.nu = d->nu;
    h.beta = d->beta;
    h.Jx = Jx;
    for (int q = 0; q < Jx; ++q) h.ex[q] = kEX[Jx][q];
    ck(adj_hopbc(g, h, st), "hopbc^T");
    zero(d, ah(a, n), d->hsize);
    zero(d, aun(a, n), d->hsize);
  }
  // nonlinear terms N^n = DSS(F(N_phys(u^n)))
  if (form >= 0) {
    double cw, cb;
    form_weights(form, cw, cb);
    physical(a, un, a->Up);
    for (int c = 0; c < ncom; ++c) zero(d, a->A[c], d->fsize);
    const DevNumbering& Nm = ctx->fields.at(d->names[0]).dn;
    for (int i = 0; i < ncom; ++i) {
      ck(adj_mass(g, an(a, n, i), a->Pb, 1, st), "mass");
      ck(dns_smooth(g, Nm, a->Pb, d->dsswork, st), "smooth");
      ck(adj_mass(g, a->Pb, a->Pb, 0, st), "mass");
      forward_t(d, a->Pb);
      const bool zc = z3 && cw != 0.0, zk = z3 && cb != 0.0;
      if (zc) {  // Tc = inverse transform of dU_i/dz
        ck(dns_grad_z(g, un[i], a->Tc, d->beta, st), "gradz");
        ztrans(d, a->Tc, STX_INVERSE);
      }
      NlAdjArgs na{};
      na.Pb = a->Pb;
      na.U0 = a->Up[0];
      na.U1 = a->Up[1];
      na.U2 = z3 ? a->Up[2] : nullptr;
      na.Ui = a->Up[i];
      na.Tc = zc ? a->Tc : nullptr;
      na.A0 = a->A[0];
      na.A1 = a->A[1];
      na.A2 = z3 ? a->A[2] : nullptr;
      na.Ai = a->A[i];
      na.Tcb = zc ? a->Tcb : nullptr;
      na.Bz = zk ? a->Bz : nullptr;
      na.cw = cw;
      na.cb = cb;
      ck(adj_nonlinear(g, na, st), "nonlinear^T");
      if (zc) {  // -U2 F^-1(dz u_i): u_i gets -dz G^T of its adjoint
        inverse_t(d, a->Tcb);
        ck(adj_grad_z_acc(g, a->Tcb, au(a, n, i), -1.0, d->beta, st), "gradz^T");
      }
      if (zk) {  // -F^-1(dz F(U_i U_2))
        inverse_t(d, a->Bz);
        zero(d, a->Y, d->fsize);
        ck(adj_grad_z_acc(g, a->Bz, a->Y, 1.0, d->beta, st), "gradz");
        forward_t(d, a->Y);
        ck(adj_product2(g, a->Up[2], a->Up[i], a->Y, a->A[i], a->A[2], st), "product^T");
      }
    }
    for (int c = 0; c < ncom; ++c) {
      inverse_t(d, a->A[c]);
      axpy(d, au(a, n, c), 1.0, a->A[c]);
    }
  }
  for (int c = 0; c < ncom; ++c) {
    zero(d, an(a, n, c), d->fsize);
    zero_nyquist(d, au(a, n, c));
  }
}

// The transpose of step s on u^n in a->ucur: directly, or as the replay of
// the captured graph of its class (steady steps: every order at N_TIME).
void run_reverse(stx_dns_adjoint* a, int s, int form) {
  stx_dns* d = a->d;
  cudaStream_t st = d->ctx->stream;
  if (!a->use_graph || s <= d->nord) {
    reverse_step(a, s, a->ucur.data(), form);
    return;
  }
  const int key = ring(a, s) * 4 + (form + 1);
  const auto it = a->rgraph.find(key);
  if (it != a->rgraph.end()) {
    ck(cudaGraphLaunch(it->second, st), "graph launch");
    return;
  }
  if (a->rseen.insert(key).second) {
    reverse_step(a, s, a->ucur.data(), form);
    return;
  }
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    a->use_graph = false;
    reverse_step(a, s, a->ucur.data(), form);
    return;
  }
  bool ok = true;
  try {
    reverse_step(a, s, a->ucur.data(), form);
  } catch (const std::exception&) {
    ok = false;
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &graph);
  cudaGraphExec_t exec = nullptr;
  ok = ok && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();  // clear a capture error: the step runs directly instead
  if (!ok) {
    a->use_graph = false;
    reverse_step(a, s, a->ucur.data(), form);
    return;
  }
  a->rgraph[key] = exec;
  ck(cudaGraphLaunch(exec, st), "graph launch");
}

// -- the tangent-linear step s along the trajectory (u^n given) -------------
void tangent_step(stx_dns_adjoint* a, int s, const double* const* un, int form) {
  stx_dns* d = a->d;
  stx_context* ctx = d->ctx;
  const DevGeom& g = ctx->dg;
  cudaStream_t st = ctx->stream;
  const int n = s - 1, ncom = d->ncom;
  const bool z3 = d->ndim == 3;
  const DevNumbering& Nm = ctx->fields.at(d->names[0]).dn;
  // dN^n = N'(u^n) du^n = B(du, u) + B(u, du), B(a, b) the forward kernel's
  // bilinear form (advecting a, advected b)
  std::vector<const double*> du(ncom);
  for (int c = 0; c < ncom; ++c) du[c] = au(a, n, c);
  if (form >= 0) {
    physical(a, un, a->Up);
    physical(a, du.data(), a->dUp);
    for (int i = 0; i < ncom; ++i) {
      double* N = an(a, n, i);
      for (int call = 0; call < 2; ++call) {
        const std::vector<double*>& adv = call ? a->Up : a->dUp;
        const double* bi = call ? a->dUp[i] : a->Up[i];
        const double* bf = call ? du[i] : un[i];  // Fourier of the advected component
        NonlinearArgs na{};
        na.U0 = adv[0];
        na.U1 = adv[1];
        na.U2 = z3 ? adv[2] : nullptr;
        na.Ui = bi;
        na.N = call ? a->Y : a->X;
        na.form = form;
        if (z3 && form != 2) {
          ck(dns_grad_z(g, bf, a->Tc, d->beta, st), "gradz");
          ztrans(d, a->Tc, STX_INVERSE);
          na.Tc = a->Tc;
        }
        if (z3 && form != 1) {
          ck(dns_product(g, bi, adv[2], a->Tcb, st), "product");
          ztrans(d, a->Tcb, STX_FORWARD);
          ck(dns_grad_z(g, a->Tcb, a->Bz, d->beta, st), "gradz");
          ztrans(d, a->Bz, STX_INVERSE);
          na.Tk = a->Bz;
        }
        ck(dns_nonlinear(g, na, st), "nonlinear");
      }
      scale(d, N, 1.0, a->X);
      axpy(d, N, 1.0, a->Y);
      ztrans(d, N, STX_FORWARD);
      ck(dns_smooth(g, Nm, N, d->dsswork, st), "smooth");
    }
  } else {
    for (int i = 0; i < ncom; ++i) zero(d, an(a, n, i), d->fsize);
  }
  // high-order pressure BCs from the tangent levels
  if (d->nh) {
    const FieldDev& P = ctx->fields.at(d->names[ncom]);
    const int Jh = std::min(s - 1, d->nord), Jx = std::min(s, d->nord);
    HopbcArgs h{};
    h.U = du[0];
    h.V = du[1];
    h.W = z3 ? du[2] : nullptr;
    h.Nx = an(a, n, 0);
    h.Ny = an(a, n, 1);
    h.nh = d->nh;
    h.elmt = d->h_elmt;
    h.side = d->h_side;
    h.line = d->h_line;
    h.nx = d->h_nx;
    h.ny = d->h_ny;
    for (int q = 0; q < Jh; ++q) h.un_old[q] = aun(a, n - 1 - q);
    h.un_new = aun(a, n);
    h.hop_new = ah(a, n);
    for (int q = 0; q + 1 < Jx; ++q) h.hop_old[q] = ah(a, n - 1 - q);
    h.lines = a->dlines;
    h.nline = P.nline;
    h.Je = Jh;
    for (int q = 0; q <= Jh; ++q) h.alpha[q] = kSS[Jh][q];
    h.invdt = 1.0 / d->dt;
    h.nu = d->nu;
    h.beta = d->beta;
    h.Jx = Jx;
    for (int q = 0; q < Jx; ++q) h.ex[q] = kEX[Jx][q];
    ck(dns_hopbc(g, h, st), "hopbc");
  }
  // waveProp
  const int Je = std::min(s, d->nord);
  for (int c = 0; c < ncom; ++c) {
    CombineArgs w{};
    for (int q = 0; q < Je; ++q) {
      w.c[w.n] = -kSS[Je][q + 1];
      w.p[w.n++] = au(a, n - q, c);
      w.c[w.n] = kEX[Je][q] * d->dt;
      w.p[w.n++] = an(a, n - q, c);
    }
    w.out = a->Uh[c];
    ck(dns_combine(g, w, st), "waveProp");
  }
  // setPForce, pressure solve with the tangent BC lines, project
  ck(dns_divergence(g, a->Uh[0], a->Uh[1], z3 ? a->Uh[2] : nullptr, a->X, d->dt, d->beta, st), "setPForce");
  ckstx(field_solve_with_lines(d->psys, a->X, a->sp, d->nh ? a->dlines : a->zero_lines));
  zero_nyquist(d, a->sp);
  const double alpha = -1.0 / (d->dt * d->nu), bcoef = 1.0 / d->nu;
  for (int i = 0; i < ncom; ++i)
    ck(dns_project(g, a->Uh[i], a->sp, i < d->ndim ? i : -1, alpha, bcoef, d->beta, st), "project");
  // viscous solves with zero BC data into level s
  for (int i = 0; i < ncom; ++i) {
    double* out = au(a, s, i);
    ckstx(field_solve_with_lines(velocity_system(a, i, Je), a->Uh[i], out, a->zero_lines));
    zero_nyquist(d, out);
  }
}

// -- checkpoints ----------------------------------------------------------
void save_state(stx_dns_adjoint* a, DevBuf& buf) {
  stx_dns* d = a->d;
  size_t off = 0;
  for (const auto& b : dns_state_blocks(d)) {
    ck(cudaMemcpyAsync(buf.p + off, b.first, sizeof(double) * b.second, cudaMemcpyDeviceToDevice, d->ctx->stream),
       "checkpoint");
    off += b.second;
  }
}

void load_state(stx_dns_adjoint* a, int j) {
  stx_dns* d = a->d;
  size_t off = 0;
  for (const auto& b : dns_state_blocks(d)) {
    ck(cudaMemcpyAsync(b.first, a->ckpt[j].p + off, sizeof(double) * b.second, cudaMemcpyDeviceToDevice,
                       d->ctx->stream),
       "restore");
    off += b.second;
  }
  dns_set_host_state(d, a->ckpt_host[j]);
}

// Host physical fields [ncom][nz][nplane] <-> device Fourier-layout planes.
void upload(stx_dns* d, const double* h, double* f) {
  const Mesh& M = d->ctx->M;
  zero(d, f, d->fsize);
  ck(cudaMemcpy2DAsync(f, sizeof(double) * M.plane_size, h, sizeof(double) * M.nplane, sizeof(double) * M.nplane,
                       M.nz, cudaMemcpyHostToDevice, d->ctx->stream),
     "upload");
}

void download(stx_dns* d, const double* f, double* h) {
  const Mesh& M = d->ctx->M;
  ck(cudaMemcpy2DAsync(h, sizeof(double) * M.nplane, f, sizeof(double) * M.plane_size, sizeof(double) * M.nplane,
                       M.nz, cudaMemcpyDeviceToHost, d->ctx->stream),
     "download");
}

void require_recorded(const stx_dns_adjoint* a) {
  if (a->s0 < 0 || a->ckpt_host.empty()) throw AdjError(STX_EINVAL, "no recorded run (stx_dns_adjoint_record)");
}

}  // namespace

extern "C" {

int stx_dns_adjoint_create(stx_dns* d, int checkpoint_every, stx_dns_adjoint** out) {
  return adj_guarded([&] {
    if (!d || !out) throw AdjError(STX_EINVAL, "null argument");
    if (checkpoint_every < 1) throw AdjError(STX_EINVAL, "checkpoint interval must be >= 1");
    *out = nullptr;
    const Session& S = d->ctx->S;
    const TokenTable& T = S.tokens;
    if (d->nz32) throw AdjError(STX_EUNSUPPORTED, "adjoint: 3/2-rule products (DEALIAS) are not differentiated");
    if (d->oe.no) throw AdjError(STX_EUNSUPPORTED, "adjoint: computed outflow BCs are not differentiated");
    if (d->mixed) throw AdjError(STX_EUNSUPPORTED, "adjoint: mixed-precision velocity solves (STX_DNS_MIXED)");
    if (T.value("SVV_EPSN") > 6.0e-14 || T.value("SVV_EPSZ") > 6.0e-14)
      throw AdjError(STX_EUNSUPPORTED, "adjoint: spectral vanishing viscosity is not differentiated");
    const auto& F = d->force;
    if (F.mask || F.drag || F.coriolis || F.qbar[0] || F.qbar[1] || F.qbar[2])
      throw AdjError(STX_EUNSUPPORTED,
                     "adjoint: velocity-dependent forcing (sponge, drag, Coriolis, SFD) is not differentiated");
    if (d->ndim == 3 && d->ncom != 3) throw AdjError(STX_EUNSUPPORTED, "adjoint: 3D needs u v w");
    if (d->ctx->dg.npnp > 256) throw AdjError(STX_EUNSUPPORTED, "adjoint: N_P > 16");
    cudaSetDevice(d->ctx->device);
    auto a = new stx_dns_adjoint();
    std::unique_ptr<stx_dns_adjoint> guard(a);
    a->d = d;
    a->every = checkpoint_every;
    for (const auto& b : dns_state_blocks(d)) a->state_doubles += b.second;
    a->nring = d->nord + 1;
    const int ncom = d->ncom;
    const size_t fs = d->fsize;
    const int nwork = 2 * a->nring * ncom + 6 * ncom + 9;
    double* base = static_cast<double*>(a->arena.alloc(sizeof(double) * fs * nwork));
    ck(cudaMemset(base, 0, sizeof(double) * fs * nwork), "memset");
    int k = 0;
    a->Au.assign(a->nring, {});
    a->AN.assign(a->nring, {});
    for (int r = 0; r < a->nring; ++r)
      for (int c = 0; c < ncom; ++c) {
        a->Au[r].push_back(base + fs * k++);
        a->AN[r].push_back(base + fs * k++);
      }
    for (auto* v : {&a->Uh, &a->Fb, &a->Up, &a->A, &a->dUp, &a->ucur})
      for (int c = 0; c < ncom; ++c) v->push_back(base + fs * k++);
    for (double** p : {&a->pb, &a->sp, &a->T1, &a->Pb, &a->Tc, &a->Tcb, &a->Bz, &a->X, &a->Y}) *p = base + fs * k++;
    if (d->nh) {
      double* hb = static_cast<double*>(a->arena.alloc(sizeof(double) * d->hsize * 2 * a->nring));
      ck(cudaMemset(hb, 0, sizeof(double) * d->hsize * 2 * a->nring), "memset");
      for (int r = 0; r < a->nring; ++r) {
        a->AH.push_back(hb + d->hsize * (2 * r));
        a->AUn.push_back(hb + d->hsize * (2 * r + 1));
      }
    }
    const size_t nl = static_cast<size_t>(d->ctx->M.nz) * std::max<size_t>(nline_max(d), 1);
    a->zero_lines = static_cast<double*>(a->arena.alloc(sizeof(double) * nl));
    a->dlines = static_cast<double*>(a->arena.alloc(sizeof(double) * nl));
    ck(cudaMemset(a->zero_lines, 0, sizeof(double) * nl), "memset");
    ck(cudaMemset(a->dlines, 0, sizeof(double) * nl), "memset");
    double* sb = static_cast<double*>(a->arena.alloc(sizeof(double) * fs * ncom * checkpoint_every));
    for (int j = 0; j < ncom * checkpoint_every; ++j) a->seg.push_back(sb + fs * j);
    a->seg_form.assign(checkpoint_every, 0);
    a->use_graph = d->use_graph;
    *out = guard.release();
  });
}

int stx_dns_adjoint_destroy(stx_dns_adjoint* a) {
  return adj_guarded([&] {
    if (!a) return;
    cudaSetDevice(a->d->ctx->device);
    cudaStreamSynchronize(a->d->ctx->stream);
    for (auto& g : a->rgraph) cudaGraphExecDestroy(g.second);
    for (stx_modal* m : a->own_sys) stx_modal_destroy(m);
    delete a;
  });
}

int stx_dns_adjoint_record(stx_dns_adjoint* a, int nsteps) {
  return adj_guarded([&] {
    if (!a || nsteps < 1) throw AdjError(STX_EINVAL, "bad argument");
    stx_dns* d = a->d;
    cudaSetDevice(d->ctx->device);
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    // checkpoint buffers are kept from record to record (allocated only
    // when a longer run needs more of them)
    a->ckpt_host.clear();
    a->s0 = a->s1 = -1;
    const int s0 = d->step;
    auto keep = [&] {
      const size_t j = a->ckpt_host.size();
      if (j == a->ckpt.size()) a->ckpt.emplace_back(a->state_doubles);
      save_state(a, a->ckpt[j]);
      a->ckpt_host.push_back(dns_host_state(d));
    };
    keep();
    for (int left = nsteps; left > 0;) {
      const int k = std::min(a->every, left);
      ckstx(stx_dns_advance(d, k));
      left -= k;
      keep();
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    a->s0 = s0;
    a->s1 = d->step;
  });
}

int stx_dns_adjoint_backward(stx_dns_adjoint* a, const double* h_seed, double* h_grad) {
  return adj_guarded([&] {
    if (!a || !h_seed || !h_grad) throw AdjError(STX_EINVAL, "null argument");
    require_recorded(a);
    stx_dns* d = a->d;
    const Mesh& M = d->ctx->M;
    const int ncom = d->ncom;
    const size_t nphys = static_cast<size_t>(M.nz) * M.nplane;
    cudaSetDevice(d->ctx->device);
    clear_rings(a);
    // seed: the final velocity read as stx_dns_get_field does (Nyquist
    // plane zeroed, inverse transform), so its adjoint is Z G^T seed
    for (int c = 0; c < ncom; ++c) {
      double* f = au(a, a->s1, c);
      upload(d, h_seed + nphys * c, f);
      inverse_t(d, f);
      zero_nyquist(d, f);
    }
    const int nseg = static_cast<int>(a->ckpt_host.size()) - 1;
    for (int j = nseg - 1; j >= 0; --j) {
      const int sa = a->s0 + j * a->every, sb = std::min(sa + a->every, a->s1);
      load_state(a, j);
      for (int s = sa + 1; s <= sb; ++s) {
        const int slot = s - sa - 1;
        for (int c = 0; c < ncom; ++c) copyf(d, a->seg[slot * ncom + c], d->u[c]);
        a->seg_form[slot] = dns_next_form(d);
        if (s < sb) dns_advance_one(d);
      }
      for (int s = sb; s > sa; --s) {
        const int slot = s - sa - 1;
        for (int c = 0; c < ncom; ++c) copyf(d, a->ucur[c], a->seg[slot * ncom + c]);
        run_reverse(a, s, a->seg_form[slot]);
      }
    }
    // gradient w.r.t. the physical velocity given to stx_dns_set_field
    // (forward transform, Nyquist plane zeroed): F^T Z ub
    for (int c = 0; c < ncom; ++c) {
      double* f = au(a, a->s0, c);
      zero_nyquist(d, f);
      forward_t(d, f);
      download(d, f, h_grad + nphys * c);
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    load_state(a, nseg);
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_adjoint_tangent(stx_dns_adjoint* a, const double* h_dir, double* h_out) {
  return adj_guarded([&] {
    if (!a || !h_dir || !h_out) throw AdjError(STX_EINVAL, "null argument");
    require_recorded(a);
    stx_dns* d = a->d;
    const Mesh& M = d->ctx->M;
    const int ncom = d->ncom;
    const size_t nphys = static_cast<size_t>(M.nz) * M.nplane;
    cudaSetDevice(d->ctx->device);
    clear_rings(a);
    for (int c = 0; c < ncom; ++c) {
      double* f = au(a, a->s0, c);
      upload(d, h_dir + nphys * c, f);
      ztrans(d, f, STX_FORWARD);
      zero_nyquist(d, f);
    }
    if (d->nh) {
      const size_t nl = static_cast<size_t>(M.nz) * std::max<size_t>(nline_max(d), 1);
      zero(d, a->dlines, nl);
    }
    load_state(a, 0);
    for (int s = a->s0 + 1; s <= a->s1; ++s) {
      std::vector<const double*> un(d->u.begin(), d->u.begin() + ncom);
      tangent_step(a, s, un.data(), dns_next_form(d));
      dns_advance_one(d);
    }
    for (int c = 0; c < ncom; ++c) {
      double* f = au(a, a->s1, c);
      copyf(d, a->X, f);
      zero_nyquist(d, a->X);
      ztrans(d, a->X, STX_INVERSE);
      download(d, a->X, h_out + nphys * c);
    }
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
    load_state(a, static_cast<int>(a->ckpt_host.size()) - 1);
    ck(cudaStreamSynchronize(d->ctx->stream), "sync");
  });
}

int stx_dns_adjoint_info(const stx_dns_adjoint* a, int* first_step, int* last_step,
                         unsigned long long* checkpoint_bytes) {
  return adj_guarded([&] {
    if (!a) throw AdjError(STX_EINVAL, "null argument");
    if (first_step) *first_step = a->s0;
    if (last_step) *last_step = a->s1;
    if (checkpoint_bytes) *checkpoint_bytes = sizeof(double) * a->state_doubles * a->ckpt_host.size();
  });
}

}  // extern "C"
