// Launchers of the DNS step kernels (asynchronous on the given stream).
// All field arguments are nz planes of plane_size doubles.
#pragma once

#include <cstddef>

#include "device.hpp"

namespace stx {

struct NonlinearArgs {
  const double* U0;  // physical velocity components
  const double* U1;
  const double* U2;  // null in 2D
  const double* Ui;  // component i, physical
  const double* Tc;  // inverse FFT of dUi/dz (convective z term) or null
  const double* Tk;  // inverse FFT of d(Ui U2)/dz (conservative z term) or null
  double* N;
  int form;          // 0 skew-symmetric average, 1 convective, 2 conservative
};

struct CombineArgs {
  int n;
  double c[8];
  const double* p[8];
  double* out;
};

// High-order pressure BC terms of one step (BCmgr::maintainFourier,
// src/bcmgr.cpp:1036-1296; Edge::curlCurl, src/edge.cpp:110-256) and their
// extrapolation into the pressure BC lines (BCmgr::evaluateCNBCp,
// :1299-1331).  Edge storage is [nz][nh*np], edge h at h*np, knots in the
// CCW side traverse.
struct HopbcArgs {
  const double* U;            // Fourier velocity components (current level)
  const double* V;
  const double* W;            // null in 2D
  const double* Nx;           // Fourier nonlinear terms of the same level
  const double* Ny;
  int nh;                     // high-order pressure edges
  const int* elmt;            // [nh] element, side and BC line edge number
  const int* side;
  const int* line;
  const double* nx;           // [nh*np] unit outward normal
  const double* ny;
  const double* un_old[3];    // u.n of the previous steps, newest first
  double* un_new;             // u.n of this step (may be un_old[Je-1]: each entry is read first)
  const double* hop_old[2];   // earlier pressure BC levels, newest first
  double* hop_new;
  double* lines;              // pressure BC lines [nz][nline]
  int nline;
  int Je;                     // time-derivative order (0: no -d(u.n)/dt term)
  double alpha[4];            // stiffly stable coefficients of order Je
  double invdt, nu, beta;
  int Jx;                     // extrapolation order
  double ex[3];               // extrapolation coefficients of order Jx
};

size_t dns_hopbc_smem(const DevGeom& g);
cudaError_t dns_hopbc(const DevGeom& g, const HopbcArgs& a, cudaStream_t st);

// Analysis reductions, as per-block partials (dns_analysis_blocks() per
// mode) that the host sums in a fixed order: Q4-weighted energy of every
// mode of a Fourier field (part[m * blocks + b]); the CFL maxima of plane 0.
int dns_analysis_blocks();
cudaError_t dns_mode_energy_partials(const DevGeom& g, const double* f, double* part, cudaStream_t st);
cudaError_t dns_cfl_partials(const DevGeom& g, const double* u, int dir, double d, double* part, cudaStream_t st);

// History-point values: out[p * nf + f] for fields f[0..nf) at points
// p < npts on elements elmt[p], with per-point weights w[p][2 np + nzc]
// (interpolants in s, in r, then nzc Fourier coefficients).
struct ProbeArgs {
  int npts, nf, nzc;
  const int* elmt;
  const double* w;
  const double* f[8];
  double* out;
};
cudaError_t dns_probe(const DevGeom& g, const ProbeArgs& a, cudaStream_t st);

// Wall forces: per edge b (element elmt[b], side nodes node[b][np] in the
// side traverse, unit normal and quadrature-weighted length per node) the
// five sums out[5 b ..] of the plane-0 data (pressure x, y; viscous x, y;
// flux of w, 0 when w is null).
struct WallArgs {
  int nw;
  const int* elmt;
  const int* node;
  const double* nx;
  const double* ny;
  const double* area;
  const double* p;
  const double* u;
  const double* v;
  const double* w;
  double* out;
};
cudaError_t dns_wall_forces(const DevGeom& g, const WallArgs& a, cudaStream_t st);

// Wall tractions of every Fourier mode: plane k of out (npad doubles a
// plane) holds the normal (pressure) values of the wall lines at [0, nline),
// the in-plane viscous traction at [nline, 2 nline) and the out-of-plane one
// at [2 nline, 3 nline) (zero when w is null), edges as in WallArgs.
struct TractionArgs {
  int nw, nline, npad, nz;
  const int* elmt;
  const int* node;
  const double* nx;
  const double* ny;
  const double* p;
  const double* u;
  const double* v;
  const double* w;
  double mu, beta;
  double* out;
};
cudaError_t dns_wall_traction(const DevGeom& g, const TractionArgs& a, cudaStream_t st);

cudaError_t dns_grad_xy(const DevGeom& g, const double* in, double* out, int dir, cudaStream_t st);
cudaError_t dns_grad_z(const DevGeom& g, const double* in, double* out, double beta, cudaStream_t st);
cudaError_t dns_product(const DevGeom& g, const double* a, const double* b, double* out, cudaStream_t st);
cudaError_t dns_nonlinear(const DevGeom& g, const NonlinearArgs& a, cudaStream_t st);
size_t dns_smooth_workspace_doubles(const DevGeom& g, const DevNumbering& N);
cudaError_t dns_smooth(const DevGeom& g, const DevNumbering& N, double* io, double* work, cudaStream_t st);
cudaError_t dns_combine(const DevGeom& g, const CombineArgs& a, cudaStream_t st);
cudaError_t dns_divergence(const DevGeom& g, const double* a0, const double* a1, const double* a2, double* out,
                           double dt, double beta, cudaStream_t st);
cudaError_t dns_project(const DevGeom& g, double* io, const double* p, int dir, double alpha, double b,
                        double beta, cudaStream_t st);

}  // namespace stx
