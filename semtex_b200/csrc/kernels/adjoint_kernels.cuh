// Launchers of the kernels of the DNS step's discrete adjoint (transposes of
// the step's linear operators and of the linearised nonlinear terms).  All
// field arguments are nz planes of plane_size doubles; only the first
// nel * npnp doubles of each plane are read or written.
#pragma once

#include <cstddef>

#include "device.hpp"

namespace stx {

// io *= Q4 (mode 0) or io /= Q4 (mode 1) at every node of every plane;
// out-of-place when in != io.
cudaError_t adj_mass(const DevGeom& g, const double* in, double* io, int mode, cudaStream_t st);

// io[plane k] *= w0 (k = 0), w1 (k = 1), wc (k >= 2): the diagonal that
// turns the z transforms into their transposes.
cudaError_t adj_plane_weights(const DevGeom& g, double* io, double w0, double w1, double wc, cudaStream_t st);

// The transpose of the N_Z = 2 inverse transform (plane 1 a copy of plane
// 0): plane 0 += plane 1, plane 1 = 0.
cudaError_t adj_fold_nz2(const DevGeom& g, double* io, cudaStream_t st);

// out += s * transpose(d/dx_dir) in  (dir 0: x, 1: y; element by element).
cudaError_t adj_grad_t(const DevGeom& g, const double* in, double* out, int dir, double s, cudaStream_t st);

// out += s * d/dz in  (Fourier planes, wavenumber factor beta; d/dz is
// antisymmetric, so s = -c applies c times its transpose).
cudaError_t adj_grad_z_acc(const DevGeom& g, const double* in, double* out, double s, double beta,
                           cudaStream_t st);

// Transpose of the linearised nonlinear term of one component i at the
// physical velocity U: given Pb (adjoint of the physical term, before its
// forward transform), with weights cw (convective part) and cb
// (conservative part):
//   A0, A1 (and A2 in 3D) += the element and pointwise parts of the
//   transpose (A_i included); Tcb = -cw U2 Pb (3D, cw != 0) and
//   Bz = cb Pb (3D, cb != 0) are written for the z terms.
struct NlAdjArgs {
  const double* Pb;
  const double* U0;
  const double* U1;
  const double* U2;   // null in 2D
  const double* Ui;
  const double* Tc;   // inverse transform of dU_i/dz (3D, cw != 0), else null
  double* A0;
  double* A1;
  double* A2;         // null in 2D
  double* Ai;         // one of A0, A1, A2
  double* Tcb;        // null unless 3D and cw != 0
  double* Bz;         // null unless 3D and cb != 0
  double cw, cb;
};
cudaError_t adj_nonlinear(const DevGeom& g, const NlAdjArgs& a, cudaStream_t st);

// Ai += U2 Z; A2 += Ui Z  (the transpose of the product in the
// conservative z term, d(U_i U_2)/dz).
cudaError_t adj_product2(const DevGeom& g, const double* U2, const double* Ui, const double* Z, double* Ai,
                         double* A2, cudaStream_t st);

// Transpose of one step's high-order pressure BC terms (the kernel of
// dns_hopbc) for the edges' element data at Us[0] / Uf[0].
struct HopbcAdjArgs {
  const double* sp;           // pressure solve of the adjoint (element layout, Fourier)
  const double* edge_area;    // pressure BC weights [nedge*np]
  int nh;
  const int* elmt;
  const int* side;
  const int* line;
  const double* nx;
  const double* ny;
  const double* hop_adj;      // adjoint of this step's pressure BC level (edge storage)
  const double* un_adj;       // adjoint of this step's u.n level
  double* hop_old_adj[2];     // adjoints of the earlier BC levels, newest first
  double* un_old_adj[3];      // adjoints of the earlier u.n levels, newest first
  double* Au;                 // adjoint of the step's velocity (Fourier), components
  double* Av;
  double* Aw;                 // null in 2D
  double* ANx;                // adjoint of the step's nonlinear terms, x and y
  double* ANy;
  int Je;
  double alpha[4];
  double invdt, nu, beta;
  int Jx;
  double ex[3];
};
size_t adj_hopbc_smem(const DevGeom& g);
cudaError_t adj_hopbc(const DevGeom& g, const HopbcAdjArgs& a, cudaStream_t st);

}  // namespace stx
