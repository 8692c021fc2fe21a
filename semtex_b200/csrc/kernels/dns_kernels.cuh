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
