// Body-forcing kernels of the DNS nonlinear terms (dns/fieldforce.cpp).
//
// The reference sums the force of every active class into a scratch field,
// one field operation per term, then adds the scratch field to N
// (FieldForce::addPhysical, dns/fieldforce.cpp:75-107).  Here one pass per
// component reads each input once and keeps the force in a register: the
// same terms, added in the same order.
#include "force.cuh"

namespace stx {

namespace {

inline unsigned point_blocks(size_t n) {
  const size_t b = (n + 255) / 256;
  return static_cast<unsigned>(b > 148 * 16 ? 148 * 16 : (b ? b : 1));
}

// com-th component of a x X, X = (x, y, z) (Element::crossXPlus,
// src/element.cpp:1752-1785), added to f.
__device__ __forceinline__ double cross_x_plus(double f, int com, const double* a, double x, double y, double z) {
  if (com == 0) return (f + a[1] * z) - a[2] * y;
  if (com == 1) return (f + a[2] * x) - a[0] * z;
  return (f + a[0] * y) - a[1] * x;
}

// com-th component of a x b added to f (AuxField::crossProductPlus,
// src/auxfield.cpp:325-383).  With two components (2-D) the reference adds
// -2 a_z b_y and 2 a_z b_x, which is what this returns there.
__device__ __forceinline__ double cross_plus(double f, int com, int ncom, const double* a, const double* b) {
  if (ncom == 2) {
    if (com == 0) return f + (-2.0 * a[2]) * b[1];
    return f + (2.0 * a[2]) * b[0];
  }
  const int c0 = com == 0 ? 1 : com == 1 ? 2 : 0;
  const int c1 = com == 0 ? 2 : com == 1 ? 0 : 1;
  return (f + a[c0] * b[c1]) - a[c1] * b[c0];
}

__global__ void k_force(ForceArgs a) {
  const size_t n = static_cast<size_t>(a.nzl) * a.nplane;
  for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(q / a.nplane);
    const int i = static_cast<int>(q - static_cast<size_t>(k) * a.nplane);
    const size_t p = static_cast<size_t>(k) * a.plane_size + i;
    double u[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < a.ncom; ++c) u[c] = a.U[c][p];
    const double uc = u[a.com];
    double f = 0.0;
    if (a.mask) f = (a.uref[p] - uc) * a.mask[p];
    if (a.coriolis) {
      if (a.coriolis == 2) {
        const double x = a.x[i], y = a.y[i], z = k * a.dz;
        f = cross_x_plus(f, a.com, a.dodt, x, y, z);
        double w[3] = {0.0, 0.0, 0.0};  // (-Omega) x X
        for (int c = 0; c < a.ncom; ++c) w[c] = cross_x_plus(0.0, c, a.mo, x, y, z);
        f = cross_plus(f, a.com, a.ncom, a.o, w);
      }
      f = cross_plus(f, a.com, a.ncom, a.m2o, u);
    }
    if (a.steady) f += a.steady[p];
    if (a.moda) f += a.alpha * a.moda[p];
    if (a.st) f += expr_run(a.st, a.nst, a.x[i], a.y[i], k * a.dz, a.t);
    if (a.drag) {
      const double mag = a.ncom == 2 ? sqrt(u[0] * u[0] + u[1] * u[1])
                                     : sqrt(u[2] * u[2] + u[0] * u[0] + u[1] * u[1]);
      f -= (mag * a.drag[p]) * uc;
    }
    if (a.qbar) {
      double qb = a.sfd_init ? uc : a.qbar[p];
      f += -a.chi * uc;
      f += a.chi * qb;
      qb *= 1.0 - a.rate;
      qb += a.rate * uc;
      a.qbar[p] = qb;
    }
    a.N[p] += f;
  }
}

__global__ void k_force_const(double* N, int nplane, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nplane; i += gridDim.x * blockDim.x) N[i] += v;
}

__global__ void k_eval_program(const ExprOp* __restrict__ ops, int nops, double* out, int nzl, int plane_size,
                               int nplane, const double* __restrict__ x, const double* __restrict__ y, double dz,
                               double t) {
  const size_t n = static_cast<size_t>(nzl) * nplane;
  for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(q / nplane);
    const int i = static_cast<int>(q - static_cast<size_t>(k) * nplane);
    out[static_cast<size_t>(k) * plane_size + i] = expr_run(ops, nops, x[i], y[i], k * dz, t);
  }
}

}  // namespace

cudaError_t dns_force_physical(const ForceArgs& a, cudaStream_t st) {
  if (a.ncom < 2 || a.ncom > 3 || a.com < 0 || a.com >= a.ncom || !a.N) return cudaErrorInvalidValue;
  if ((a.mask && !a.uref) || ((a.coriolis == 2 || a.st) && (!a.x || !a.y))) return cudaErrorInvalidValue;
  const size_t n = static_cast<size_t>(a.nzl) * a.nplane;
  k_force<<<point_blocks(n), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t dns_force_const(double* N, int nplane, double v, cudaStream_t st) {
  k_force_const<<<point_blocks(nplane), 256, 0, st>>>(N, nplane, v);
  return cudaGetLastError();
}

cudaError_t eval_program_field(const ExprOp* ops, int nops, double* out, int nzl, int plane_size, int nplane,
                               const double* x, const double* y, double dz, double t, cudaStream_t st) {
  const size_t n = static_cast<size_t>(nzl) * nplane;
  k_eval_program<<<point_blocks(n), 256, 0, st>>>(ops, nops, out, nzl, plane_size, nplane, x, y, dz, t);
  return cudaGetLastError();
}

}  // namespace stx
