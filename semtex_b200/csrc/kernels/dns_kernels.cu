// Device kernels of the DNS velocity-correction step (Cartesian).
//
//   element gradient      Element::grad        src/element.cpp:521-565
//   Fourier z-derivative  AuxField::gradient(2) src/auxfield.cpp:651-672
//   nonlinear terms       skewSymmetric / altSkewSymmetric / convective
//                         dns/nonlinear.cpp:38-190, 198-381, 384-480
//   DSS smoothing         Field::smooth        src/field.cpp:282-327
//   waveProp              dns/integrate.cpp:204-239
//   setPForce, project    dns/integrate.cpp:242-289
//
// Element kernels run one block per (element, plane) with a thread per node;
// the element's plane data, D and the inverse mapping partials are read once
// and the node results are produced in a single pass over the element.
#include "dns_kernels.cuh"

namespace stx {

namespace {

// x (dir 0) or y (dir 1) derivative at node t of the element held in su.
__device__ __forceinline__ double elem_deriv(const DevGeom& g, const double* su, const double* sD, int e,
                                             int t, int dir) {
  const int np = g.np;
  const int i = t / np, j = t - (t / np) * np;
  double ur = 0.0, us = 0.0;
  for (int k = 0; k < np; ++k) {
    ur += su[i * np + k] * sD[j * np + k];  // (u D^T)[i][j] = du/dr
    us += sD[i * np + k] * su[k * np + j];  // (D u)[i][j]   = du/ds
  }
  const int q = e * g.npnp + t;
  return dir == 0 ? ur * g.drdx[q] + us * g.dsdx[q] : ur * g.drdy[q] + us * g.dsdy[q];
}

// Fourier z-derivative of plane k at offset x (planes 0 and 1 are zero).
__device__ __forceinline__ double zderiv(const double* a, int k, size_t x, int plane_size, double beta) {
  if (k < 2) return 0.0;
  const int m = k >> 1;
  if (k & 1) return beta * m * a[static_cast<size_t>(k - 1) * plane_size + x];
  return -beta * m * a[static_cast<size_t>(k + 1) * plane_size + x];
}

__global__ void k_grad_xy(DevGeom g, const double* __restrict__ in, double* __restrict__ out, int dir) {
  extern __shared__ double sm[];
  double* sD = sm;
  double* su = sD + g.np * g.np;
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  for (int q = t; q < g.np * g.np; q += blockDim.x) sD[q] = g.D[q];
  if (t < g.npnp) su[t] = in[base + t];
  __syncthreads();
  if (t < g.npnp) out[base + t] = elem_deriv(g, su, sD, e, t, dir);
}

__global__ void k_grad_z(const double* __restrict__ in, double* __restrict__ out, int nz, int plane_size,
                         double beta) {
  const size_t n = static_cast<size_t>(nz) * plane_size;
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x / plane_size);
    out[x] = zderiv(in, k, x - static_cast<size_t>(k) * plane_size, plane_size, beta);
  }
}

__global__ void k_product(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                          size_t n) {
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[x] = a[x] * b[x];
}

// N = sc * [ conv: -(U0 dUi/dx + U1 dUi/dy + U2 Tc)
//            cons: -(d(Ui U0)/dx + d(Ui U1)/dy + Tk) ] , form 0 skew (sc=1/2,
// both), 1 convective, 2 conservative.  Tc / Tk / U2 may be null (2D).
__global__ void k_nonlinear(DevGeom g, NonlinearArgs a) {
  extern __shared__ double sm[];
  const int npnp = g.npnp;
  double* sD = sm;
  double* sUi = sD + g.np * g.np;
  double* sP0 = sUi + npnp;
  double* sP1 = sP0 + npnp;
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * npnp;
  for (int q = t; q < g.np * g.np; q += blockDim.x) sD[q] = g.D[q];
  double u0 = 0.0, u1 = 0.0, ui = 0.0;
  if (t < npnp) {
    u0 = a.U0[base + t];
    u1 = a.U1[base + t];
    ui = a.Ui[base + t];
    sUi[t] = ui;
    sP0[t] = ui * u0;
    sP1[t] = ui * u1;
  }
  __syncthreads();
  if (t >= npnp) return;
  double conv = 0.0, cons = 0.0;
  if (a.form != 2) {
    conv = -(u0 * elem_deriv(g, sUi, sD, e, t, 0) + u1 * elem_deriv(g, sUi, sD, e, t, 1));
    if (a.U2 && a.Tc) conv -= a.U2[base + t] * a.Tc[base + t];
  }
  if (a.form != 1) {
    cons = -(elem_deriv(g, sP0, sD, e, t, 0) + elem_deriv(g, sP1, sD, e, t, 1));
    if (a.Tk) cons -= a.Tk[base + t];
  }
  double v = a.form == 0 ? 0.5 * (conv + cons) : (a.form == 1 ? conv : cons);
  a.N[base + t] = v;
}

__global__ void k_dss_accum(DevGeom g, DevNumbering N, const double* __restrict__ in, double* __restrict__ ds,
                            int gstride) {
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  if (t >= g.next) return;
  const int node = g.emap[t];
  const double v = g.Q4[e * g.npnp + node] *
                   in[static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp + node];
  atomicAdd(&ds[static_cast<size_t>(k) * gstride + N.btog[e * g.next + t]], v);
}

__global__ void k_dss_insert(DevGeom g, DevNumbering N, double* __restrict__ io, const double* __restrict__ ds,
                             int gstride) {
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  if (t >= g.next) return;
  const int gi = N.btog[e * g.next + t];
  io[static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp + g.emap[t]] =
      ds[static_cast<size_t>(k) * gstride + gi] * N.imass[gi];
}

__global__ void k_combine(CombineArgs a, size_t n) {
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int q = 0; q < a.n; ++q) v += a.c[q] * a.p[q][x];
    a.out[x] = v;
  }
}

// out = (du0/dx + du1/dy + [dz u2]) / dt  (setPForce)
__global__ void k_divergence(DevGeom g, const double* __restrict__ a0, const double* __restrict__ a1,
                             const double* __restrict__ a2, double* __restrict__ out, double inv_dt,
                             double beta) {
  extern __shared__ double sm[];
  double* sD = sm;
  double* s0 = sD + g.np * g.np;
  double* s1 = s0 + g.npnp;
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  for (int q = t; q < g.np * g.np; q += blockDim.x) sD[q] = g.D[q];
  if (t < g.npnp) {
    s0[t] = a0[base + t];
    s1[t] = a1[base + t];
  }
  __syncthreads();
  if (t >= g.npnp) return;
  double v = elem_deriv(g, s0, sD, e, t, 0) + elem_deriv(g, s1, sD, e, t, 1);
  if (a2) v += zderiv(a2, k, base + t - static_cast<size_t>(k) * g.plane_size, g.plane_size, beta);
  out[base + t] = v * inv_dt;
}

// io = alpha * io + b * d p / dx_dir  (dir 0, 1 element; 2 Fourier z; -1 none)
__global__ void k_project(DevGeom g, double* __restrict__ io, const double* __restrict__ p, int dir,
                          double alpha, double b, double beta) {
  extern __shared__ double sm[];
  double* sD = sm;
  double* sp = sD + g.np * g.np;
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  for (int q = t; q < g.np * g.np; q += blockDim.x) sD[q] = g.D[q];
  if (t < g.npnp) sp[t] = p[base + t];
  __syncthreads();
  if (t >= g.npnp) return;
  double v = alpha * io[base + t];
  if (dir == 0 || dir == 1) v += b * elem_deriv(g, sp, sD, e, t, dir);
  if (dir == 2) v += b * zderiv(p, k, base + t - static_cast<size_t>(k) * g.plane_size, g.plane_size, beta);
  io[base + t] = v;
}

inline int elem_threads(const DevGeom& g) {
  const int t = (g.npnp + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

inline unsigned stream_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return static_cast<unsigned>(b > 148 * 32 ? 148 * 32 : (b ? b : 1));
}

}  // namespace

cudaError_t dns_grad_xy(const DevGeom& g, const double* in, double* out, int dir, cudaStream_t st) {
  const size_t shm = sizeof(double) * (g.np * g.np + g.npnp);
  k_grad_xy<<<dim3(g.nel, g.nz), elem_threads(g), shm, st>>>(g, in, out, dir);
  return cudaGetLastError();
}

cudaError_t dns_grad_z(const DevGeom& g, const double* in, double* out, double beta, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  k_grad_z<<<stream_blocks(n), 256, 0, st>>>(in, out, g.nz, g.plane_size, beta);
  return cudaGetLastError();
}

cudaError_t dns_product(const DevGeom& g, const double* a, const double* b, double* out, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  k_product<<<stream_blocks(n), 256, 0, st>>>(a, b, out, n);
  return cudaGetLastError();
}

cudaError_t dns_nonlinear(const DevGeom& g, const NonlinearArgs& a, cudaStream_t st) {
  const size_t shm = sizeof(double) * (g.np * g.np + 3 * g.npnp);
  k_nonlinear<<<dim3(g.nel, g.nz), elem_threads(g), shm, st>>>(g, a);
  return cudaGetLastError();
}

cudaError_t dns_smooth(const DevGeom& g, const DevNumbering& N, double* io, double* work, cudaStream_t st) {
  const int gstride = (N.nglobal + 31) / 32 * 32;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(double) * gstride * static_cast<size_t>(g.nz), st);
  if (e != cudaSuccess) return e;
  const int th = (g.next + 31) / 32 * 32;
  k_dss_accum<<<dim3(g.nel, g.nz), th, 0, st>>>(g, N, io, work, gstride);
  k_dss_insert<<<dim3(g.nel, g.nz), th, 0, st>>>(g, N, io, work, gstride);
  return cudaGetLastError();
}

size_t dns_smooth_workspace_doubles(const DevGeom& g, const DevNumbering& N) {
  return static_cast<size_t>((N.nglobal + 31) / 32 * 32) * g.nz;
}

cudaError_t dns_combine(const DevGeom& g, const CombineArgs& a, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  k_combine<<<stream_blocks(n), 256, 0, st>>>(a, n);
  return cudaGetLastError();
}

cudaError_t dns_divergence(const DevGeom& g, const double* a0, const double* a1, const double* a2, double* out,
                           double dt, double beta, cudaStream_t st) {
  const size_t shm = sizeof(double) * (g.np * g.np + 2 * g.npnp);
  k_divergence<<<dim3(g.nel, g.nz), elem_threads(g), shm, st>>>(g, a0, a1, a2, out, 1.0 / dt, beta);
  return cudaGetLastError();
}

cudaError_t dns_project(const DevGeom& g, double* io, const double* p, int dir, double alpha, double b,
                        double beta, cudaStream_t st) {
  const size_t shm = sizeof(double) * (g.np * g.np + g.npnp);
  k_project<<<dim3(g.nel, g.nz), elem_threads(g), shm, st>>>(g, io, p, dir, alpha, b, beta);
  return cudaGetLastError();
}

}  // namespace stx
