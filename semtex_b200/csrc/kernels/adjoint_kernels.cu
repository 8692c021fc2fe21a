// Kernels of the discrete adjoint of the DNS step (Cartesian).
//
// Each kernel applies the exact transpose of a forward kernel of
// dns_kernels.cu (same element derivative, same quadrature and geometric
// factors, same plane layout), so that the adjoint of a step is the
// transpose of the step the forward path computes, to round-off:
//
//   element gradient      Element::grad        src/element.cpp:521-565
//   Fourier z-derivative  AuxField::gradient(2) src/auxfield.cpp:651-672
//   nonlinear terms       dns/nonlinear.cpp:38-190, 198-381 (linearised
//                         at the recorded velocity)
//   high-order pressure   BCmgr::maintainFourier / evaluateCNBCp,
//   BCs                   src/bcmgr.cpp:1036-1331, Edge::curlCurl
//                         src/edge.cpp:110-256
//
// The element kernels run one warp per (element, plane), kPlanes planes of
// one element per block, as the forward element kernels do.
#include "adjoint_kernels.cuh"
#include "elemderiv.cuh"
#include "launch.hpp"

namespace stx {

namespace {

constexpr int kPlanes = 8;    // planes (warps) per block
constexpr int kThreads = 32 * kPlanes;

// Transposed element derivative at node t = (a, b): with sr = (dr/dx_dir) v
// and ss = (ds/dx_dir) v staged (row-major np x np),
//   (d/dx_dir)^T v [a][b] = sum_j D[j][b] sr[a][j] + sum_i D[i][a] ss[i][b],
// the transpose of elem_deriv's  rx (u D^T) + sx (D u).
__device__ __forceinline__ double elem_deriv_t(const double* sr, const double* ss, const double* sD, int np, int t) {
  const int a = t / np, b = t - (t / np) * np;
  double v = 0.0;
  for (int k = 0; k < np; ++k) {
    v = fma(sD[k * np + b], sr[a * np + k], v);
    v = fma(sD[k * np + a], ss[k * np + b], v);
  }
  return v;
}

__device__ __forceinline__ double zderiv(const double* a, int k, size_t x, int plane_size, double beta) {
  if (k < 2) return 0.0;
  const int m = k >> 1;
  if (k & 1) return beta * m * a[static_cast<size_t>(k - 1) * plane_size + x];
  return -beta * m * a[static_cast<size_t>(k + 1) * plane_size + x];
}

// Stage D and return this warp's plane (-1 past the last) and its area of
// `fields` element planes.
__device__ __forceinline__ int warp_plane(const DevGeom& g, double* sm, int fields, double*& ws) {
  for (int q = threadIdx.x; q < g.np * g.np; q += blockDim.x) sm[q] = g.D[q];
  __syncthreads();
  const int w = threadIdx.x >> 5;
  ws = sm + g.np * g.np + static_cast<size_t>(w) * fields * g.npnp;
  const int k = blockIdx.y * kPlanes + w;
  return k < g.nz ? k : -1;
}

__global__ void k_adj_mass(DevGeom g, const double* in, double* io, int mode) {  // in may be io
  const size_t nn = static_cast<size_t>(g.nel) * g.npnp, n = nn * g.nz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nn, q = i - k * nn, x = k * g.plane_size + q;
    io[x] = mode ? in[x] / g.Q4[q] : in[x] * g.Q4[q];
  }
}

__global__ void k_adj_weights(DevGeom g, double* __restrict__ io, double w0, double w1, double wc) {
  const size_t nn = static_cast<size_t>(g.nel) * g.npnp, n = nn * g.nz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nn, x = k * g.plane_size + (i - k * nn);
    io[x] *= k == 0 ? w0 : (k == 1 ? w1 : wc);
  }
}

__global__ void k_adj_fold2(DevGeom g, double* __restrict__ io) {
  const size_t n = static_cast<size_t>(g.nel) * g.npnp;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    io[i] += io[g.plane_size + i];
    io[g.plane_size + i] = 0.0;
  }
}

__global__ void k_adj_grad_z(DevGeom g, const double* __restrict__ in, double* __restrict__ out, double s,
                             double beta) {
  const size_t nn = static_cast<size_t>(g.nel) * g.npnp, n = nn * g.nz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nn, q = i - k * nn;
    out[k * g.plane_size + q] += s * zderiv(in, static_cast<int>(k), q, g.plane_size, beta);
  }
}

__global__ void k_adj_product2(DevGeom g, const double* __restrict__ U2, const double* __restrict__ Ui,
                               const double* __restrict__ Z, double* Ai, double* A2) {
  const size_t nn = static_cast<size_t>(g.nel) * g.npnp, n = nn * g.nz;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t k = i / nn, x = k * g.plane_size + (i - k * nn);
    const double z = Z[x];
    Ai[x] += U2[x] * z;  // Ai and A2 may be the same array: both terms land
    A2[x] += Ui[x] * z;
  }
}

__global__ void k_adj_grad_t(DevGeom g, const double* __restrict__ in, double* __restrict__ out, int dir,
                             double s) {
  extern __shared__ double sm[];
  double* ws;
  const int k = warp_plane(g, sm, 2, ws);
  if (k < 0) return;
  const int e = blockIdx.x, ln = threadIdx.x & 31, nn = g.npnp;
  double* sr = ws;
  double* ss = ws + nn;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn;
  const double* fr = dir == 0 ? g.drdx : g.drdy;
  const double* fs = dir == 0 ? g.dsdx : g.dsdy;
  for (int t = ln; t < nn; t += 32) {
    const double v = in[base + t];
    const int q = e * nn + t;
    sr[t] = fr[q] * v;
    ss[t] = fs[q] * v;
  }
  __syncwarp();
  for (int t = ln; t < nn; t += 32) out[base + t] += s * elem_deriv_t(sr, ss, sm, g.np, t);
}

__global__ void __launch_bounds__(kThreads) k_adj_nonlinear(DevGeom g, NlAdjArgs a) {
  extern __shared__ double sm[];
  double* ws;
  const int k = warp_plane(g, sm, 8, ws);
  if (k < 0) return;
  const int np = g.np, nn = g.npnp, e = blockIdx.x, ln = threadIdx.x & 31;
  double* sUi = ws;
  double* sP = sUi + nn;
  double* Hr = sP + nn;
  double* Hs = Hr + nn;
  double* G0r = Hs + nn;
  double* G0s = G0r + nn;
  double* G1r = G0s + nn;
  double* G1s = G1r + nn;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn;
  const bool cons = a.cb != 0.0;
  for (int t = ln; t < nn; t += 32) {
    const int q = e * nn + t;
    const double rx = g.drdx[q], ry = g.drdy[q], sx = g.dsdx[q], sy = g.dsdy[q];
    const double p = a.Pb[base + t];
    const double u0 = a.U0[base + t], u1 = a.U1[base + t];
    sUi[t] = a.Ui[base + t];
    sP[t] = p;
    const double av = a.cw * p;
    Hr[t] = (rx * u0 + ry * u1) * av;
    Hs[t] = (sx * u0 + sy * u1) * av;
    if (cons) {
      const double bv = a.cb * p;
      G0r[t] = rx * bv;
      G0s[t] = sx * bv;
      G1r[t] = ry * bv;
      G1s[t] = sy * bv;
    }
  }
  __syncwarp();
  for (int t = ln; t < nn; t += 32) {
    const int i = t / np, j = t - i * np;
    double ur = 0.0, us = 0.0;  // reference derivatives of U_i (elem_deriv)
    for (int kk = 0; kk < np; ++kk) {
      ur = fma(sUi[i * np + kk], sm[j * np + kk], ur);
      us = fma(sm[i * np + kk], sUi[kk * np + j], us);
    }
    const int q = e * nn + t;
    const double dx = ur * g.drdx[q] + us * g.dsdx[q];
    const double dy = ur * g.drdy[q] + us * g.dsdy[q];
    const double av = a.cw * sP[t];
    const double ui = sUi[t];
    const double u0 = a.U0[base + t], u1 = a.U1[base + t];
    // convective part  -(U0 dUi/dx + U1 dUi/dy + U2 Tc)
    double d0 = -av * dx, d1 = -av * dy;
    double di = -elem_deriv_t(Hr, Hs, sm, np, t);
    double d2 = 0.0;
    if (a.A2 && a.Tc) d2 = -av * a.Tc[base + t];
    // conservative part  -(d(Ui U0)/dx + d(Ui U1)/dy)
    if (cons) {
      const double G0 = elem_deriv_t(G0r, G0s, sm, np, t);
      const double G1 = elem_deriv_t(G1r, G1s, sm, np, t);
      d0 -= ui * G0;
      d1 -= ui * G1;
      di -= u0 * G0 + u1 * G1;
    }
    if (a.Ai == a.A0) d0 += di;
    else if (a.Ai == a.A1) d1 += di;
    else d2 += di;
    a.A0[base + t] += d0;
    a.A1[base + t] += d1;
    if (a.A2) a.A2[base + t] += d2;
    if (a.Tcb) a.Tcb[base + t] = -av * a.U2[base + t];
    if (a.Bz) a.Bz[base + t] = a.cb * sP[t];
  }
}

// One block per (high-order edge h, Fourier mode m), as k_hopbc.  Per
// (plane, knot): the adjoint of the knot's pressure BC value (from the
// pressure solve of the adjoint, sp, and the BC weight) and of the level
// hv = -d(u.n)/dt + n.N - nu curlcurl(u).n; the parts of hv and u.n that
// are pointwise land at once, the curl curl seeds go to shared memory and
// are spread over the element by the transposed derivatives.
__global__ void k_adj_hopbc(DevGeom g, HopbcAdjArgs a) {
  extern __shared__ double sm[];
  const int np = g.np, nn = g.npnp;
  const int h = blockIdx.x, m = blockIdx.y;
  const int e = a.elmt[h], side = a.side[h];
  const int nplane = m ? 2 : 1;
  const bool z3 = a.Aw != nullptr && m > 0;
  const double bk = m * a.beta;
  double* sD = sm;
  // per plane p, 11 element arrays at f + 11 nn p:
  // Cx Cy R1 S1 R2 S2 Om Wrx Wsx Wry Wsy
  double* f = sm + np * np;
  for (int q = threadIdx.x; q < np * np; q += blockDim.x) sD[q] = g.D[q];
  for (int q = threadIdx.x; q < nplane * 2 * nn; q += blockDim.x) {
    const int p = q / (2 * nn), t = q - p * 2 * nn;
    f[11 * nn * p + t] = 0.0;  // Cx and Cy of plane p
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * np; q += blockDim.x) {
    const int p = q / np, r = q - p * np;
    const int k = m ? 2 * m + p : 0;
    const int t = side_node(side, r, np);
    const double nxv = a.nx[h * np + r], nyv = a.ny[h * np + r];
    const size_t pos = static_cast<size_t>(k) * a.nh * np + static_cast<size_t>(h) * np + r;
    const size_t x = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn + t;
    const double lb = -a.edge_area[static_cast<size_t>(a.line[h]) * np + r] * a.sp[x];
    const double hb = a.ex[0] * lb + a.hop_adj[pos];
    for (int o = 0; o + 1 < a.Jx; ++o) a.hop_old_adj[o][pos] += a.ex[o + 1] * lb;
    double ub = a.un_adj[pos];
    if (a.Je) {
      ub += -a.invdt * a.alpha[0] * hb;
      for (int o = 0; o < a.Je; ++o) a.un_old_adj[o][pos] += -a.invdt * a.alpha[o + 1] * hb;
    }
    atomicAdd(&a.ANx[x], nxv * hb);
    atomicAdd(&a.ANy[x], nyv * hb);
    const double cxb = -a.nu * nxv * hb, cyb = -a.nu * nyv * hb;
    atomicAdd(&a.Au[x], nxv * ub + (z3 ? bk * bk * cxb : 0.0));
    atomicAdd(&a.Av[x], nyv * ub + (z3 ? bk * bk * cyb : 0.0));
    double* fp = f + 11 * nn * p;
    fp[t] += cxb;  // a knot is visited once per plane; += keeps the zero fill
    fp[nn + t] += cyb;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    double* fp = f + 11 * nn * p;
    const int i = e * nn + t;
    const double rx = g.drdx[i], ry = g.drdy[i], sx = g.dsdx[i], sy = g.dsdy[i];
    const double cx = fp[t], cy = fp[nn + t];
    // curl curl: cx = d(om)/dy, cy = -d(om)/dx  =>  om_b = Dy^T cx - Dx^T cy
    fp[2 * nn + t] = ry * cx - rx * cy;
    fp[3 * nn + t] = sy * cx - sx * cy;
    // beta k terms of W: Dx^T cx + Dy^T cy
    fp[4 * nn + t] = rx * cx + ry * cy;
    fp[5 * nn + t] = sx * cx + sy * cy;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    double* fp = f + 11 * nn * p;
    fp[6 * nn + t] = elem_deriv_t(fp + 2 * nn, fp + 3 * nn, sD, np, t);
    if (z3) {
      // Re plane (p = 0): cx -= bk dW_im/dx ...; Im plane: += bk dW_re/dx
      const double wv = elem_deriv_t(fp + 4 * nn, fp + 5 * nn, sD, np, t);
      const int ko = 2 * m + (1 - p);
      const size_t xo = static_cast<size_t>(ko) * g.plane_size + static_cast<size_t>(e) * nn + t;
      atomicAdd(&a.Aw[xo], (p == 0 ? -bk : bk) * wv);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    double* fp = f + 11 * nn * p;
    const int i = e * nn + t;
    const double om = fp[6 * nn + t];
    fp[7 * nn + t] = g.drdx[i] * om;
    fp[8 * nn + t] = g.dsdx[i] * om;
    fp[9 * nn + t] = g.drdy[i] * om;
    fp[10 * nn + t] = g.dsdy[i] * om;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    const double* fp = f + 11 * nn * p;
    const int k = m ? 2 * m + p : 0;
    const size_t x = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn + t;
    // om = dV/dx - dU/dy
    atomicAdd(&a.Av[x], elem_deriv_t(fp + 7 * nn, fp + 8 * nn, sD, np, t));
    atomicAdd(&a.Au[x], -elem_deriv_t(fp + 9 * nn, fp + 10 * nn, sD, np, t));
  }
}

inline dim3 plane_grid(const DevGeom& g) { return dim3(g.nel, (g.nz + kPlanes - 1) / kPlanes); }
inline size_t plane_smem(const DevGeom& g, int fields) {
  return sizeof(double) * (static_cast<size_t>(g.np) * g.np + static_cast<size_t>(kPlanes) * fields * g.npnp);
}
inline unsigned stream_blocks(const DevGeom& g) {
  const size_t n = static_cast<size_t>(g.nel) * g.npnp * g.nz;
  size_t b = (n + 255) / 256;
  return static_cast<unsigned>(b > 148 * 32 ? 148 * 32 : (b ? b : 1));
}

}  // namespace

cudaError_t adj_mass(const DevGeom& g, const double* in, double* io, int mode, cudaStream_t st) {
  k_adj_mass<<<stream_blocks(g), 256, 0, st>>>(g, in, io, mode);
  return cudaGetLastError();
}

cudaError_t adj_plane_weights(const DevGeom& g, double* io, double w0, double w1, double wc, cudaStream_t st) {
  k_adj_weights<<<stream_blocks(g), 256, 0, st>>>(g, io, w0, w1, wc);
  return cudaGetLastError();
}

cudaError_t adj_fold_nz2(const DevGeom& g, double* io, cudaStream_t st) {
  k_adj_fold2<<<stream_blocks(g), 256, 0, st>>>(g, io);
  return cudaGetLastError();
}

cudaError_t adj_grad_t(const DevGeom& g, const double* in, double* out, int dir, double s, cudaStream_t st) {
  if (g.npnp > 32 * 8) return cudaErrorInvalidValue;
  const size_t sh = plane_smem(g, 2);
  raise_smem_limit(reinterpret_cast<const void*>(k_adj_grad_t), sh);
  k_adj_grad_t<<<plane_grid(g), kThreads, sh, st>>>(g, in, out, dir, s);
  return cudaGetLastError();
}

cudaError_t adj_grad_z_acc(const DevGeom& g, const double* in, double* out, double s, double beta,
                           cudaStream_t st) {
  k_adj_grad_z<<<stream_blocks(g), 256, 0, st>>>(g, in, out, s, beta);
  return cudaGetLastError();
}

cudaError_t adj_nonlinear(const DevGeom& g, const NlAdjArgs& a, cudaStream_t st) {
  if (g.npnp > 32 * 8) return cudaErrorInvalidValue;
  const size_t sh = plane_smem(g, 8);
  raise_smem_limit(reinterpret_cast<const void*>(k_adj_nonlinear), sh);
  k_adj_nonlinear<<<plane_grid(g), kThreads, sh, st>>>(g, a);
  return cudaGetLastError();
}

cudaError_t adj_product2(const DevGeom& g, const double* U2, const double* Ui, const double* Z, double* Ai,
                         double* A2, cudaStream_t st) {
  k_adj_product2<<<stream_blocks(g), 256, 0, st>>>(g, U2, Ui, Z, Ai, A2);
  return cudaGetLastError();
}

size_t adj_hopbc_smem(const DevGeom& g) { return sizeof(double) * (g.np * g.np + 22 * g.npnp); }

cudaError_t adj_hopbc(const DevGeom& g, const HopbcAdjArgs& a, cudaStream_t st) {
  if (a.nh == 0) return cudaSuccess;
  const int nmodes = g.nz > 1 ? g.nz / 2 : 1;
  const size_t sh = adj_hopbc_smem(g);
  raise_smem_limit(reinterpret_cast<const void*>(k_adj_hopbc), sh);
  k_adj_hopbc<<<dim3(a.nh, nmodes), 128, sh, st>>>(g, a);
  return cudaGetLastError();
}

}  // namespace stx
