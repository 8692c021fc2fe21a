// Device kernels of the DNS velocity-correction step (Cartesian).
//
//   element gradient      Element::grad        src/element.cpp:521-565
//   Fourier z-derivative  AuxField::gradient(2) src/auxfield.cpp:651-672
//   nonlinear terms       skewSymmetric / altSkewSymmetric / convective
//                         dns/nonlinear.cpp:38-190, 198-381, 384-480
//   DSS smoothing         Field::smooth        src/field.cpp:282-327
//   waveProp              dns/integrate.cpp:204-239
//   setPForce, project    dns/integrate.cpp:242-289
//   high-order pressure   BCmgr::maintainFourier / evaluateCNBCp
//   BCs                   src/bcmgr.cpp:1036-1331, src/edge.cpp:110-256
//   modal energy, CFL     AuxField::mode_L2 / CFL, Element::CFL
//                         src/auxfield.cpp:919-947, 1719-1762, src/element.cpp:1207-1250
//
// Element kernels run one warp per (element, plane), kEpPlanes planes of one
// element per block: D is staged once per block, each warp holds its plane's
// element data in its own shared memory (lanes over nodes, a few nodes per
// lane loaded together) and synchronises only with itself.
#include <type_traits>

#include "dns_kernels.cuh"
#include "elemderiv.cuh"
#include "launch.hpp"
#include "ptx.cuh"
#include "twolevel.cuh"

namespace stx {

namespace {

// Fourier z-derivative of plane k at offset x (planes 0 and 1 are zero).
__device__ __forceinline__ double zderiv(const double* a, int k, size_t x, int plane_size, double beta) {
  if (k < 2) return 0.0;
  const int m = k >> 1;
  if (k & 1) return beta * m * a[static_cast<size_t>(k - 1) * plane_size + x];
  return -beta * m * a[static_cast<size_t>(k + 1) * plane_size + x];
}

constexpr int kEpPlanes = 8;  // planes (warps) per block of the element kernels
constexpr int kEpNodes = 8;   // nodes per lane loaded together (np <= 16)

// Block (element, planes [kEpPlanes y, +kEpPlanes)): stage D, return this
// warp's plane (or -1 past the last plane) and its shared-memory area of
// `fields` element planes.
__device__ __forceinline__ int ep_setup(const DevGeom& g, double* sm, int fields, double*& ws) {
  for (int q = threadIdx.x; q < g.np * g.np; q += blockDim.x) sm[q] = g.D[q];
  __syncthreads();
  const int w = threadIdx.x >> 5;
  ws = sm + g.np * g.np + static_cast<size_t>(w) * fields * g.npnp;
  const int k = blockIdx.y * kEpPlanes + w;
  return k < g.nz ? k : -1;
}

// dst[t] = src[t] for the element's nodes (lanes over nodes, loads first).
__device__ __forceinline__ void ep_load(const double* __restrict__ src, double* dst, int npnp) {
  const int ln = threadIdx.x & 31;
  double v[kEpNodes];
#pragma unroll
  for (int u = 0; u < kEpNodes; ++u) {
    const int t = ln + 32 * u;
    v[u] = t < npnp ? src[t] : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kEpNodes; ++u) {
    const int t = ln + 32 * u;
    if (t < npnp) dst[t] = v[u];
  }
}

// The nodes of an ElemMma result fragment held by this lane: f(node, m, n, c)
// for every node (8 m + g, 8 n + 2 t + c) inside the np x np element.
template <int MT, class F>
__device__ __forceinline__ void for_frag_nodes(int np, F&& f) {
  const int ln = threadIdx.x & 31, g8 = ln >> 2, t4 = ln & 3;
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int n = 0; n < MT; ++n)
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int i = 8 * m + g8, j = 8 * n + 2 * t4 + c;
        if (i < np && j < np) f(i * np + j, m, n, c);
      }
}

template <int MT, int KS>
__global__ void k_grad_xy(DevGeom g, const double* __restrict__ in, double* __restrict__ out, int dir) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ double sm[];
  double* su;
  const int k = ep_setup(g, sm, 1, su);
  if (k < 0) return;
  const int e = blockIdx.x, np = g.np;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  ep_load(in + base, su, g.npnp);
  __syncwarp();
  ElemMma<MT, KS> M;
  M.load_d(sm, np);
  double ur[MT][MT][2], us[MT][MT][2];
  M.grad(su, np, ur, us);
  const double* fr = dir == 0 ? g.drdx : g.drdy;
  const double* fs = dir == 0 ? g.dsdx : g.dsdy;
  for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
    const int q = e * g.npnp + t;
    out[base + t] = ur[m][n][c] * fr[q] + us[m][n][c] * fs[q];
  });
}

// One block per (high-order edge h, Fourier mode m): planes 0 (m = 0) or
// 2m, 2m+1.  The element's U, V (W) planes and the vorticity dV/dx - dU/dy
// are staged in shared memory; one thread per (plane, edge knot) forms
//   curl curl u . n   (x = dw/dy, y = -dw/dx, plus the beta k terms of W and
//                      beta^2 k^2 U, V in 3D, Edge::curlCurl),
//   -d(u.n)/dt        (stiffly stable difference of the stored u.n),
//   n . N,
// the new level  hop = -d(u.n)/dt + n.N - nu curlcurl(u).n  and the
// extrapolated pressure BC value  sum_q ex[q] hop_q.  The Nyquist plane is
// never touched (its lines stay zero).
__global__ void k_hopbc(DevGeom g, HopbcArgs a) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ double sm[];
  const int np = g.np, nn = g.npnp;
  const int h = blockIdx.x, m = blockIdx.y;
  const int e = a.elmt[h], side = a.side[h];
  const int nplane = m ? 2 : 1;
  const bool z3 = a.W != nullptr && m > 0;
  double* sD = sm;
  double* f = sm + np * np;  // plane p: U at f + 4 nn p, V +nn, W +2nn, vorticity +3nn
  for (int q = threadIdx.x; q < np * np; q += blockDim.x) sD[q] = g.D[q];
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    const int k = m ? 2 * m + p : 0;
    const size_t x = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn + t;
    double* fp = f + 4 * nn * p;
    fp[t] = a.U[x];
    fp[nn + t] = a.V[x];
    if (z3) fp[2 * nn + t] = a.W[x];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nplane * nn; q += blockDim.x) {
    const int p = q / nn, t = q - p * nn;
    double* fp = f + 4 * nn * p;
    fp[3 * nn + t] = elem_deriv(g, fp + nn, sD, e, t, 0) - elem_deriv(g, fp, sD, e, t, 1);
  }
  __syncthreads();
  if (threadIdx.x >= nplane * np) return;
  const int p = threadIdx.x / np, r = threadIdx.x - p * np;
  int i, j;  // knot r of the side in CCW traverse (row i = s, column j = r)
  switch (side) {
    case 0: i = 0; j = r; break;
    case 1: i = r; j = np - 1; break;
    case 2: i = np - 1; j = np - 1 - r; break;
    default: i = np - 1 - r; j = 0; break;
  }
  const int t = i * np + j;
  const double* fp = f + 4 * nn * p;
  double cx = elem_deriv(g, fp + 3 * nn, sD, e, t, 1);
  double cy = -elem_deriv(g, fp + 3 * nn, sD, e, t, 0);
  if (z3) {
    const double bk = m * a.beta;
    const double* Wo = f + 4 * nn * (1 - p) + 2 * nn;  // W of the other plane of the mode
    if (p == 0) {  // real part: -beta k d(W_im)
      cx -= bk * elem_deriv(g, Wo, sD, e, t, 0);
      cy -= bk * elem_deriv(g, Wo, sD, e, t, 1);
    } else {       // imaginary part: +beta k d(W_re)
      cx += bk * elem_deriv(g, Wo, sD, e, t, 0);
      cy += bk * elem_deriv(g, Wo, sD, e, t, 1);
    }
    cx += bk * bk * fp[t];
    cy += bk * bk * fp[nn + t];
  }
  const int k = m ? 2 * m + p : 0;
  const double nxv = a.nx[h * np + r], nyv = a.ny[h * np + r];
  const size_t pos = static_cast<size_t>(k) * a.nh * np + static_cast<size_t>(h) * np + r;
  const double un = fp[t] * nxv + fp[nn + t] * nyv;
  double hv = 0.0;
  if (a.Je) {
    double w = a.alpha[0] * un;
    for (int q = 0; q < a.Je; ++q) w += a.alpha[q + 1] * a.un_old[q][pos];
    hv = -a.invdt * w;
  }
  const size_t x = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn + t;
  hv += a.Nx[x] * nxv + a.Ny[x] * nyv;
  hv += -a.nu * cx * nxv;
  hv += -a.nu * cy * nyv;
  a.un_new[pos] = un;
  a.hop_new[pos] = hv;
  double v = a.ex[0] * hv;
  for (int q = 0; q + 1 < a.Jx; ++q) v += a.ex[q + 1] * a.hop_old[q][pos];
  a.lines[static_cast<size_t>(k) * a.nline + static_cast<size_t>(a.line[h]) * np + r] = v;
}

// Block sum (kAnaThreads threads) of v into part[slot].
constexpr int kAnaThreads = 256;
__device__ __forceinline__ void block_store(double v, double* part, int slot, bool use_max) {
  __shared__ double red[kAnaThreads / 32];
  for (int o = 16; o; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = use_max ? fmax(v, w) : v + w;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = red[0];
    for (int w = 1; w < kAnaThreads / 32; ++w) t = use_max ? fmax(t, red[w]) : t + red[w];
    part[slot] = t;
  }
}

// Per (block, mode m): sum of Q4 (Re^2 + Im^2) over the block's share of the
// element nodes of mode m (planes 2m, 2m+1; plane 0 alone when nz == 1).
__global__ void __launch_bounds__(kAnaThreads) k_mode_energy(DevGeom g, const double* __restrict__ f,
                                                             double* __restrict__ part) {
  const int m = blockIdx.y;
  const size_t n = static_cast<size_t>(g.nel) * g.npnp;
  const double* re = f + static_cast<size_t>(g.nz > 1 ? 2 * m : 0) * g.plane_size;
  const double* im = g.nz > 1 ? re + g.plane_size : nullptr;
  double s = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double q = g.Q4[i];
    s += q * re[i] * re[i];
    if (im) s += q * im[i] * im[i];
  }
  block_store(s, part, m * gridDim.x + blockIdx.x, false);
}

// Per block: max over plane 0 (the zeroth mode) of |u| / (d (|dr/dx_dir| +
// |ds/dx_dir|)) for dir 0, 1 (Element::CFL), or of |u| for dir 2.
__global__ void __launch_bounds__(kAnaThreads) k_cfl(DevGeom g, const double* __restrict__ u, int dir, double d,
                                                     double* __restrict__ part) {
  const size_t n = static_cast<size_t>(g.nel) * g.npnp;
  double s = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    double v;
    if (dir == 2) {
      v = fabs(u[i]);
    } else {
      const double w = dir == 0 ? d * fabs(g.drdx[i]) + d * fabs(g.dsdx[i]) : d * fabs(g.drdy[i]) + d * fabs(g.dsdy[i]);
      v = fabs(u[i] / w);
    }
    s = fmax(s, v);
  }
  block_store(s, part, blockIdx.x, true);
}

// History-point values (AuxField::probe, src/auxfield.cpp:1621-1700, over
// Element::probe, src/element.cpp:1186-1203): block (point, field); the
// point's interpolants is (rows) and ir (columns) and Fourier coefficients
// c_k in w[point][2 np + nz], so that value = sum_k c_k is^T F_k ir on the
// point's element (c_0 = 1, c_1 = cos(nz/2 beta z), 2 cos / -2 sin of
// k beta z on the Re / Im planes of mode k).
__global__ void __launch_bounds__(kAnaThreads) k_probe(DevGeom g, ProbeArgs a) {
  const int p = blockIdx.x, f = blockIdx.y;
  const int np = g.np, nn = g.npnp;
  const double* w = a.w + static_cast<size_t>(p) * (2 * np + a.nzc);
  const double* is = w;
  const double* ir = w + np;
  const double* c = w + 2 * np;
  const double* src = a.f[f] + static_cast<size_t>(a.elmt[p]) * nn;
  double v = 0.0;
  for (int q = threadIdx.x; q < a.nzc * nn; q += blockDim.x) {
    const int k = q / nn, t = q - k * nn;
    const int i = t / np, j = t - i * np;
    v += c[k] * is[i] * ir[j] * src[static_cast<size_t>(k) * g.plane_size + t];
  }
  block_store(v, a.out, p * a.nf + f, false);
}

// Forces on the wall edges (Edge::normTraction / tangTraction / scalarFlux,
// src/edge.cpp:259-378, with Element::sideGrad, :621-700 of
// src/element.cpp): one warp per edge on plane 0 (the mean mode); per edge
// out[5 e ..] = sum of n p area (x, y), of the viscous traction sums
// (2 ux nx + uy ny + vx ny, uy nx + 2 vy ny + vx nx) area and of
// (wx nx + wy ny) area.  The gradients are the element's at the side nodes.
__global__ void __launch_bounds__(32) k_wall_forces(DevGeom g, WallArgs a) {
  const int b = blockIdx.x, ln = threadIdx.x;
  const int np = g.np, nn = g.npnp;
  const int e = a.elmt[b];
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (ln < np) {
    const int t = a.node[b * np + ln];
    const int i = t / np, j = t - i * np;
    const size_t o = static_cast<size_t>(e) * nn;
    const double nx = a.nx[b * np + ln], ny = a.ny[b * np + ln], area = a.area[b * np + ln];
    auto grad = [&](const double* f, double& fx, double& fy) {
      double dr = 0.0, ds = 0.0;
      for (int k = 0; k < np; ++k) {
        dr += g.D[j * np + k] * f[o + i * np + k];
        ds += g.D[i * np + k] * f[o + k * np + j];
      }
      fx = g.drdx[o + t] * dr + g.dsdx[o + t] * ds;
      fy = g.drdy[o + t] * dr + g.dsdy[o + t] * ds;
    };
    const double pv = a.p[o + t];
    acc[0] = nx * pv * area;
    acc[1] = ny * pv * area;
    double ux, uy, vx, vy;
    grad(a.u, ux, uy);
    grad(a.v, vx, vy);
    acc[2] = (2.0 * ux * nx + uy * ny) * area + vx * ny * area;
    acc[3] = uy * nx * area + (2.0 * vy * ny + vx * nx) * area;
    if (a.w) {
      double wx, wy;
      grad(a.w, wx, wy);
      acc[4] = (wx * nx + wy * ny) * area;
    }
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    double v = acc[q];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (ln == 0) a.out[5 * b + q] = v;
  }
}

// Wall tractions (Field::traction, src/field.cpp:533-593, over
// Edge::traction, src/edge.cpp:381-540): block (edge b, mode m), one lane
// per side node.  Mode 0 (plane 0; plane 1 left zero): n = p,
// t = -mu [(-2 ux nx ny - uy ny^2 + uy nx^2) + (2 vy nx ny - vx ny^2 + vx nx^2)],
// s = -mu (wx nx + wy ny).  Mode m > 0, planes 2m (Re), 2m + 1 (Im): n and t
// of each part alike, s_Re = -mu ((wx - bk u_Im) nx + (wy - bk v_Im) ny),
// s_Im = -mu ((wx + bk u_Re) nx + (wy + bk v_Re) ny) with the w gradients
// of the same part and bk = m BETA.
__global__ void __launch_bounds__(32) k_wall_traction(DevGeom g, TractionArgs a) {
  const int b = blockIdx.x, m = blockIdx.y, ln = threadIdx.x;
  const int np = g.np, nn = g.npnp;
  if (ln >= np) return;
  const int t = a.node[b * np + ln];
  const int i = t / np, j = t - i * np;
  const size_t o = static_cast<size_t>(a.elmt[b]) * nn;
  const double nx = a.nx[b * np + ln], ny = a.ny[b * np + ln];
  auto grad = [&](const double* f, double& fx, double& fy) {
    double dr = 0.0, ds = 0.0;
    for (int k = 0; k < np; ++k) {
      dr += g.D[j * np + k] * f[o + i * np + k];
      ds += g.D[i * np + k] * f[o + k * np + j];
    }
    fx = g.drdx[o + t] * dr + g.dsdx[o + t] * ds;
    fy = g.drdy[o + t] * dr + g.dsdy[o + t] * ds;
  };
  auto tang = [&](const double* U, const double* V) {
    double ux, uy, vx, vy;
    grad(U, ux, uy);
    grad(V, vx, vy);
    return (-2.0 * ux * nx * ny - uy * ny * ny + uy * nx * nx) + (2.0 * vy * nx * ny - vx * ny * ny + vx * nx * nx);
  };
  const int q = b * np + ln;
  const size_t ps = g.plane_size;
  if (m == 0) {
    double* o0 = a.out;
    o0[q] = a.p[o + t];
    o0[a.nline + q] = -a.mu * tang(a.u, a.v);
    double sv = 0.0;
    if (a.w) {
      double wx, wy;
      grad(a.w, wx, wy);
      sv = -a.mu * (wx * nx + wy * ny);
    }
    o0[2 * a.nline + q] = sv;
    return;
  }
  const double bk = m * a.beta;
  const size_t re = 2 * m * ps, im = re + ps;
  double* orr = a.out + static_cast<size_t>(2 * m) * a.npad;
  double* oi = orr + a.npad;
  orr[q] = a.p[re + o + t];
  oi[q] = a.p[im + o + t];
  orr[a.nline + q] = -a.mu * tang(a.u + re, a.v + re);
  oi[a.nline + q] = -a.mu * tang(a.u + im, a.v + im);
  double wx, wy;
  grad(a.w + re, wx, wy);
  orr[2 * a.nline + q] = -a.mu * ((wx - bk * a.u[im + o + t]) * nx + (wy - bk * a.v[im + o + t]) * ny);
  grad(a.w + im, wx, wy);
  oi[2 * a.nline + q] = -a.mu * ((wx + bk * a.u[re + o + t]) * nx + (wy + bk * a.v[re + o + t]) * ny);
}

__global__ void k_grad_z(const double* __restrict__ in, double* __restrict__ out, int nz, int plane_size,
                         double beta) {
  pdl_trigger();
  pdl_wait();
  const size_t n = static_cast<size_t>(nz) * plane_size;
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(x / plane_size);
    out[x] = zderiv(in, k, x - static_cast<size_t>(k) * plane_size, plane_size, beta);
  }
}

__global__ void k_product(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                          size_t n) {
  pdl_trigger();
  pdl_wait();
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[x] = a[x] * b[x];
}

// N = sc * [ conv: -(U0 dUi/dx + U1 dUi/dy + U2 Tc)
//            cons: -(d(Ui U0)/dx + d(Ui U1)/dy + Tk) ] , form 0 skew (sc=1/2,
// both), 1 convective, 2 conservative.  Tc / Tk / U2 may be null (2D).  The
// element derivatives run on the FP64 tensor cores (ElemMma), the products
// Ui U0, Ui U1 staged in shared memory first.
template <int MT, int KS>
__global__ void __launch_bounds__(32 * kEpPlanes, 2) k_nonlinear(DevGeom g, NonlinearArgs a) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ double sm[];
  double* ws;
  const int k = ep_setup(g, sm, 5, ws);
  if (k < 0) return;
  const int np = g.np, npnp = g.npnp, e = blockIdx.x, ln = threadIdx.x & 31;
  double* sUi = ws;
  double* sP0 = sUi + npnp;
  double* sP1 = sP0 + npnp;
  double* sU0 = sP1 + npnp;
  double* sU1 = sU0 + npnp;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * npnp;
  ep_load(a.U0 + base, sU0, npnp);
  ep_load(a.U1 + base, sU1, npnp);
  ep_load(a.Ui + base, sUi, npnp);
  __syncwarp();
  for (int t = ln; t < npnp; t += 32) {
    sP0[t] = sUi[t] * sU0[t];
    sP1[t] = sUi[t] * sU1[t];
  }
  __syncwarp();
  const bool conv_on = a.form != 2, cons_on = a.form != 1;
  const double wconv = a.form == 0 ? 0.5 : 1.0, wcons = a.form == 0 ? 0.5 : 1.0;
  ElemMma<MT, KS> M;
  M.load_d(sm, np);
  double acc[MT][MT][2];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int n = 0; n < MT; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
  double ur[MT][MT][2], us[MT][MT][2];
  if (conv_on) {  // -(U0 dUi/dx + U1 dUi/dy + U2 Tc)
    M.grad(sUi, np, ur, us);
    for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
      const int q = e * npnp + t;
      const double dx = ur[m][n][c] * g.drdx[q] + us[m][n][c] * g.dsdx[q];
      const double dy = ur[m][n][c] * g.drdy[q] + us[m][n][c] * g.dsdy[q];
      double v = -(sU0[t] * dx + sU1[t] * dy);
      if (a.U2 && a.Tc) v -= a.U2[base + t] * a.Tc[base + t];
      acc[m][n][c] += wconv * v;
    });
  }
  if (cons_on) {  // -(d(Ui U0)/dx + d(Ui U1)/dy + Tk)
    M.grad(sP0, np, ur, us);
    for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
      const int q = e * npnp + t;
      acc[m][n][c] -= wcons * (ur[m][n][c] * g.drdx[q] + us[m][n][c] * g.dsdx[q]);
    });
    M.grad(sP1, np, ur, us);
    for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
      const int q = e * npnp + t;
      double v = ur[m][n][c] * g.drdy[q] + us[m][n][c] * g.dsdy[q];
      if (a.Tk) v += a.Tk[base + t];
      acc[m][n][c] -= wcons * v;
    });
  }
  for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) { a.N[base + t] = acc[m][n][c]; });
}

__global__ void k_dss_accum(DevGeom g, DevNumbering N, const double* __restrict__ in, double* __restrict__ ds,
                            int gstride) {
  pdl_trigger();
  pdl_wait();
  const int e = blockIdx.x, k = blockIdx.y * kEpPlanes + (threadIdx.x >> 5), ln = threadIdx.x & 31;
  if (k >= g.nz) return;
  const double* src = in + static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  for (int t = ln; t < g.next; t += 32) {
    const int node = g.emap[t];
    atomicAdd(&ds[static_cast<size_t>(k) * gstride + N.btog[e * g.next + t]], g.Q4[e * g.npnp + node] * src[node]);
  }
}

__global__ void k_dss_insert(DevGeom g, DevNumbering N, double* __restrict__ io, const double* __restrict__ ds,
                             int gstride) {
  pdl_trigger();
  pdl_wait();
  const int e = blockIdx.x, k = blockIdx.y * kEpPlanes + (threadIdx.x >> 5), ln = threadIdx.x & 31;
  if (k >= g.nz) return;
  double* dst = io + static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  for (int t = ln; t < g.next; t += 32) {
    const int gi = N.btog[e * g.next + t];
    dst[g.emap[t]] = ds[static_cast<size_t>(k) * gstride + gi] * N.imass[gi];
  }
}

__global__ void k_combine(CombineArgs a, size_t n) {
  pdl_trigger();
  pdl_wait();
  for (size_t x = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; x < n;
       x += static_cast<size_t>(gridDim.x) * blockDim.x) {
    double v = 0.0;
    for (int q = 0; q < a.n; ++q) v += a.c[q] * a.p[q][x];
    a.out[x] = v;
  }
}

// out = (du0/dx + du1/dy + [dz u2]) / dt  (setPForce), element derivatives
// on the FP64 tensor cores
template <int MT, int KS>
__global__ void k_divergence(DevGeom g, const double* __restrict__ a0, const double* __restrict__ a1,
                             const double* __restrict__ a2, double* __restrict__ out, double inv_dt,
                             double beta) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ double sm[];
  double* ws;
  const int k = ep_setup(g, sm, 2, ws);
  if (k < 0) return;
  const int e = blockIdx.x, np = g.np;
  double* s0 = ws;
  double* s1 = ws + g.npnp;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  ep_load(a0 + base, s0, g.npnp);
  ep_load(a1 + base, s1, g.npnp);
  __syncwarp();
  ElemMma<MT, KS> M;
  M.load_d(sm, np);
  double acc[MT][MT][2], ur[MT][MT][2], us[MT][MT][2];
  M.grad(s0, np, ur, us);
  for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
    const int q = e * g.npnp + t;
    acc[m][n][c] = ur[m][n][c] * g.drdx[q] + us[m][n][c] * g.dsdx[q];
  });
  M.grad(s1, np, ur, us);
  for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
    const int q = e * g.npnp + t;
    double v = acc[m][n][c] + ur[m][n][c] * g.drdy[q] + us[m][n][c] * g.dsdy[q];
    if (a2) v += zderiv(a2, k, base + t - static_cast<size_t>(k) * g.plane_size, g.plane_size, beta);
    out[base + t] = v * inv_dt;
  });
}

// io = alpha * io + b * d p / dx_dir  (dir 0, 1 element, on the FP64 tensor
// cores; 2 Fourier z; -1 none)
template <int MT, int KS>
__global__ void k_project(DevGeom g, double* __restrict__ io, const double* __restrict__ p, int dir,
                          double alpha, double b, double beta) {
  pdl_trigger();
  pdl_wait();
  extern __shared__ double sm[];
  double* sp;
  const int k = ep_setup(g, sm, 1, sp);
  if (k < 0) return;
  const int e = blockIdx.x, ln = threadIdx.x & 31, np = g.np;
  const size_t base = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  if (dir == 0 || dir == 1) {
    ep_load(p + base, sp, g.npnp);
    __syncwarp();
    ElemMma<MT, KS> M;
    M.load_d(sm, np);
    double ur[MT][MT][2], us[MT][MT][2];
    M.grad(sp, np, ur, us);
    const double* fr = dir == 0 ? g.drdx : g.drdy;
    const double* fs = dir == 0 ? g.dsdx : g.dsdy;
    for_frag_nodes<MT>(np, [&](int t, int m, int n, int c) {
      const int q = e * g.npnp + t;
      io[base + t] = alpha * io[base + t] + b * (ur[m][n][c] * fr[q] + us[m][n][c] * fs[q]);
    });
    return;
  }
  for (int t = ln; t < g.npnp; t += 32) {
    double v = alpha * io[base + t];
    if (dir == 2) v += b * zderiv(p, k, base + t - static_cast<size_t>(k) * g.plane_size, g.plane_size, beta);
    io[base + t] = v;
  }
}

// Call f(MT, KS) (std::integral_constant arguments) for the ElemMma instance
// that covers np (np <= 16).
template <class F>
cudaError_t mma_dispatch(int np, F&& f) {
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  using I4 = std::integral_constant<int, 4>;
  const int mt = mma_tiles(np), ks = mma_ksteps(np);
  if (mt == 1 && ks == 1) return f(I1{}, I1{});
  if (mt == 1 && ks == 2) return f(I1{}, I2{});
  if (mt == 2 && ks == 3) return f(I2{}, I3{});
  if (mt == 2 && ks == 4) return f(I2{}, I4{});
  return cudaErrorInvalidValue;
}

inline dim3 ep_grid(const DevGeom& g) { return dim3(g.nel, (g.nz + kEpPlanes - 1) / kEpPlanes); }
// the warp-per-plane kernels hold up to 32 * kEpNodes nodes per element
inline bool ep_fits(const DevGeom& g) { return g.npnp <= 32 * kEpNodes; }
constexpr int kEpThreads = 32 * kEpPlanes;
inline size_t ep_smem(const DevGeom& g, int fields) {
  return sizeof(double) * (static_cast<size_t>(g.np) * g.np + static_cast<size_t>(kEpPlanes) * fields * g.npnp);
}

inline unsigned stream_blocks(size_t n) {
  size_t b = (n + 255) / 256;
  return static_cast<unsigned>(b > 148 * 32 ? 148 * 32 : (b ? b : 1));
}

}  // namespace

cudaError_t dns_grad_xy(const DevGeom& g, const double* in, double* out, int dir, cudaStream_t st) {
  if (!ep_fits(g)) return cudaErrorInvalidValue;
  return mma_dispatch(g.np, [&](auto mt_, auto ks_) {
    constexpr int MT = decltype(mt_)::value, KS = decltype(ks_)::value;
    raise_smem_limit(reinterpret_cast<const void*>(k_grad_xy<MT, KS>), ep_smem(g, 1));
    launch_ex(g.pdl != 0, k_grad_xy<MT, KS>, ep_grid(g), dim3(kEpThreads), ep_smem(g, 1), st, g, in, out, dir);
    return cudaGetLastError();
  });
}

cudaError_t dns_grad_z(const DevGeom& g, const double* in, double* out, double beta, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  launch_ex(g.pdl != 0, k_grad_z, dim3(stream_blocks(n)), dim3(256), 0, st, in, out, g.nz, g.plane_size, beta);
  return cudaGetLastError();
}

cudaError_t dns_product(const DevGeom& g, const double* a, const double* b, double* out, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  launch_ex(g.pdl != 0, k_product, dim3(stream_blocks(n)), dim3(256), 0, st, a, b, out, n);
  return cudaGetLastError();
}

cudaError_t dns_nonlinear(const DevGeom& g, const NonlinearArgs& a, cudaStream_t st) {
  if (!ep_fits(g)) return cudaErrorInvalidValue;
  return mma_dispatch(g.np, [&](auto mt_, auto ks_) {
    constexpr int MT = decltype(mt_)::value, KS = decltype(ks_)::value;
    raise_smem_limit(reinterpret_cast<const void*>(k_nonlinear<MT, KS>), ep_smem(g, 5));
    launch_ex(g.pdl != 0, k_nonlinear<MT, KS>, ep_grid(g), dim3(kEpThreads), ep_smem(g, 5), st, g, a);
    return cudaGetLastError();
  });
}

cudaError_t dns_smooth(const DevGeom& g, const DevNumbering& N, double* io, double* work, cudaStream_t st) {
  const int gstride = (N.nglobal + 31) / 32 * 32;
  cudaError_t e = zero_ranges(g.pdl != 0, work, static_cast<size_t>(gstride) * g.nz, nullptr, 0, st);
  if (e != cudaSuccess) return e;
  launch_ex(g.pdl != 0, k_dss_accum, ep_grid(g), dim3(kEpThreads), 0, st, g, N, io, work, gstride);
  launch_ex(g.pdl != 0, k_dss_insert, ep_grid(g), dim3(kEpThreads), 0, st, g, N, io, work, gstride);
  return cudaGetLastError();
}

size_t dns_smooth_workspace_doubles(const DevGeom& g, const DevNumbering& N) {
  return static_cast<size_t>((N.nglobal + 31) / 32 * 32) * g.nz;
}

int dns_analysis_blocks() { return 64; }

cudaError_t dns_mode_energy_partials(const DevGeom& g, const double* f, double* part, cudaStream_t st) {
  const int nmodes = (g.nz + 1) / 2;
  k_mode_energy<<<dim3(dns_analysis_blocks(), nmodes), kAnaThreads, 0, st>>>(g, f, part);
  return cudaGetLastError();
}

cudaError_t dns_cfl_partials(const DevGeom& g, const double* u, int dir, double d, double* part, cudaStream_t st) {
  k_cfl<<<dns_analysis_blocks(), kAnaThreads, 0, st>>>(g, u, dir, d, part);
  return cudaGetLastError();
}

cudaError_t dns_probe(const DevGeom& g, const ProbeArgs& a, cudaStream_t st) {
  if (a.npts <= 0) return cudaSuccess;
  if (a.nf < 1 || a.nf > 8) return cudaErrorInvalidValue;
  k_probe<<<dim3(a.npts, a.nf), kAnaThreads, 0, st>>>(g, a);
  return cudaGetLastError();
}

cudaError_t dns_wall_forces(const DevGeom& g, const WallArgs& a, cudaStream_t st) {
  if (a.nw <= 0) return cudaSuccess;
  if (g.np > 32) return cudaErrorInvalidValue;
  k_wall_forces<<<a.nw, 32, 0, st>>>(g, a);
  return cudaGetLastError();
}

cudaError_t dns_wall_traction(const DevGeom& g, const TractionArgs& a, cudaStream_t st) {
  if (a.nw <= 0) return cudaSuccess;
  if (g.np > 32 || (g.nz > 2 && !a.w)) return cudaErrorInvalidValue;
  k_wall_traction<<<dim3(a.nw, g.nz > 2 ? g.nz / 2 : 1), 32, 0, st>>>(g, a);
  return cudaGetLastError();
}

size_t dns_hopbc_smem(const DevGeom& g) { return sizeof(double) * (g.np * g.np + 8 * g.npnp); }

cudaError_t dns_hopbc(const DevGeom& g, const HopbcArgs& a, cudaStream_t st) {
  if (a.nh == 0) return cudaSuccess;
  if (2 * g.np > 128 || a.Je < 0 || a.Je > 3 || a.Jx < 1 || a.Jx > 3) return cudaErrorInvalidValue;
  const dim3 grid(a.nh, g.nz > 1 ? g.nz / 2 : 1);
  return launch_ex(g.pdl != 0, k_hopbc, grid, dim3(128), dns_hopbc_smem(g), st, g, a);
}

cudaError_t dns_combine(const DevGeom& g, const CombineArgs& a, cudaStream_t st) {
  const size_t n = static_cast<size_t>(g.nz) * g.plane_size;
  launch_ex(g.pdl != 0, k_combine, dim3(stream_blocks(n)), dim3(256), 0, st, a, n);
  return cudaGetLastError();
}

cudaError_t dns_divergence(const DevGeom& g, const double* a0, const double* a1, const double* a2, double* out,
                           double dt, double beta, cudaStream_t st) {
  if (!ep_fits(g)) return cudaErrorInvalidValue;
  return mma_dispatch(g.np, [&](auto mt_, auto ks_) {
    constexpr int MT = decltype(mt_)::value, KS = decltype(ks_)::value;
    raise_smem_limit(reinterpret_cast<const void*>(k_divergence<MT, KS>), ep_smem(g, 2));
    launch_ex(g.pdl != 0, k_divergence<MT, KS>, ep_grid(g), dim3(kEpThreads), ep_smem(g, 2), st, g, a0, a1, a2, out,
              1.0 / dt, beta);
    return cudaGetLastError();
  });
}

cudaError_t dns_project(const DevGeom& g, double* io, const double* p, int dir, double alpha, double b,
                        double beta, cudaStream_t st) {
  if (!ep_fits(g)) return cudaErrorInvalidValue;
  return mma_dispatch(g.np, [&](auto mt_, auto ks_) {
    constexpr int MT = decltype(mt_)::value, KS = decltype(ks_)::value;
    raise_smem_limit(reinterpret_cast<const void*>(k_project<MT, KS>), ep_smem(g, 1));
    launch_ex(g.pdl != 0, k_project<MT, KS>, ep_grid(g), dim3(kEpThreads), ep_smem(g, 1), st, g, io, p, dir, alpha,
              b, beta);
    return cudaGetLastError();
  });
}

}  // namespace stx
