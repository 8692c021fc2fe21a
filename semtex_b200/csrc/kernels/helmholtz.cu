// Condensed direct Helmholtz solve for all Fourier planes of a field.
//
// Device restatement of Field::solve DIRECT (src/field.cpp:598-709):
//   1. essential values g into a globally numbered vector per plane
//      (Field::getEssential, src/field.cpp:1078-1103);
//   2. per (element, plane): F = -(M f + H g) (Field::constrain,
//      src/field.cpp:812-852), boundary-major gather, condensation
//      F_b -= (h_bi h_ii^-1) F_i and direct-stiffness scatter-sum into the
//      boundary RHS (Element::local2globalSumSC, src/element.cpp:326-365);
//   3. natural-BC edge integrals <h, w> (Natural::sum, src/condition.cpp:192);
//   4. banded Cholesky forward / backward solves per mode, Re and Im planes
//      of a mode sharing one factor read (Lapack::pbtrs, src/field.cpp:693);
//   5. per (element, plane): interior recovery u_i = h_ii^-1 F_i -
//      (h_ii^-1 h_ib) u_b (Element::global2localSC, src/element.cpp:368-407)
//      and imposition of essential values (Field::setEssential,
//      src/field.cpp:1106-1124).
#include "helmholtz.cuh"
#include "twolevel.cuh"
#include "ptx.cuh"
#include "element.cuh"
#include "launch.hpp"

#include <algorithm>
#include <vector>

namespace stx {

namespace {

// Plane index k of a locally held mode m and RHS slot r (0 = Re, 1 = Im).
__device__ __forceinline__ int plane_of(int m, int r) { return 2 * m + r; }

// Constrained forcing -(Q4 f + [emask] H g) of element e in boundary-major
// order, left in sF (length npnp).  Uses blockDim.x >= npnp.
__device__ void constrained_forcing(const DevGeom& g, const DevNumbering& N,
                                    const double* __restrict__ fplane,
                                    const double* __restrict__ Gplane, double hcon,
                                    int e, double* su, double* sR, double* sS,
                                    double* sF, const double* sD) {
  const int np = g.np, nn = g.npnp, t = threadIdx.x;
  const int i = t / np, j = t - (t / np) * np;
  double F = 0.0;
  if (t < nn) F = g.Q4[e * nn + t] * fplane[e * nn + t];
  if (N.emask && N.emask[e]) {
    if (t < nn) su[t] = 0.0;
    __syncthreads();
    if (t < g.next) su[g.emap[t]] = Gplane[N.btog[e * g.next + t]];
    __syncthreads();
    double r = 0.0, s = 0.0;
    if (t < nn) {
      for (int k = 0; k < np; ++k) {
        r += su[i * np + k] * sD[j * np + k];  // (u D^T)[i][j]
        s += sD[i * np + k] * su[k * np + j];  // (D u)[i][j]
      }
      const double q1 = g.Q1[e * nn + t], q2 = g.Q2[e * nn + t], q3 = g.Q3[e * nn + t];
      sR[t] = q1 * r + q3 * s;
      sS[t] = q2 * s + q3 * r;
    }
    __syncthreads();
    if (t < nn) {
      double h = g.Q4[e * nn + t] * su[t] * hcon;
      for (int k = 0; k < np; ++k) {
        h += sD[k * np + i] * sS[k * np + j];  // D^T S'
        h += sR[i * np + k] * sD[k * np + j];  // R' D
      }
      F += h;
    }
  }
  if (t < nn) sF[g.pmap[t]] = -F;
  __syncthreads();
}

__global__ void k_essential(DevGeom g, DevNumbering N, const double* __restrict__ lines,
                            int nline, double* __restrict__ G, int gstride, int nz, int k0) {
  pdl_trigger();
  pdl_wait();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = k0 + blockIdx.y;
  if (k >= nz || idx >= N.nedge * g.np) return;
  const int b = idx / g.np;
  if (N.edge_kind[b] != 'D') return;
  G[static_cast<size_t>(k) * gstride + N.edge_gid[idx]] = lines[static_cast<size_t>(k) * nline + idx];
}

// y += x over n entries.
__global__ void k_add(double* __restrict__ y, const double* __restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    y[i] += x[i];
}

__global__ void k_natural(DevGeom g, DevNumbering N, const double* __restrict__ lines,
                          int nline, double* __restrict__ R, int rstride, int nz, int k0) {
  pdl_trigger();
  pdl_wait();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = k0 + blockIdx.y;
  if (k >= nz || (nz > 1 && k == 1) || idx >= N.nedge * g.np) return;
  const int b = idx / g.np;
  if (N.edge_kind[b] != 'N') return;
  atomicAdd(&R[static_cast<size_t>(k) * rstride + N.edge_gid[idx]],
            lines[static_cast<size_t>(k) * nline + idx] * N.edge_area[idx]);
}

__global__ void k_condense(DevGeom g, DevNumbering N, DevModal S,
                           const double* __restrict__ F, const double* __restrict__ G,
                           int gstride, double* __restrict__ R, int rstride) {
  extern __shared__ double smem[];
  const int nn = g.npnp;
  double* sD = smem;
  double* su = sD + g.np * g.np;
  double* sR = su + nn;
  double* sS = sR + nn;
  double* sF = sS + nn;
  const int e = blockIdx.x;
  const int k = blockIdx.y;
  if (g.nz > 1 && k == 1) return;  // Nyquist plane is never solved
  const int m = k >> 1;
  for (int t = threadIdx.x; t < g.np * g.np; t += blockDim.x) sD[t] = S.D[t];
  __syncthreads();
  constrained_forcing(g, N, F + static_cast<size_t>(k) * g.plane_size,
                      G ? G + static_cast<size_t>(k) * gstride : nullptr,
                      S.lambda2[m] + S.betak2[m], e, su, sR, sS, sF, sD);
  const int t = threadIdx.x;
  if (t < g.next) {
    const double* hbi = S.hbi + (static_cast<size_t>(m) * S.nfamily + g.family[e]) * g.next * g.nint;
    double v = sF[t];
    const double* row = hbi + static_cast<size_t>(t) * g.nint;
    for (int b = 0; b < g.nint; ++b) v -= row[b] * sF[g.next + b];
    atomicAdd(&R[static_cast<size_t>(k) * rstride + N.btog[e * g.next + t]], v);
  }
}

__global__ void k_recover(DevGeom g, DevNumbering N, DevModal S,
                          const double* __restrict__ F, const double* __restrict__ G,
                          int gstride, const double* __restrict__ R, int rstride,
                          double* __restrict__ U) {
  extern __shared__ double smem[];
  const int nn = g.npnp;
  double* sD = smem;
  double* su = sD + g.np * g.np;
  double* sR = su + nn;
  double* sS = sR + nn;
  double* sF = sS + nn;
  double* sub = sF + nn;
  const int e = blockIdx.x;
  const int k = blockIdx.y;
  if (g.nz > 1 && k == 1) return;
  const int m = k >> 1;
  for (int t = threadIdx.x; t < g.np * g.np; t += blockDim.x) sD[t] = S.D[t];
  __syncthreads();
  const double* Gp = G ? G + static_cast<size_t>(k) * gstride : nullptr;
  constrained_forcing(g, N, F + static_cast<size_t>(k) * g.plane_size, Gp,
                      S.lambda2[m] + S.betak2[m], e, su, sR, sS, sF, sD);
  const int t = threadIdx.x;
  const int nsolve = S.nsolve[m];
  const double* Rp = R + static_cast<size_t>(k) * rstride;
  double* Up = U + static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn;
  if (t < g.next) {
    const int gi = N.btog[e * g.next + t];
    const double ub = gi < nsolve ? Rp[gi] : 0.0;
    sub[t] = ub;
    Up[g.emap[t]] = (N.bmask[e * g.next + t] && Gp) ? Gp[gi] : ub;
  }
  __syncthreads();
  if (t < g.nint) {
    const size_t fm = static_cast<size_t>(m) * S.nfamily + g.family[e];
    const double* hii = S.hii + fm * g.nint * g.nint + static_cast<size_t>(t) * g.nint;
    const double* hbi = S.hbi + fm * g.next * g.nint;
    double v = 0.0;
    for (int c = 0; c < g.nint; ++c) v += hii[c] * sF[g.next + c];
    for (int a = 0; a < g.next; ++a) v -= hbi[static_cast<size_t>(a) * g.nint + t] * sub[a];
    Up[g.emap[g.next + t]] = v;
  }
}


// ---------------------------------------------------------------------------
// Batched element kernels.  One block per (chunk of up to chunk_max elements of
// one geometry family, Fourier mode): the chunk's constrained forcing for the
// mode's Re and Im planes forms the columns of a small dense operand in
// shared memory (column stride padded odd against bank conflicts), and the
// family's condensation matrices are applied to all columns at once as a
// register-tiled GEMM (4 rows x 4 columns per thread), each matrix entry read
// through L1 once per column tile.
// ---------------------------------------------------------------------------

constexpr int kTile = 4;

constexpr int kGather = 4;

// Constrained forcing -(Q4 f + [emask] H g) of the chunk's elements for the
// planes of mode m into columns of sB (column c = slot*cnt + l, row =
// boundary-major node, stride ldb).  The lift term H g is formed one column
// per warp in warp-private scratch (wsc: 3*nn doubles per warp) and skipped
// where the element's essential values are all zero (H 0 = 0).
__device__ void chunk_forcing2(const DevGeom& g, const DevNumbering& N, const double* __restrict__ F,
                               const double* __restrict__ G, int gstride, double hcon, const int* el, int cnt, int m,
                               int nr, double* sB, int ldb, double* wsc, const double* sD, int lift_warps = 8) {
  const int nn = g.npnp, np = g.np;
  // One warp per column (nr <= 2, so slot = col >= cnt), lanes over the
  // element's nodes in natural order: coalesced rows of F and Q4, all loads
  // of a batch issued before its shared-memory stores.
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  for (int col = wp; col < nr * cnt; col += nwp) {
    const int slot = col >= cnt ? 1 : 0, l = col - slot * cnt;
    const int e = __ldg(el + l);
    const double* f = F + static_cast<size_t>(2 * m + slot) * g.plane_size + static_cast<size_t>(e) * nn;
    const double* q = g.Q4 + static_cast<size_t>(e) * nn;
    double* b = sB + col * ldb;
    for (int t0 = ln; t0 < nn; t0 += 32 * kGather) {
      double v[kGather];
      int d[kGather];
#pragma unroll
      for (int u = 0; u < kGather; ++u) {
        const int t = t0 + 32 * u;
        d[u] = t < nn ? __ldg(g.pmap + t) : -1;
        v[u] = t < nn ? -__ldg(q + t) * __ldg(f + t) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kGather; ++u)
        if (d[u] >= 0) b[d[u]] = v[u];
    }
  }
  __syncthreads();
  if (!G) return;
  // warps [0, lift_warps) form the lift, each in its own 3*nn scratch
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31,
            nwarp = min(lift_warps, static_cast<int>(blockDim.x >> 5));
  double* su = wsc + static_cast<size_t>(warp) * 3 * nn;
  double* sR = su + nn;
  double* sS = sR + nn;
  for (int c = warp; warp < nwarp && c < nr * cnt; c += nwarp) {
    const int slot = c / cnt, l = c - slot * cnt;
    const int k = 2 * m + slot;
    const int e = el[l];
    if (!N.emask[e]) continue;  // uniform across the warp
    const double* Gp = G + static_cast<size_t>(k) * gstride;
    for (int q = lane; q < nn; q += 32) su[q] = 0.0;
    __syncwarp();
    bool nonzero = false;
    for (int q = lane; q < g.next; q += 32) {
      const double v = N.bmask[e * g.next + q] ? Gp[N.btog[e * g.next + q]] : 0.0;
      su[g.emap[q]] = v;
      nonzero = nonzero || v != 0.0;
    }
    if (!__any_sync(0xffffffffu, nonzero)) continue;
    __syncwarp();
    for (int q = lane; q < nn; q += 32) {
      const int i = q / np, j = q - (q / np) * np;
      double r = 0.0, s2 = 0.0;
      for (int kk = 0; kk < np; ++kk) {
        r += su[i * np + kk] * sD[j * np + kk];
        s2 += sD[i * np + kk] * su[kk * np + j];
      }
      const double q1 = g.Q1[e * nn + q], q2 = g.Q2[e * nn + q], q3 = g.Q3[e * nn + q];
      sR[q] = q1 * r + q3 * s2;
      sS[q] = q2 * s2 + q3 * r;
    }
    __syncwarp();
    for (int q = lane; q < nn; q += 32) {
      const int i = q / np, j = q - (q / np) * np;
      double h = g.Q4[e * nn + q] * su[q] * hcon;
      for (int kk = 0; kk < np; ++kk) {
        h += sD[kk * np + i] * sS[kk * np + j];
        h += sR[i * np + kk] * sD[kk * np + j];
      }
      sB[c * ldb + g.pmap[q]] -= h;
    }
    __syncwarp();
  }
  __syncthreads();
}

// acc[4][4] += A[r0+ii][k] * B[cb+jj*cs][k], k < K; A row-major (lda) in
// global memory (rows clamped to M-1), B columns in shared memory (ldb).
// Threads of a warp share r0 and take consecutive cb: A reads broadcast, B
// reads hit distinct banks (odd ldb).
__device__ __forceinline__ void tile_gemm(double (&acc)[kTile][kTile], const double* __restrict__ A, int lda,
                                          int M, int r0, const double* B, int ldb, int cb, int cs, int ncol, int K,
                                          int boff) {
  const double* a[kTile];
  const double* b[kTile];
#pragma unroll
  for (int ii = 0; ii < kTile; ++ii) a[ii] = A + static_cast<size_t>(min(r0 + ii, M - 1)) * lda;
#pragma unroll
  for (int jj = 0; jj < kTile; ++jj) b[jj] = B + min(cb + jj * cs, ncol - 1) * ldb + boff;
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    double av[kTile], bv[kTile];
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii) av[ii] = __ldg(a[ii] + k);
#pragma unroll
    for (int jj = 0; jj < kTile; ++jj) bv[jj] = b[jj][k];
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii)
#pragma unroll
      for (int jj = 0; jj < kTile; ++jj) acc[ii][jj] = fma(av[ii], bv[jj], acc[ii][jj]);
  }
}

// Same with A transposed: A^T[r][k] = A[k][r] (A row-major, lda).
__device__ __forceinline__ void tile_gemm_t(double (&acc)[kTile][kTile], const double* __restrict__ A, int lda,
                                            int M, int r0, const double* B, int ldb, int cb, int cs, int ncol,
                                            int K) {
  const double* b[kTile];
#pragma unroll
  for (int jj = 0; jj < kTile; ++jj) b[jj] = B + min(cb + jj * cs, ncol - 1) * ldb;
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    double av[kTile], bv[kTile];
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii) av[ii] = __ldg(A + static_cast<size_t>(k) * lda + min(r0 + ii, M - 1));
#pragma unroll
    for (int jj = 0; jj < kTile; ++jj) bv[jj] = b[jj][k];
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii)
#pragma unroll
      for (int jj = 0; jj < kTile; ++jj) acc[ii][jj] = fma(av[ii], bv[jj], acc[ii][jj]);
  }
}

struct ChunkSmem {
  int ldb, ldu;
};

__host__ __device__ inline ChunkSmem chunk_layout(int nn, int next) {
  ChunkSmem c;
  c.ldb = nn | 1;      // odd strides: conflict-free column reads
  c.ldu = next | 1;
  return c;
}

__global__ void k_condense_chunk(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ F,
                                 const double* __restrict__ G, int gstride, double* __restrict__ R, int rstride) {
  extern __shared__ double smem[];
  const int c = blockIdx.x, m = blockIdx.y;
  const int nz = g.nz;
  const int nr = (nz > 1 && m > 0) ? 2 : 1;
  const int nn = g.npnp, next = g.next, nint = g.nint;
  const int cnt = g.chunk_count[c];
  const int* el = g.elem_sorted + g.chunk_start[c];
  const ChunkSmem L = chunk_layout(nn, next);
  double* sB = smem;                                   // [2*chunk][ldb]
  double* sD = sB + 2 * g.chunk_max * L.ldb;
  double* wsc = sD + g.np * g.np;                      // [warps][3*nn]
  for (int w = threadIdx.x; w < g.np * g.np; w += blockDim.x) sD[w] = S.D[w];
  __syncthreads();
  chunk_forcing2(g, N, F, G, gstride, S.lambda2[m] + S.betak2[m], el, cnt, m, nr, sB, L.ldb, wsc, sD);
  const double* hbi = S.hbi + (static_cast<size_t>(m) * S.nfamily + g.family[el[0]]) * next * nint;
  const int ncol = nr * cnt;
  const int rt = (next + kTile - 1) / kTile, cs = (ncol + kTile - 1) / kTile;
  for (int tile = threadIdx.x; tile < rt * cs; tile += blockDim.x) {
    const int cb = tile % cs, r0 = (tile / cs) * kTile;
    double acc[kTile][kTile] = {};
    if (nint) tile_gemm(acc, hbi, nint, next, r0, sB, L.ldb, cb, cs, ncol, nint, next);
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii)
#pragma unroll
      for (int jj = 0; jj < kTile; ++jj) {
        const int a = r0 + ii, col = cb + jj * cs;
        if (a < next && col < ncol) {
          const int slot = col / cnt, l = col - slot * cnt;
          const double v = sB[col * L.ldb + a] - acc[ii][jj];
          atomicAdd(&R[static_cast<size_t>(2 * m + slot) * rstride + N.btog[el[l] * next + a]], v);
        }
      }
  }
}

__global__ void k_recover_chunk(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ F,
                                const double* __restrict__ G, int gstride, const double* __restrict__ R, int rstride,
                                double* __restrict__ U) {
  extern __shared__ double smem[];
  const int c = blockIdx.x, m = blockIdx.y;
  const int nz = g.nz;
  const int nr = (nz > 1 && m > 0) ? 2 : 1;
  const int nn = g.npnp, next = g.next, nint = g.nint;
  const int cnt = g.chunk_count[c];
  const int* el = g.elem_sorted + g.chunk_start[c];
  const ChunkSmem L = chunk_layout(nn, next);
  double* sB = smem;                                   // [2*chunk][ldb] forcing columns
  double* sU = sB + 2 * g.chunk_max * L.ldb;           // [2*chunk][ldu] boundary solution
  double* sD = sU + 2 * g.chunk_max * L.ldu;
  double* wsc = sD + g.np * g.np;                      // [warps][3*nn]
  for (int w = threadIdx.x; w < g.np * g.np; w += blockDim.x) sD[w] = S.D[w];
  __syncthreads();
  chunk_forcing2(g, N, F, G, gstride, S.lambda2[m] + S.betak2[m], el, cnt, m, nr, sB, L.ldb, wsc, sD);
  const int nsolve = S.nsolve[m];
  const int ncol = nr * cnt;
#pragma unroll 8
  for (int w = threadIdx.x; w < ncol * next; w += blockDim.x) {
    const int col = w / next, a = w - col * next;
    const int slot = col / cnt, l = col - slot * cnt;
    const int k = 2 * m + slot;
    const int e = el[l];
    const int gi = N.btog[e * next + a];
    const double ub = gi < nsolve ? R[static_cast<size_t>(k) * rstride + gi] : 0.0;
    sU[col * L.ldu + a] = ub;
    U[static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn + g.emap[a]] =
        (N.bmask[e * next + a] && G) ? G[static_cast<size_t>(k) * gstride + gi] : ub;
  }
  __syncthreads();
  const size_t fm = static_cast<size_t>(m) * S.nfamily + g.family[el[0]];
  const double* hii = S.hii + fm * nint * nint;
  const double* hbi = S.hbi + fm * next * nint;
  const int rt = (nint + kTile - 1) / kTile, cs = (ncol + kTile - 1) / kTile;
  for (int tile = threadIdx.x; tile < rt * cs; tile += blockDim.x) {
    const int cb = tile % cs, r0 = (tile / cs) * kTile;
    double acc[kTile][kTile] = {};
    tile_gemm(acc, hii, nint, nint, r0, sB, L.ldb, cb, cs, ncol, nint, next);
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii)
#pragma unroll
      for (int jj = 0; jj < kTile; ++jj) acc[ii][jj] = -acc[ii][jj];
    tile_gemm_t(acc, hbi, nint, nint, r0, sU, L.ldu, cb, cs, ncol, next);
#pragma unroll
    for (int ii = 0; ii < kTile; ++ii)
#pragma unroll
      for (int jj = 0; jj < kTile; ++jj) {
        const int i = r0 + ii, col = cb + jj * cs;
        if (i < nint && col < ncol) {
          const int slot = col / cnt, l = col - slot * cnt;
          U[static_cast<size_t>(2 * m + slot) * g.plane_size + static_cast<size_t>(el[l]) * nn + g.emap[next + i]] =
              -acc[ii][jj];
        }
      }
  }
}

// Banded lower-triangular solve L z = c, in place, for the planes of one mode
// per block (simple form, used for bands too wide for the pipelined sweep).  Row j of L is contiguous: L[j*nband + t] multiplies z[j-kd+t],
// t = kd holds 1/L[j][j].  `reversed` addresses vector entry r at n-1-r.
// Rows are processed in blocks of 32: all warps form the contributions of
// already-solved columns, then warp 0 finishes the block's 32x32 triangle.
__global__ void k_band_solve(DevModal S, const double* __restrict__ Lall,
                             double* __restrict__ R, int rstride, int nz, int reversed) {
  __shared__ double acc[32][2];
  __shared__ double tri[32][33];
  __shared__ double rdiag[32];
  const int m = blockIdx.x;
  const int n = S.nsolve[m];
  const int nb = S.nbp, kd = S.nband - 1;
  const double* L = Lall + static_cast<size_t>(m) * S.mode_stride;
  const int nr = (nz > 1 && m > 0) ? 2 : 1;
  double* z0 = R + static_cast<size_t>(plane_of(m, 0)) * rstride;
  double* z1 = R + static_cast<size_t>(plane_of(m, 1)) * rstride;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  auto at = [&](int r) { return reversed ? n - 1 - r : r; };
  for (int j0 = 0; j0 < n; j0 += 32) {
    const int bn = min(32, n - j0);
    for (int rr = warp; rr < bn; rr += nwarp) {
      const int j = j0 + rr;
      const double* Lj = L + static_cast<size_t>(j) * nb + ((j - kd) & 1);  // skewed row
      const int tlo = max(0, kd - j);
      const int thi = kd - rr;  // columns < j0
      double s0 = 0.0, s1 = 0.0;
      for (int t = tlo + lane; t < thi; t += 32) {
        const int c = at(j - kd + t);
        const double l = Lj[t];
        s0 += l * z0[c];
        if (nr > 1) s1 += l * z1[c];
      }
      for (int o = 16; o; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      }
      if (lane == 0) {
        acc[rr][0] = z0[at(j)] - s0;
        acc[rr][1] = nr > 1 ? z1[at(j)] - s1 : 0.0;
        rdiag[rr] = Lj[kd];
      }
      if (lane < rr) tri[rr][lane] = (rr - lane <= kd) ? Lj[kd - rr + lane] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      double a0 = lane < bn ? acc[lane][0] : 0.0;
      double a1 = lane < bn ? acc[lane][1] : 0.0;
      for (int s = 0; s < bn; ++s) {
        double y0 = a0 * rdiag[s], y1 = a1 * rdiag[s];
        y0 = __shfl_sync(0xffffffffu, y0, s);
        y1 = __shfl_sync(0xffffffffu, y1, s);
        if (lane > s && lane < bn) {
          const double l = tri[lane][s];
          a0 -= l * y0;
          a1 -= l * y1;
        }
        if (lane == s) {
          z0[at(j0 + s)] = y0;
          if (nr > 1) z1[at(j0 + s)] = y1;
        }
      }
    }
    __syncthreads();
  }
}


// ---------------------------------------------------------------------------
// Jacobi-PCG (Field::solve JACPCG, src/field.cpp:711-805): all planes iterate
// in lockstep, each with its own scalars and stopping test, so every plane
// takes exactly the iterations the reference loop takes for it.
// Global vectors per plane: [0, nglobal) element-boundary nodes, then nel
// blocks of nint interior nodes in boundary-major order.
// ---------------------------------------------------------------------------

struct PcgScalars {
  double rho1, rho2, r2, eps, dotp;
  int iter, active, hit_max, solved;
};

// y = H x (Field::HelmholtzOperator, src/field.cpp:855-940) per (element,
// plane); y's boundary part must be zero on entry.
__global__ void k_global_op(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ X,
                            double* __restrict__ Y, int vstride, const PcgScalars* sc) {
  extern __shared__ double smem[];
  const int nn = g.npnp, np = g.np;
  double* sD = smem;
  double* su = sD + np * np;
  double* sR = su + nn;
  double* sS = sR + nn;
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  if (!sc[k].active) return;
  const int m = k >> 1;
  const double hcon = S.lambda2[m] + S.betak2[m];
  const double* x = X + static_cast<size_t>(k) * vstride;
  double* y = Y + static_cast<size_t>(k) * vstride;
  if (N.mixdiag && e == 0)  // <K x, w> on mixed-BC edges (Mixed::augmentOp, src/condition.cpp:379-407)
    for (int q = t; q < N.nglobal; q += blockDim.x) atomicAdd(&y[q], N.mixdiag[q] * x[q]);
  for (int q = t; q < np * np; q += blockDim.x) sD[q] = S.D[q];
  if (t < g.next) su[g.emap[t]] = x[N.btog[e * g.next + t]];
  if (t < g.nint) su[g.emap[g.next + t]] = x[N.nglobal + static_cast<size_t>(e) * g.nint + t];
  __syncthreads();
  const int i = t / np, j = t - (t / np) * np;
  if (t < nn) {
    double r = 0.0, s = 0.0;
    for (int q = 0; q < np; ++q) {
      r += su[i * np + q] * sD[j * np + q];
      s += sD[i * np + q] * su[q * np + j];
    }
    const double q1 = g.Q1[e * nn + t], q2 = g.Q2[e * nn + t], q3 = g.Q3[e * nn + t];
    sR[t] = q1 * r + q3 * s;
    sS[t] = q2 * s + q3 * r;
  }
  __syncthreads();
  if (t < nn) {
    double h = g.Q4[e * nn + t] * su[t] * hcon;
    for (int q = 0; q < np; ++q) {
      h += sD[q * np + i] * sS[q * np + j];
      h += sR[i * np + q] * sD[q * np + j];
    }
    const int b = g.pmap[t];
    if (b < g.next)
      atomicAdd(&y[N.btog[e * g.next + b]], h);
    else
      y[N.nglobal + static_cast<size_t>(e) * g.nint + (b - g.next)] = h;
  }
}

// r = assembled constrained forcing (buildRHS without condensation).
__global__ void k_pcg_rhs(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ F,
                          const double* __restrict__ G, int gstride, double* __restrict__ Rv,
                          int vstride) {
  extern __shared__ double smem[];
  const int nn = g.npnp;
  double* sD = smem;
  double* su = sD + g.np * g.np;
  double* sR = su + nn;
  double* sS = sR + nn;
  double* sF = sS + nn;
  const int e = blockIdx.x, k = blockIdx.y;
  if (g.nz > 1 && k == 1) return;
  const int m = k >> 1;
  for (int t = threadIdx.x; t < g.np * g.np; t += blockDim.x) sD[t] = S.D[t];
  __syncthreads();
  constrained_forcing(g, N, F + static_cast<size_t>(k) * g.plane_size,
                      G ? G + static_cast<size_t>(k) * gstride : nullptr,
                      S.lambda2[m] + S.betak2[m], e, su, sR, sS, sF, sD);
  const int t = threadIdx.x;
  double* r = Rv + static_cast<size_t>(k) * vstride;
  if (t < g.next) atomicAdd(&r[N.btog[e * g.next + t]], sF[t]);
  if (t < g.nint) r[N.nglobal + static_cast<size_t>(e) * g.nint + t] = sF[g.next + t];
}

// x <- local2global(unknown) boundary + interior (Field::local2global).
__global__ void k_local2global(DevGeom g, DevNumbering N, const double* __restrict__ U,
                               double* __restrict__ X, int vstride) {
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  if (g.nz > 1 && k == 1) return;
  const double* u = U + static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  double* x = X + static_cast<size_t>(k) * vstride;
  if (t < g.next) x[N.btog[e * g.next + t]] = u[g.emap[t]];
  if (t < g.nint) x[N.nglobal + static_cast<size_t>(e) * g.nint + t] = u[g.emap[g.next + t]];
}

// unknown <- global2local(x), essential values imposed from G.
__global__ void k_global2local(DevGeom g, DevNumbering N, const double* __restrict__ X, int vstride,
                               const double* __restrict__ G, int gstride, double* __restrict__ U) {
  const int e = blockIdx.x, k = blockIdx.y, t = threadIdx.x;
  if (g.nz > 1 && k == 1) return;
  double* u = U + static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp;
  const double* x = X + static_cast<size_t>(k) * vstride;
  if (t < g.next) {
    const int gi = N.btog[e * g.next + t];
    u[g.emap[t]] = (G && N.bmask[e * g.next + t]) ? G[static_cast<size_t>(k) * gstride + gi] : x[gi];
  }
  if (t < g.nint) u[g.emap[g.next + t]] = x[N.nglobal + static_cast<size_t>(e) * g.nint + t];
}

// Zero entries [lo, hi) of each plane's vector; lo = lo_mode[mode] if given.
__global__ void k_zero_range(double* V, int vstride, int lo, const int* lo_mode, int hi, int nz) {
  const int k = blockIdx.y;
  if (k >= nz) return;
  const int l = lo_mode ? lo_mode[k >> 1] : lo;
  for (int i = l + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    V[static_cast<size_t>(k) * vstride + i] = 0.0;
}

// out[k] += sum_i a[k][i] * b[k][i] over active (or all, if force) planes.
__global__ void k_dot(const double* __restrict__ A, const double* __restrict__ B, int n, int vstride,
                      double* out, const PcgScalars* sc, int force) {
  const int k = blockIdx.y;
  if (!force && !sc[k].active) return;
  double s = 0.0;
  const double* a = A + static_cast<size_t>(k) * vstride;
  const double* b = B + static_cast<size_t>(k) * vstride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(&out[k], s);
  }
}

// r -= p on solved planes.
__global__ void k_sub(double* __restrict__ R, const double* __restrict__ P, int n, int vstride,
                      const PcgScalars* sc) {
  const int k = blockIdx.y;
  if (!sc[k].solved) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    R[static_cast<size_t>(k) * vstride + i] -= P[static_cast<size_t>(k) * vstride + i];
}

// Per-plane scalar bookkeeping.
__global__ void k_pcg_init(PcgScalars* sc, const double* bb, const double* rr, double tol, int nz) {
  const int k = threadIdx.x;
  if (k >= nz) return;
  PcgScalars s{};
  const bool solved = !(nz > 1 && k == 1);
  const double e = tol * sqrt(bb[k]);
  s.eps = e * e;
  s.r2 = rr[k];
  s.iter = 0;
  s.solved = solved;
  s.active = solved ? 1 : 0;
  s.hit_max = 0;
  sc[k] = s;
}

// Loop head `while (r2 > epsb2 && ++i < StepMax)`.
__global__ void k_pcg_head(PcgScalars* sc, int step_max, int nz, int* any_active) {
  const int k = threadIdx.x;
  if (k >= nz) return;
  PcgScalars& s = sc[k];
  if (s.active) {
    if (s.r2 > s.eps) {
      s.iter += 1;
      if (s.iter >= step_max) {
        s.active = 0;
        s.hit_max = 1;
      }
    } else {
      s.active = 0;
    }
  }
  if (s.active) atomicOr(any_active, 1);
}

// z = PC r ; (after rho1 computed) p = z + beta p.
__global__ void k_pcg_precond(const double* __restrict__ PC, int npts, const double* __restrict__ R,
                              double* __restrict__ Z, int vstride, const PcgScalars* sc) {
  const int k = blockIdx.y;
  if (!sc[k].active) return;
  const double* pc = PC + static_cast<size_t>(k >> 1) * npts;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += gridDim.x * blockDim.x)
    Z[static_cast<size_t>(k) * vstride + i] = pc[i] * R[static_cast<size_t>(k) * vstride + i];
}

__global__ void k_pcg_dir(const double* __restrict__ Z, double* __restrict__ P, int n, int vstride,
                          PcgScalars* sc, const double* rho1) {
  const int k = blockIdx.y;
  if (!sc[k].active) return;
  const double beta = sc[k].iter == 1 ? 0.0 : rho1[k] / sc[k].rho2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t o = static_cast<size_t>(k) * vstride + i;
    P[o] = sc[k].iter == 1 ? Z[o] : Z[o] + beta * P[o];
  }
}

__global__ void k_pcg_step(double* __restrict__ X, double* __restrict__ R, const double* __restrict__ P,
                           const double* __restrict__ Q, int n, int vstride, const PcgScalars* sc,
                           const double* rho1, const double* dotp) {
  const int k = blockIdx.y;
  if (!sc[k].active) return;
  const double alpha = rho1[k] / dotp[k];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t o = static_cast<size_t>(k) * vstride + i;
    X[o] += alpha * P[o];
    R[o] -= alpha * Q[o];
  }
}

__global__ void k_pcg_tail(PcgScalars* sc, const double* rho1, const double* r2, int nz) {
  const int k = threadIdx.x;
  if (k >= nz || !sc[k].active) return;
  sc[k].rho2 = rho1[k];
  sc[k].r2 = r2[k];
}


// ---------------------------------------------------------------------------
// Pipelined banded sweep.  Same contract as k_band_solve.  The factor rows of
// a 16-row block are contiguous in HBM, so one bulk (TMA) copy per block and
// one for the block's inverse diagonal move them into a shared-memory ring of
// `stages` buffers, issued `stages` blocks ahead and completed on an mbarrier
// per buffer.  The solved entries live in a shared-memory window of W
// (power of two >= kd + 16) columns per RHS.  Per block: all warps form
// acc = c - L_far z_far from shared memory, then z_B = T_B^{-1} acc with the
// precomputed inverse of the block's triangle.  Waits are bounded: on
// expiry the kernel records an error in S.status and stops.
// ---------------------------------------------------------------------------



constexpr int kSweepWarps = 1 + kBandRows;  // one chain warp + one warp per block row
constexpr int kSweepThreads = 32 * kSweepWarps;

// Skewed row layout (built on the host): row j holds the coefficients of
// columns [cs_j, cs_j + nbq) with cs_j = (j - kd) rounded down to even, so
// that column pairs (2p, 2p+1) are 16-byte aligned in both the factor row
// and the solution window; entries outside the band are zero.
__device__ __forceinline__ int skew_start(int j, int kd) {
  const int c = j - kd;
  return c - (c & 1);
}

template <int NR>
__device__ __forceinline__ void sweep_body(const DevModal& S, const double* __restrict__ Lall,
                                           const double* __restrict__ Dall, double* __restrict__ R,
                                           int rstride, int reversed, int stages, int W, int m,
                                           unsigned char* smraw) {
  constexpr int B = kBandRows;
  const int n = S.nsolve[m];
  const int nbq = S.nbp, kd = S.nband - 1;
  const size_t stage_doubles = static_cast<size_t>(B) * nbq + B * B;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);  // [stages] in a 128-byte slot
  double* ring = reinterpret_cast<double*>(smraw + 128);
  double* win = ring + stage_doubles * stages;  // [NR][W]
  double* fbuf = win + static_cast<size_t>(NR) * W;  // [2][B][NR] far sums
  double* cbuf = fbuf + 2 * B * NR;                   // [2][B][NR] right-hand sides
  __shared__ int failed;
  const double* L = Lall + static_cast<size_t>(m) * S.mode_stride;
  const double* Dv = Dall + static_cast<size_t>(m) * S.dinv_stride;
  double* z[2] = {R + static_cast<size_t>(2 * m) * rstride, R + static_cast<size_t>(2 * m + 1) * rstride};
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nblk = (n + B - 1) / B;
  auto at = [&](int r) { return reversed ? n - 1 - r : r; };
  auto issue = [&](int b) {
    const int j0 = b * B;
    const int bn = min(B, n - j0);
    double* dst = ring + static_cast<size_t>(b % stages) * stage_doubles;
    const unsigned rows_bytes = static_cast<unsigned>(bn) * nbq * 8u;
    mbar_expect_tx(&bar[b % stages], rows_bytes + B * B * 8u);
    bulk_g2s(dst, L + static_cast<size_t>(j0) * nbq, rows_bytes, &bar[b % stages]);
    bulk_g2s(dst + static_cast<size_t>(B) * nbq, Dv + static_cast<size_t>(b) * B * B, B * B * 8u,
             &bar[b % stages]);
  };
  for (int i = tid; i < NR * W; i += kSweepThreads) win[i] = 0.0;
  if (tid == 0) {
    failed = 0;
    for (int s2 = 0; s2 < stages; ++s2) mbar_init(&bar[s2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // block 0: right-hand sides, no far part
  if (warp >= 1 && lane < NR) {
    const int rr = warp - 1;
    cbuf[rr * NR + lane] = rr < min(B, n) ? z[lane][at(rr)] : 0.0;
    fbuf[rr * NR + lane] = 0.0;
  }
  __syncthreads();
  if (tid == 0)
    for (int b = 0; b < min(stages, nblk); ++b) issue(b);
  double zprev = 0.0;  // chain warp: z of the previous block, lane = r*16 + rr
  for (int b = 0; b < nblk; ++b) {
    const int j0 = b * B;
    if (warp == 0) {
      // ---- chain: z_b = Tinv_b (c_b - far_b - N_b z_{b-1})
      if (!mbar_wait(&bar[b % stages], (b / stages) & 1)) {
        if (lane == 0) {
          failed = 1;
          atomicExch(S.status, 1);
        }
      }
      __syncwarp();
      const double* Lb = ring + static_cast<size_t>(b % stages) * stage_doubles;
      const double* Tinv = Lb + static_cast<size_t>(B) * nbq;
      const int bn = min(B, n - j0);
      const int rr = lane & (B - 1), r = lane >> 4;
      const bool live = rr < bn && r < NR;
      const int j = j0 + rr;
      const int cs = skew_start(j, kd);
      const double* Lr = Lb + static_cast<size_t>(rr) * nbq;
      double acc = live ? cbuf[(b & 1) * B * NR + rr * NR + r] - fbuf[(b & 1) * B * NR + rr * NR + r] : 0.0;
      for (int s2 = 0; s2 < B; ++s2) {
        const double zs = __shfl_sync(0xffffffffu, zprev, (lane & 16) | s2);
        const int pos = j0 - B + s2 - cs;
        if (live && pos >= 0) acc = fma(-Lr[pos], zs, acc);
      }
      double zb = 0.0;
      for (int s2 = 0; s2 < B; ++s2) {
        const double as = __shfl_sync(0xffffffffu, acc, (lane & 16) | s2);
        if (live && s2 <= rr) zb = fma(Tinv[rr * B + s2], as, zb);
      }
      if (live) {
        win[r * W + ((j0 + rr) & (W - 1))] = zb;
        z[r][at(j0 + rr)] = zb;
      }
      zprev = live ? zb : 0.0;
    } else if (b + 1 < nblk) {
      // ---- far part of block b+1: columns < j0(b), rows one per warp
      const int rr = warp - 1;
      const int j1 = j0 + B;
      const int bn1 = min(B, n - j1);
      if (!mbar_wait(&bar[(b + 1) % stages], ((b + 1) / stages) & 1)) {
        if (lane == 0) {
          failed = 1;
          atomicExch(S.status, 1);
        }
      }
      if (rr < bn1) {
        const int j = j1 + rr;
        double c[NR];
        if (lane == 0)
          for (int r = 0; r < NR; ++r) c[r] = z[r][at(j)];
        const double* Lr = ring + static_cast<size_t>((b + 1) % stages) * stage_doubles +
                           static_cast<size_t>(rr) * nbq;
        const int cs = skew_start(j, kd);
        double s0[NR], s1[NR];
        for (int r = 0; r < NR; ++r) s0[r] = s1[r] = 0.0;
#pragma unroll 4
        for (int col = cs + 2 * lane; col < j0; col += 64) {
          const double2 l = *reinterpret_cast<const double2*>(Lr + (col - cs));
          const int wi = col & (W - 1);
          for (int r = 0; r < NR; ++r) {
            const double2 zz = *reinterpret_cast<const double2*>(win + r * W + wi);
            s0[r] = fma(l.x, zz.x, s0[r]);
            s1[r] = fma(l.y, zz.y, s1[r]);
          }
        }
        for (int r = 0; r < NR; ++r) {
          double v = s0[r] + s1[r];
          for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) {
            fbuf[((b + 1) & 1) * B * NR + rr * NR + r] = v;
            cbuf[((b + 1) & 1) * B * NR + rr * NR + r] = c[r];
          }
        }
      }
    }
    __syncthreads();
    if (failed) break;
    if (tid == 32 && b + stages < nblk) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(b + stages);
    }
  }
  if (failed && tid == 0)
    for (int s2 = 0; s2 < stages; ++s2) {
      mbar_wait(&bar[s2], 0);  // bounded
      mbar_wait(&bar[s2], 1);
    }
}

// One block per mode; mode 0 (and every mode when nz == 1) holds one real
// plane, the others a Re/Im pair that shares each factor read.
__global__ void __launch_bounds__(kSweepThreads) k_band_sweep(DevModal S, const double* __restrict__ Lall,
                                                              const double* __restrict__ Dall,
                                                              double* __restrict__ R, int rstride, int nz,
                                                              int reversed, int stages, int W) {
  extern __shared__ __align__(128) unsigned char smraw[];
  const int m = blockIdx.x;
  if (nz > 1 && m > 0)
    sweep_body<2>(S, Lall, Dall, R, rstride, reversed, stages, W, m, smraw);
  else
    sweep_body<1>(S, Lall, Dall, R, rstride, reversed, stages, W, m, smraw);
}

// Shared-memory plan of k_band_sweep for a band row stride; 0 stages if the
// band is too wide for two buffers.
struct SweepPlan {
  int stages = 0, W = 0;
  size_t smem = 0;
};

SweepPlan sweep_plan(int nbp, int nband) {
  SweepPlan p;
  int W = 64;
  while (W < nband - 1 + 2 * kBandRows + 2) W <<= 1;
  const size_t stage = sizeof(double) * (static_cast<size_t>(kBandRows) * nbp + kBandRows * kBandRows);
  const size_t fixed = 128 + sizeof(double) * (2 * static_cast<size_t>(W) + 8 * kBandRows);
  const size_t limit = 220 * 1024;
  if (fixed + 2 * stage > limit) return p;
  p.stages = static_cast<int>(std::min<size_t>(4, (limit - fixed) / stage));
  p.W = W;
  p.smem = fixed + stage * p.stages;
  return p;
}

}  // namespace

size_t helmholtz_workspace_doubles(const DevGeom& g, const DevNumbering& N, const DevModal& S) {
  const size_t stride = (static_cast<size_t>(N.nglobal) + 31) / 32 * 32;
  size_t n = 2 * stride * g.nz;
  if (S.l2) {
    n += twolevel_workspace_doubles(static_cast<int>(stride), g.nz);
    // mixed precision: the condensed right-hand side, the residual and the
    // correction's solve
    if (S.refine > 0) n += 2 * stride * g.nz + twolevel_workspace_doubles(static_cast<int>(stride), g.nz);
  }
  return n;
}

int helmholtz_direct_launches(const DevNumbering& N, const DevModal& S, int np) {
  const bool has_ess = N.nglobal > N.nsolve;
  const int nedge_nodes = N.nedge * np;
  const int refine = S.l2 ? S.refine * (twolevel_launches(S) + 2) : 0;
  return 2 + (S.l2 ? twolevel_launches(S) : 2) + (has_ess && nedge_nodes ? 1 : 0) + (nedge_nodes ? 1 : 0) + refine;
}

cudaError_t helmholtz_direct_solve(const DevGeom& g, const DevNumbering& N, const DevModal& S,
                                   const double* F, double* U, const double* lines, int nline,
                                   double* work, cudaStream_t st, cudaEvent_t* ev, cudaEvent_t after_condense) {
  const int rstride = (N.nglobal + 31) / 32 * 32;
  double* R = work;
  double* G = work + static_cast<size_t>(rstride) * g.nz;
  const int nz = g.nz;
  // planes of the launch's modes [mode0, mode0 + nmodes): [k0, k1)
  const int k0 = nz > 1 ? 2 * S.mode0 : 0, k1 = nz > 1 ? std::min(nz, 2 * (S.mode0 + S.nmodes)) : 1;
  const size_t pz = static_cast<size_t>(rstride) * (k1 - k0);
  if (ev) cudaEventRecord(ev[0], st);
  const bool pdl = S.pdl != 0;
  // R, G and (two-level) the skeleton solution zeroed in one kernel
  ZeroRanges zr;
  zr.add(R + static_cast<size_t>(rstride) * k0, pz);
  zr.add(G + static_cast<size_t>(rstride) * k0, pz);
  if (S.l2) zr.add(twolevel_solution(work + 2 * static_cast<size_t>(rstride) * nz, rstride, nz) +
                       static_cast<size_t>(rstride) * k0,
                   pz);
  cudaError_t err = zero_ranges(pdl, zr, st);
  if (err != cudaSuccess) return err;
  const bool has_ess = N.nglobal > N.nsolve;
  const int nedge_nodes = N.nedge * g.np;
  if (has_ess && nedge_nodes && N.ness) {
    dim3 grid((nedge_nodes + 127) / 128, k1 - k0);
    launch_ex(pdl, k_essential, grid, dim3(128), 0, st, g, N, lines, nline, G, rstride, nz, k0);
  }
  const int threads = ((g.npnp + 31) / 32) * 32 < 64 ? 64 : ((g.npnp + 31) / 32) * 32;
  const size_t shm = sizeof(double) * (static_cast<size_t>(g.np) * g.np + 5 * g.npnp);
  dim3 egrid(g.nel, nz);
  const size_t nn = g.npnp, cm = g.chunk_max;
  const size_t ldb = nn | 1, ldu = g.next | 1;
  const size_t wsc = 8 * 3 * nn;  // warp scratch of the lift term, 8 warps
  const size_t shm_cond = sizeof(double) * (2 * cm * ldb + g.np * g.np + wsc);
  const size_t shm_rec = sizeof(double) * (2 * cm * ldb + 2 * cm * ldu + g.np * g.np + wsc);
  const bool chunked = g.nchunk > 0 && shm_rec <= 200 * 1024;
  const ElementPlan ep = element_plan(g, S, has_ess);
  if (ep.ok) {
    element_condense(ep, g, N, S, F, has_ess ? G : nullptr, rstride, R, rstride, st);
  } else if (chunked) {
    raise_smem_limit(reinterpret_cast<const void*>(k_condense_chunk), 200 * 1024);
    raise_smem_limit(reinterpret_cast<const void*>(k_recover_chunk), 200 * 1024);
    k_condense_chunk<<<dim3(g.nchunk, S.nmodes), 256, shm_cond, st>>>(g, N, S, F, has_ess ? G : nullptr, rstride,
                                                                      R, rstride);
  } else {
    k_condense<<<egrid, threads, shm, st>>>(g, N, S, F, has_ess ? G : nullptr, rstride, R, rstride);
  }
  if (nedge_nodes && N.nnat) {
    dim3 grid((nedge_nodes + 127) / 128, k1 - k0);
    launch_ex(pdl && ep.ok, k_natural, grid, dim3(128), 0, st, g, N, lines, nline, R, rstride, nz, k0);
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (after_condense) cudaEventRecord(after_condense, st);
  const SweepPlan plan = S.l2 ? SweepPlan() : sweep_plan(S.nbp, S.nband);
  const double* Rsol = R;  // skeleton solution
  if (S.l2) {
    double* w2 = work + 2 * static_cast<size_t>(rstride) * nz;
    // mixed precision: skeleton products with FP32 matrices, then `refine`
    // corrections  Y += S^-1_32 (R - S Y)  whose residual uses the FP64
    // element Schur complements (the operator the FP64 inverses invert)
    const bool mixed = S.l2_pack32 != nullptr;
    const size_t off = static_cast<size_t>(rstride) * k0;
    double* R0 = w2 + twolevel_workspace_doubles(rstride, nz);
    double* rr = R0 + static_cast<size_t>(rstride) * nz;
    double* w3 = rr + static_cast<size_t>(rstride) * nz;
    if (mixed && S.refine > 0)
      err = cudaMemcpyAsync(R0 + off, R + off, sizeof(double) * pz, cudaMemcpyDeviceToDevice, st);
    if (err == cudaSuccess)
      err = twolevel_solve(S, g, N, R, rstride, w2, nz, st, ev ? ev[2] : nullptr, mixed, /*y_zeroed=*/true);
    if (err != cudaSuccess) return err;
    double* Y = twolevel_solution(w2, rstride, nz);
    for (int it = 0; it < S.refine; ++it) {
      err = cudaMemcpyAsync(rr + off, R0 + off, sizeof(double) * pz, cudaMemcpyDeviceToDevice, st);
      if (err != cudaSuccess) return err;
      element_schur_apply(2, g, N, S, Y, rr, rstride, st);
      err = twolevel_solve(S, g, N, rr, rstride, w3, nz, st, nullptr, true);
      if (err != cudaSuccess) return err;
      const double* D = twolevel_solution(w3, rstride, nz);
      k_add<<<(static_cast<unsigned>(pz) + 255) / 256, 256, 0, st>>>(Y + off, D + off, pz);
    }
    Rsol = Y;
  } else if (plan.stages >= 2) {
    raise_smem_limit(reinterpret_cast<const void*>(k_band_sweep), 220 * 1024);
    k_band_sweep<<<S.nmodes, kSweepThreads, plan.smem, st>>>(S, S.fwd, S.dinv_fwd, R, rstride, nz, 0,
                                                             plan.stages, plan.W);
    if (ev) cudaEventRecord(ev[2], st);
    k_band_sweep<<<S.nmodes, kSweepThreads, plan.smem, st>>>(S, S.bwd, S.dinv_bwd, R, rstride, nz, 1,
                                                             plan.stages, plan.W);
  } else {
    k_band_solve<<<S.nmodes, 256, 0, st>>>(S, S.fwd, R, rstride, nz, 0);
    if (ev) cudaEventRecord(ev[2], st);
    k_band_solve<<<S.nmodes, 256, 0, st>>>(S, S.bwd, R, rstride, nz, 1);
  }
  if (ev) cudaEventRecord(ev[3], st);
  if (ep.ok)
    element_recover(ep, g, N, S, F, has_ess ? G : nullptr, rstride, Rsol, rstride, U, st);
  else if (chunked)
    k_recover_chunk<<<dim3(g.nchunk, S.nmodes), 256, shm_rec, st>>>(g, N, S, F, has_ess ? G : nullptr, rstride,
                                                                    Rsol, rstride, U);
  else
    k_recover<<<egrid, threads, shm + sizeof(double) * g.next, st>>>(g, N, S, F, has_ess ? G : nullptr,
                                                                     rstride, Rsol, rstride, U);
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

bool helmholtz_fields_supported(const DevGeom& g, const DevNumbering& N, const DevModal& S) {
  return S.l2 && !S.l2_pack32 && S.refine == 0 && element_plan(g, S, N.nglobal > N.nsolve).ok;
}

size_t helmholtz_fields_workspace_doubles(const DevGeom& g, const DevNumbering& N, int nf) {
  const size_t stride = (static_cast<size_t>(N.nglobal) + 31) / 32 * 32;
  return 3 * stride * g.nz * nf;
}

cudaError_t helmholtz_direct_solve_fields(const DevGeom& g, const DevNumbering* const* N, const DevModal& S,
                                          const double* const* F, double* const* U, const double* const* lines,
                                          const int* nline, int nf, double* work, cudaStream_t st,
                                          cudaEvent_t after_condense) {
  if (nf < 1 || nf > 3 || !helmholtz_fields_supported(g, *N[0], S)) return cudaErrorInvalidValue;
  const int rstride = (N[0]->nglobal + 31) / 32 * 32;
  const int nz = g.nz;
  const size_t fs = static_cast<size_t>(rstride) * nz;  // field stride of each region
  double* R = work;             // [nf] skeleton right-hand sides
  double* G = R + nf * fs;      // [nf] essential values
  double* Y = G + nf * fs;      // [nf] skeleton solutions
  const int k0 = nz > 1 ? 2 * S.mode0 : 0, k1 = nz > 1 ? std::min(nz, 2 * (S.mode0 + S.nmodes)) : 1;
  const size_t pz = static_cast<size_t>(rstride) * (k1 - k0), off = static_cast<size_t>(rstride) * k0;
  const bool has_ess = N[0]->nglobal > N[0]->nsolve;
  const ElementPlan ep = element_plan(g, S, has_ess);
  const bool pdl = S.pdl != 0;
  // every field's R, G and skeleton solution zeroed in one kernel
  ZeroRanges zr;
  for (int f = 0; f < nf; ++f) {
    zr.add(R + f * fs + off, pz);
    zr.add(G + f * fs + off, pz);
    zr.add(Y + f * fs + off, pz);
  }
  cudaError_t err = zero_ranges(pdl, zr, st);
  if (err != cudaSuccess) return err;
  for (int f = 0; f < nf; ++f) {
    double* Rf = R + f * fs;
    double* Gf = G + f * fs;
    const int nedge_nodes = N[f]->nedge * g.np;
    if (has_ess && nedge_nodes && N[f]->ness) {
      dim3 grid((nedge_nodes + 127) / 128, k1 - k0);
      launch_ex(pdl, k_essential, grid, dim3(128), 0, st, g, *N[f], lines[f], nline[f], Gf, rstride, nz, k0);
    }
    element_condense(ep, g, *N[f], S, F[f], has_ess ? Gf : nullptr, rstride, Rf, rstride, st);
    if (nedge_nodes && N[f]->nnat) {
      dim3 grid((nedge_nodes + 127) / 128, k1 - k0);
      launch_ex(pdl, k_natural, grid, dim3(128), 0, st, g, *N[f], lines[f], nline[f], Rf, rstride, nz, k0);
    }
  }
  if (after_condense) cudaEventRecord(after_condense, st);
  err = twolevel_solve_fields(S, g, *N[0], R, Y, fs, nf, rstride, nz, st, /*y_zeroed=*/true);
  if (err != cudaSuccess) return err;
  for (int f = 0; f < nf; ++f)
    element_recover(ep, g, *N[f], S, F[f], has_ess ? G + f * fs : nullptr, rstride, Y + f * fs, rstride, U[f], st);
  return cudaGetLastError();
}

}  // namespace stx

namespace stx {

size_t jacpcg_workspace_doubles(const DevGeom& g, const DevNumbering& N) {
  const size_t npts = static_cast<size_t>(N.nglobal) + static_cast<size_t>(g.nel) * g.nint;
  const size_t vs = (npts + 31) / 32 * 32;
  const size_t gs = (static_cast<size_t>(N.nglobal) + 31) / 32 * 32;
  // 5 vectors + essential values + scalars (rho1, dotp, r2, bb, flag) + PcgScalars
  return (5 * vs + gs) * g.nz + 8 * static_cast<size_t>(g.nz) + 8 * static_cast<size_t>(g.nz) + 64;
}

cudaError_t helmholtz_jacpcg_solve(const DevGeom& g, const DevNumbering& N, const DevModal& S,
                                   const double* F, double* U, const double* lines, int nline,
                                   double tol_rel, int step_max, double* work, int* iters,
                                   cudaStream_t st) {
  const int nz = g.nz;
  const int npts = N.nglobal + g.nel * g.nint;
  const int vs = (npts + 31) / 32 * 32;
  const int gs = (N.nglobal + 31) / 32 * 32;
  double* r = work;
  double* p = r + static_cast<size_t>(vs) * nz;
  double* q = p + static_cast<size_t>(vs) * nz;
  double* x = q + static_cast<size_t>(vs) * nz;
  double* z = x + static_cast<size_t>(vs) * nz;
  double* G = z + static_cast<size_t>(vs) * nz;
  double* scal = G + static_cast<size_t>(gs) * nz;   // 8*nz doubles
  double* rho1 = scal;
  double* dotp = scal + nz;
  double* r2 = scal + 2 * nz;
  double* bb = scal + 3 * nz;
  int* flag = reinterpret_cast<int*>(scal + 4 * nz);
  PcgScalars* sc = reinterpret_cast<PcgScalars*>(scal + 8 * nz);
  const int nzero_lo = N.nsolve;
  const int nzt = std::min(1024, (nz + 31) / 32 * 32);  // one thread per plane
  cudaError_t err;
  // The per-mode pinned node of a singular system moves nsolve down by one.
  // S.nsolve is on the device; zero [nsolve_m, nglobal) per plane.
  err = cudaMemsetAsync(work, 0, sizeof(double) * ((5 * static_cast<size_t>(vs) + gs) * nz + 8 * nz), st);
  if (err != cudaSuccess) return err;
  const bool has_ess = N.nglobal > N.nsolve;
  const int nedge_nodes = N.nedge * g.np;
  if (has_ess && nedge_nodes) {
    dim3 grid((nedge_nodes + 127) / 128, nz);
    k_essential<<<grid, 128, 0, st>>>(g, N, lines, nline, G, gs, nz, 0);
  }
  const int threads = ((g.npnp + 31) / 32) * 32 < 64 ? 64 : ((g.npnp + 31) / 32) * 32;
  const size_t shm = sizeof(double) * (static_cast<size_t>(g.np) * g.np + 5 * g.npnp);
  dim3 egrid(g.nel, nz);
  k_pcg_rhs<<<egrid, threads, shm, st>>>(g, N, S, F, has_ess ? G : nullptr, gs, r, vs);
  if (nedge_nodes) {
    dim3 grid((nedge_nodes + 127) / 128, nz);
    k_natural<<<grid, 128, 0, st>>>(g, N, lines, nline, r, vs, nz, 0);
  }
  const dim3 vgrid(std::min(1024, (npts + 255) / 256), nz);
  const dim3 zgrid(std::max(1, std::min(64, (N.nglobal + 255) / 256)), nz);
  k_zero_range<<<zgrid, 256, 0, st>>>(r, vs, nzero_lo, S.nsolve, N.nglobal, nz);
  k_dot<<<vgrid, 256, 0, st>>>(r, r, npts, vs, bb, sc, 1);
  // x = local2global(unknown) with essential part zeroed; r -= H x
  k_local2global<<<egrid, threads, 0, st>>>(g, N, U, x, vs);
  k_zero_range<<<zgrid, 256, 0, st>>>(x, vs, nzero_lo, S.nsolve, N.nglobal, nz);
  // all solved planes active for the first operator apply
  k_pcg_init<<<1, nzt, 0, st>>>(sc, bb, bb, tol_rel, nz);
  k_global_op<<<egrid, threads, shm, st>>>(g, N, S, x, p, vs, sc);
  k_zero_range<<<zgrid, 256, 0, st>>>(p, vs, nzero_lo, S.nsolve, N.nglobal, nz);
  k_sub<<<vgrid, 256, 0, st>>>(r, p, npts, vs, sc);
  k_dot<<<vgrid, 256, 0, st>>>(r, r, npts, vs, r2, sc, 1);
  k_pcg_init<<<1, nzt, 0, st>>>(sc, bb, r2, tol_rel, nz);
  // -- iterations
  std::vector<int> hflag(1);
  for (int it = 0; it < step_max + 1; ++it) {
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    k_pcg_head<<<1, nzt, 0, st>>>(sc, step_max, nz, flag);
    if ((it & 7) == 0) {
      cudaMemcpyAsync(hflag.data(), flag, sizeof(int), cudaMemcpyDeviceToHost, st);
      err = cudaStreamSynchronize(st);
      if (err != cudaSuccess) return err;
      if (!hflag[0]) break;
    }
    k_pcg_precond<<<vgrid, 256, 0, st>>>(S.pc, S.npts, r, z, vs, sc);
    cudaMemsetAsync(rho1, 0, sizeof(double) * nz, st);
    k_dot<<<vgrid, 256, 0, st>>>(r, z, npts, vs, rho1, sc, 0);
    k_pcg_dir<<<vgrid, 256, 0, st>>>(z, p, npts, vs, sc, rho1);
    cudaMemsetAsync(q, 0, sizeof(double) * static_cast<size_t>(vs) * nz, st);
    k_global_op<<<egrid, threads, shm, st>>>(g, N, S, p, q, vs, sc);
    k_zero_range<<<zgrid, 256, 0, st>>>(q, vs, nzero_lo, S.nsolve, N.nglobal, nz);
    cudaMemsetAsync(dotp, 0, sizeof(double) * nz, st);
    k_dot<<<vgrid, 256, 0, st>>>(p, q, npts, vs, dotp, sc, 0);
    k_pcg_step<<<vgrid, 256, 0, st>>>(x, r, p, q, npts, vs, sc, rho1, dotp);
    cudaMemsetAsync(r2, 0, sizeof(double) * nz, st);
    k_dot<<<vgrid, 256, 0, st>>>(r, r, npts, vs, r2, sc, 0);
    k_pcg_tail<<<1, nzt, 0, st>>>(sc, rho1, r2, nz);
  }
  k_global2local<<<egrid, threads, 0, st>>>(g, N, x, vs, has_ess ? G : nullptr, gs, U);
  std::vector<PcgScalars> hs(nz);
  cudaMemcpyAsync(hs.data(), sc, sizeof(PcgScalars) * nz, cudaMemcpyDeviceToHost, st);
  err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) return err;
  bool hit = false;
  for (int k = 0; k < nz; ++k) {
    iters[k] = hs[k].solved ? hs[k].iter : -1;
    hit = hit || hs[k].hit_max;
  }
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  return hit ? cudaErrorNotReady : cudaSuccess;
}

}  // namespace stx
