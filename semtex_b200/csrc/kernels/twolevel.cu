// Two-level condensed solve of the skeleton system (all planes at once).
//
// After the element-level condensation has produced the skeleton right-hand
// side R (Element::local2globalSumSC, src/element.cpp:326-365), the reference
// solves the banded skeleton system with dpbtrs (src/field.cpp:693).  Here
// the same linear system is solved by block elimination over patches of
// elements: with I the skeleton unknowns interior to a patch and B those on
// patch interfaces,
//   y_I = S_II^-1 R_I                    (per patch)
//   r_B = R_B - S_BI y_I                 (per element: S is assembled from
//                                         the element Schur complements)
//   x_B = A^-1 r_B                       (A = S_BB - S_BI S_II^-1 S_IB)
//   x_I = S_II^-1 (R_I - S_IB x_B)       (per element, then per patch)
// S_II^-1 and A^-1 are symmetric and stored packed (symtile.hpp); each
// product streams its tiles with bulk copies, the Re and Im planes of a mode
// sharing every tile read, each tile applied as itself and as its transpose.
#include "twolevel.cuh"

#include <algorithm>

#include "ptx.cuh"
#include "symtile.hpp"

namespace stx {

namespace {

constexpr int kSymWarps = 4;   // warps per block of the packed products
constexpr int kSymStages = 2;  // tile buffers per warp
constexpr int kTileDoubles = kSymTile * kSymLd;

__host__ __device__ inline size_t sym_smem(int n) {
  return 128 + sizeof(double) * kSymWarps * kSymStages * kTileDoubles +
         2 * sizeof(double) * kSymTile * static_cast<size_t>(sym_tiles(n));
}

// y[idx] += A x[idx] over the tiles [q0, q1) of one work item per block; the
// warps of the block take consecutive runs of tiles (consecutive in memory:
// packed order).  Per tile (I, J): direct part y_I += A_IJ x_J (lane = tile
// row), and for J < I the transposed part y_J += A_IJ^T x_I (lane = tile
// column); four independent partial sums per plane.  Waits are bounded; on
// expiry S.status is set and the warp stops.
__global__ void __launch_bounds__(32 * kSymWarps)
    k_psymv(const double* __restrict__ pack, const SymItem* __restrict__ items, const double* __restrict__ X,
            double* __restrict__ Y, int rstride, int nz, int* status) {
  extern __shared__ __align__(16) unsigned char sraw[];
  const SymItem it = items[blockIdx.x];
  const int n = it.n, T = sym_tiles(n), m = it.mode;
  const bool two = nz > 1 && m > 0;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sraw) + wp * kSymStages;
  double* ring = reinterpret_cast<double*>(sraw + 128) + static_cast<size_t>(wp) * kSymStages * kTileDoubles;
  double2* sx = reinterpret_cast<double2*>(sraw + 128 + sizeof(double) * kSymWarps * kSymStages * kTileDoubles);
  const int nt = it.q1 - it.q0;
  const int per = (nt + kSymWarps - 1) / kSymWarps;
  const int w0 = it.q0 + min(nt, wp * per), w1 = it.q0 + min(nt, (wp + 1) * per);
  // issue cursor (lane 0): the warp's tiles are contiguous in memory
  int cI = 0, cJ = 0;
  const double* cp = pack + it.moff;
  if (w0 < w1) {
    sym_tile_at(w0, cI, cJ);
    cp += sym_tile_offset(n, cI, cJ);
  }
  auto issue = [&](int s) {
    const int hs = sym_rows_stored(n, cI);
    const unsigned bytes = static_cast<unsigned>(sizeof(double) * kSymLd * hs);
    mbar_expect_tx(&bar[s], bytes);
    bulk_g2s(ring + s * kTileDoubles, cp, bytes, &bar[s]);
    cp += kSymLd * hs;
    if (cJ == cI) {
      ++cI;
      cJ = 0;
    } else {
      ++cJ;
    }
  };
  if (ln == 0) {
    for (int s = 0; s < kSymStages; ++s) mbar_init(&bar[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < kSymStages && w0 + s < w1; ++s) issue(s);
  }
  // x of both planes, zero past n and at the pinned unknown; gathers in
  // batches of 8 per thread
  {
    const double* X0 = X + static_cast<size_t>(2 * m) * rstride;
    const double* X1 = X + static_cast<size_t>(2 * m + 1) * rstride;
    const int nx = kSymTile * T;
    for (int i0 = threadIdx.x; i0 < nx; i0 += 8 * blockDim.x) {
      int gi[8];
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = i0 + u * blockDim.x;
        gi[u] = (i < n && i != it.pin) ? __ldg(it.idx + i) : -1;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        a[u] = gi[u] >= 0 ? X0[gi[u]] : 0.0;
        b[u] = (gi[u] >= 0 && two) ? X1[gi[u]] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = i0 + u * blockDim.x;
        if (i < nx) sx[i] = make_double2(a[u], b[u]);
      }
    }
  }
  __syncthreads();
  double* Y0 = Y + static_cast<size_t>(2 * m) * rstride;
  double* Y1 = Y + static_cast<size_t>(2 * m + 1) * rstride;
  int I = 0, J = 0;
  if (w0 < w1) sym_tile_at(w0, I, J);
  double d0 = 0.0, d1 = 0.0;  // direct part of row 32 I + ln
  int done = 0;               // tiles consumed
  for (int q = w0; q < w1; ++q, ++done) {
    const int s = done % kSymStages;
    const unsigned parity = (done / kSymStages) & 1;
    if (!__all_sync(0xffffffffu, mbar_wait(&bar[s], parity))) {
      if (ln == 0 && status) atomicExch(status, 4);
      break;
    }
    const double* A = ring + s * kTileDoubles;
    const int h = sym_rows(n, I);
    if (ln < h) {
      const double* Ar = A + ln * kSymLd;
      const double2* xJ = sx + kSymTile * J;
      double p0[4] = {0.0, 0.0, 0.0, 0.0}, p1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int c = 0; c < kSymTile; ++c) {
        const double a = Ar[c];
        const double2 x = xJ[c];
        p0[c & 3] = fma(a, x.x, p0[c & 3]);
        p1[c & 3] = fma(a, x.y, p1[c & 3]);
      }
      d0 += (p0[0] + p0[1]) + (p0[2] + p0[3]);
      d1 += (p1[0] + p1[1]) + (p1[2] + p1[3]);
    }
    if (J < I) {
      const double2* xI = sx + kSymTile * I;
      double p0[4] = {0.0, 0.0, 0.0, 0.0}, p1[4] = {0.0, 0.0, 0.0, 0.0};
      if (h == kSymTile) {
#pragma unroll
        for (int r = 0; r < kSymTile; ++r) {
          const double a = A[r * kSymLd + ln];
          const double2 x = xI[r];
          p0[r & 3] = fma(a, x.x, p0[r & 3]);
          p1[r & 3] = fma(a, x.y, p1[r & 3]);
        }
      } else {
        for (int r = 0; r < h; ++r) {
          const double a = A[r * kSymLd + ln];
          const double2 x = xI[r];
          p0[0] = fma(a, x.x, p0[0]);
          p1[0] = fma(a, x.y, p1[0]);
        }
      }
      const int gi = __ldg(it.idx + kSymTile * J + ln);  // J < T - 1: a full tile column
      atomicAdd(&Y0[gi], (p0[0] + p0[1]) + (p0[2] + p0[3]));
      if (two) atomicAdd(&Y1[gi], (p1[0] + p1[1]) + (p1[2] + p1[3]));
    }
    __syncwarp();
    if (ln == 0 && q + kSymStages < w1) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(s);
    }
    if (J == I || q + 1 == w1) {
      if (ln < h) {
        const int gi = __ldg(it.idx + kSymTile * I + ln);
        atomicAdd(&Y0[gi], d0);
        if (two) atomicAdd(&Y1[gi], d1);
      }
      d0 = d1 = 0.0;
    }
    if (J == I) {
      ++I;
      J = 0;
    } else {
      ++J;
    }
  }
  // leave no copy in flight (only after an expired wait)
  for (int q = w0 + done; q < min(w1, w0 + done + kSymStages); ++q) {
    const int k = q - w0;
    mbar_wait(&bar[k % kSymStages], (k / kSymStages) & 1);
  }
}

// Element Schur complement products of the skeleton couplings for one chunk
// of same-family elements and one mode (a warp per element, lanes over its
// boundary nodes, both planes; the family-mode matrix staged in shared
// memory):   dir 0:  dst[B] -= S_BI src[I]     dir 1:  dst[I] -= S_IB src[B]
// with I / B the element nodes of class 1 (patch interior) / 2 (interface).
__global__ void __launch_bounds__(1024)
    k_elem_sc(int dir, DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ src,
              double* __restrict__ dst, int rstride, int nz) {
  extern __shared__ double ssc[];  // [next][next] transposed element Schur complement
  const int c = blockIdx.x, m = blockIdx.y;
  const bool two = nz > 1 && m > 0;
  const int next = g.next;
  const int cnt = g.chunk_count[c];
  const int* el = g.elem_sorted + g.chunk_start[c];
  const double* sct = S.l2_sct + (static_cast<size_t>(m) * S.nfamily + g.family[el[0]]) * next * next;
  for (int i = threadIdx.x; i < next * next; i += blockDim.x) ssc[i] = __ldg(sct + i);
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const int take = dir == 0 ? 1 : 2, put = dir == 0 ? 2 : 1;
  const double* s0 = src + static_cast<size_t>(2 * m) * rstride;
  const double* s1 = src + static_cast<size_t>(2 * m + 1) * rstride;
  int cls[2] = {0, 0}, gi[2] = {0, 0};
  double x0[2] = {0.0, 0.0}, x1[2] = {0.0, 0.0};
  const bool active = wp < cnt;
  if (active) {
    const int e = __ldg(el + wp);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int a = ln + 32 * h;
      if (a < next) {
        cls[h] = __ldg(S.l2_ncls + e * next + a);
        gi[h] = __ldg(N.btog + e * next + a);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      x0[h] = cls[h] == take ? s0[gi[h]] : 0.0;
      x1[h] = (cls[h] == take && two) ? s1[gi[h]] : 0.0;
    }
  }
  __syncthreads();
  if (!active) return;
  double v0[2] = {0.0, 0.0}, v1[2] = {0.0, 0.0};
  for (int b = 0; b < next; ++b) {
    const double xb0 = __shfl_sync(0xffffffffu, b < 32 ? x0[0] : x0[1], b & 31);
    const double xb1 = __shfl_sync(0xffffffffu, b < 32 ? x1[0] : x1[1], b & 31);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int a = ln + 32 * h;
      if (a < next) {
        const double cb = ssc[b * next + a];  // S_e[a][b]
        v0[h] = fma(cb, xb0, v0[h]);
        v1[h] = fma(cb, xb1, v1[h]);
      }
    }
  }
  double* d0 = dst + static_cast<size_t>(2 * m) * rstride;
  double* d1 = dst + static_cast<size_t>(2 * m + 1) * rstride;
#pragma unroll
  for (int h = 0; h < 2; ++h)
    if (cls[h] == put) {
      atomicAdd(&d0[gi[h]], -v0[h]);
      if (two) atomicAdd(&d1[gi[h]], -v1[h]);
    }
}

cudaError_t launch_psymv(const DevModal& S, const SymItem* items, int nitems, int nmax, const double* X, double* Y,
                         int rstride, int nz, cudaStream_t st) {
  if (nitems <= 0) return cudaSuccess;
  const size_t smem = sym_smem(nmax);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaFuncSetAttribute(k_psymv, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    configured = smem;
  }
  k_psymv<<<nitems, 32 * kSymWarps, smem, st>>>(S.l2_pack, items, X, Y, rstride, nz, S.status);
  return cudaGetLastError();
}

}  // namespace

size_t twolevel_workspace_doubles(int rstride, int nz) { return 2 * static_cast<size_t>(rstride) * nz; }

cudaError_t twolevel_solve(const DevModal& S, const DevGeom& g, const DevNumbering& N, double* R, int rstride,
                           double* work, int nz, cudaStream_t st, cudaEvent_t mid) {
  double* Yv = work;
  double* Z = twolevel_solution(work, rstride, nz);
  cudaError_t err = cudaMemsetAsync(work, 0, sizeof(double) * twolevel_workspace_doubles(rstride, nz), st);
  if (err != cudaSuccess) return err;
  const dim3 egrid(g.nchunk, S.nmodes);
  const int ethreads = 32 * g.chunk_max;
  const size_t esmem = sizeof(double) * g.next * g.next;
  // y_I = S_II^-1 R_I; r_B = R_B - S_BI y_I
  err = launch_psymv(S, S.items_patch, S.n_items_patch, S.nI_max, R, Yv, rstride, nz, st);
  if (err != cudaSuccess) return err;
  k_elem_sc<<<egrid, ethreads, esmem, st>>>(0, g, N, S, Yv, R, rstride, nz);
  // x_B = A^-1 r_B
  err = launch_psymv(S, S.items_iface, S.n_items_iface, S.niface, R, Z, rstride, nz, st);
  if (err != cudaSuccess) return err;
  if (mid) cudaEventRecord(mid, st);
  // R_I -= S_IB x_B; x_I = S_II^-1 R_I
  k_elem_sc<<<egrid, ethreads, esmem, st>>>(1, g, N, S, Z, R, rstride, nz);
  err = launch_psymv(S, S.items_patch, S.n_items_patch, S.nI_max, R, Z, rstride, nz, st);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

int twolevel_launches(const DevModal& S) {
  return (S.n_items_patch > 0 ? 2 : 0) + (S.n_items_iface > 0 ? 1 : 0) + 2;
}

}  // namespace stx
