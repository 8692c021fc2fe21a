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
//   x_I = y_I - G x_B                    (per patch, G = S_II^-1 S_IB)
// S_II^-1 and A^-1 are symmetric and stored packed, G in tiles
// (symtile.hpp); each product streams its tiles with bulk copies, the Re and
// Im planes of a mode sharing every tile read, a symmetric tile applied as
// itself and as its transpose.  Tiles are read as doubles, or as floats for
// the mixed-precision solve (the same layout; sums in FP64 either way).
#include "twolevel.cuh"

#include <algorithm>

#include "element.cuh"
#include "launch.hpp"
#include "ptx.cuh"
#include "symtile.hpp"

namespace stx {

namespace {

// Warps per block of the packed products: DevModal::sym_warps (token
// STX_SYM_WARPS, 1..8, default 4: measured faster than 6 for one field).
constexpr int kSymWarpsMax = 8;
constexpr int kSymStages = 1;  // tile buffers per warp
constexpr int kTileDoubles = kSymTile * kSymLd;

// Shared memory per warp: barriers, tile ring, x entries of each buffered
// tile (32 of its column block, 32 of its row block, both planes of each of
// NF fields that share the matrices).
template <int NF>
struct SymWarpSmem {
  uint64_t bar[kSymStages];
  double2 x[kSymStages][2 * kSymTile * NF];
  double tile[kSymStages][kTileDoubles];
};
template <int NF>
constexpr size_t sym_smem(int warps) { return warps * sizeof(SymWarpSmem<NF>); }

// Position of a warp in the tiles of its problems.
struct SymCursor {
  int p, q, I, J, nt, tc;
  SymProblem P;
  __device__ void load(const SymProblem* probs, int prob, int tile) {
    p = prob;
    q = tile;
    P = probs[p];
    if (P.ncol) {
      tc = sym_tiles(P.ncol);
      nt = sym_tiles(P.n) * tc;
      I = q / tc;
      J = q - I * tc;
    } else {
      tc = 0;
      nt = sym_ntiles(P.n);
      sym_tile_at(q, I, J);
    }
  }
  __device__ bool row_last() const { return P.ncol ? J == tc - 1 : J == I; }
  __device__ long long offset() const {
    return P.ncol ? gen_tile_offset(P.n, P.ncol, I, J) : sym_tile_offset(P.n, I, J);
  }
  __device__ void next(const SymProblem* probs, bool more) {
    if (++q == nt) {
      if (more) load(probs, p + 1, 0);
    } else if (row_last()) {
      ++I;
      J = 0;
    } else {
      ++J;
    }
  }
};

// Column of a tile held in position q (0..3) by a lane of column group cq
// (0..7): two 16-byte pairs, 2 cq and 16 + 2 cq, so that the eight lanes
// reading one tile row cover it in one conflict-free 128-byte access each.
__host__ __device__ inline int col_of(int cq, int q) { return 16 * (q >> 1) + 2 * cq + (q & 1); }

// The lane's four entries of a tile row in shared memory (zero when the row
// is past the matrix).
__device__ __forceinline__ void tile_row4(const double* row, int cq, bool ok, double (&e)[4]) {
  if (ok) {
    const double2 u = *reinterpret_cast<const double2*>(row + 2 * cq);
    const double2 v = *reinterpret_cast<const double2*>(row + 16 + 2 * cq);
    e[0] = u.x;
    e[1] = u.y;
    e[2] = v.x;
    e[3] = v.y;
  } else {
    e[0] = e[1] = e[2] = e[3] = 0.0;
  }
}
__device__ __forceinline__ void tile_row4(const float* row, int cq, bool ok, double (&e)[4]) {
  if (ok) {
    const float2 u = *reinterpret_cast<const float2*>(row + 2 * cq);
    const float2 v = *reinterpret_cast<const float2*>(row + 16 + 2 * cq);
    e[0] = u.x;
    e[1] = u.y;
    e[2] = v.x;
    e[3] = v.y;
  } else {
    e[0] = e[1] = e[2] = e[3] = 0.0;
  }
}

// The last two halving exchanges (lane bits 1, 0) of a sum over the 8 lanes
// that share (lane >> 3): v[i] holds, after the first exchange (bit 2), the
// pair sums of row group i (lanes with bit 2 set: the upper row of the
// pair); lane l ends with the sum for position l & 7.
__device__ __forceinline__ double reduce_scatter4_low(const double (&w)[4], int ln) {
  double u[2];
  const bool h1 = ln & 2, h0 = ln & 1;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double send = h1 ? w[i] : w[2 + i], keep = h1 ? w[2 + i] : w[i];
    u[i] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  const double send = h0 ? u[0] : u[1], keep = h0 ? u[1] : u[0];
  return keep + __shfl_xor_sync(0xffffffffu, send, 1);
}

// Sum over the 4 lanes that share (lane & 7) of v[q], q = 0..3: lane l ends
// with the sum for q = l >> 3 (halving exchanges over lane bits 4, 3).
__device__ __forceinline__ double reduce_scatter4_high(const double (&v)[4], int ln) {
  double w[2];
  const bool h4 = ln & 16, h3 = ln & 8;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double send = h4 ? v[i] : v[2 + i], keep = h4 ? v[2 + i] : v[i];
    w[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  const double send = h3 ? w[0] : w[1], keep = h3 ? w[1] : w[0];
  return keep + __shfl_xor_sync(0xffffffffu, send, 8);
}

// y[idx] += scale A x[idx] for every problem (and each of NF fields whose
// vectors are fstride doubles apart): each warp streams its run of tiles
// (SymWarp) through a ring of kSymStages buffers.  For a tile, lane 0
// bulk-copies the tile and every lane copies (cp.async) the x entries of the
// tile's column and row blocks, all completing on the buffer's mbarrier (count 1 + 32).
// Per tile (I, J) every lane reads its 8 x 4 entries of the tile once from
// shared memory (eight lanes cover a tile row with 16-byte reads) and forms
// both products from registers: the direct part y_I += A_IJ x_J as partial
// row sums over its four columns, summed over the eight lanes of a row by a
// halving exchange of warp shuffles (one row per lane, accumulated along the
// tile row and added at its end), and for J < I the transposed part
// y_J += A_IJ^T x_I as partial column sums over its eight rows, summed over
// the four lanes of a column the same way.  Waits are bounded; on expiry `status` is set and the
// warp stops.  Two builds (DevModal::sym_regcap chooses): CAP 0, blocks of
// up to 4 warps and the registers the code wants (no minimum block count:
// giving one lets the compiler take up to 255); CAP 1, blocks of up to 8
// warps and at most 80 registers (three such blocks per SM), a few spilled,
// more resident warps.
template <class T, int NF, int CAP>
__global__ void __launch_bounds__(CAP ? 32 * kSymWarpsMax : 128, CAP ? 2 : 4)
    k_psymv(const T* __restrict__ pack, const SymProblem* __restrict__ probs, const SymWarp* __restrict__ warps,
            int nwarps, const double* __restrict__ X, double* __restrict__ Y, int rstride, size_t fstride, int nz,
            int* status, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char sraw[];
  pdl_trigger();
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + wp;
  if (gw >= nwarps) {  // the warps of a block never synchronise with each other
    pdl_wait();
    return;
  }
  SymWarpSmem<NF>& sm = reinterpret_cast<SymWarpSmem<NF>*>(sraw)[wp];
  const SymWarp W = warps[gw];
  SymCursor ic, cc;  // issue and consume cursors
  ic.load(probs, W.prob, W.q);
  cc = ic;
  if (ln == 0) {
    for (int s = 0; s < kSymStages; ++s) mbar_init(&sm.bar[s], 1 + 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  int issued = 0;
  // positions in the plane vectors of the x entries of the next tile to
  // issue (column block, row block), loaded one issue ahead
  int pf[2];
  auto prefetch = [&]() {
    const int i = kSymTile * ic.J + ln;  // column block
    if (ic.P.ncol) {
      pf[0] = i < ic.P.ncol ? __ldg(ic.P.idx_col + i) : -1;
      pf[1] = -1;  // general products have no transposed part
    } else {
      pf[0] = (i < ic.P.n && i != ic.P.pin) ? __ldg(ic.P.idx + i) : -1;
      const int r = kSymTile * ic.I + ln;  // row block
      pf[1] = (r < ic.P.n && r != ic.P.pin) ? __ldg(ic.P.idx + r) : -1;
    }
  };
  prefetch();
  auto issue = [&](int s) {
    const int n = ic.P.n, m = ic.P.mode;
    const bool two = nz > 1 && m > 0;
    if (ln == 0) {
      const unsigned bytes = static_cast<unsigned>(sizeof(T) * kSymLd * sym_rows_stored(n, ic.I));
      mbar_expect_tx(&sm.bar[s], bytes);
      bulk_g2s(sm.tile[s], pack + ic.P.moff + ic.offset(), bytes, &sm.bar[s]);
    }
    // the matrix tiles are set-up data; the x entries (and the y atomics
    // after them) depend on the previous kernel
    if (issued == 0) pdl_wait();
    const double* X0 = X + static_cast<size_t>(2 * m) * rstride;
    const double* X1 = X0 + rstride;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gi = pf[h];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        double2* d = &sm.x[s][(kSymTile * h + ln) * NF + f];
        if (gi >= 0) {
          cp_async8(&d->x, X0 + f * fstride + gi);
          if (two) cp_async8(&d->y, X1 + f * fstride + gi);
          else d->y = 0.0;
        } else {
          *d = make_double2(0.0, 0.0);
        }
      }
    }
    cp_async_arrive_noinc(&sm.bar[s]);
    ++issued;
    ic.next(probs, issued < W.count);
    if (issued < W.count) prefetch();
  };
  for (int s = 0; s < kSymStages && s < W.count; ++s) issue(s);
  if (W.count == 0) pdl_wait();
  // lane (rho, cq) = (lane >> 3, lane & 7): rows 4 t + rho (t = 0..7) and
  // columns col_of(cq, q) (q = 0..3) of every tile; it collects row
  // 4 cq + rho of the direct part and column col_of(cq, rho) of the
  // transposed part
  const int rho = ln >> 3, cq = ln & 7;
  double d0[NF], d1[NF];  // direct part of row 32 I + 4 cq + rho
#pragma unroll
  for (int f = 0; f < NF; ++f) d0[f] = d1[f] = 0.0;
  int done = 0;
  for (; done < W.count; ++done) {
    const int s = done % kSymStages;
    if (!__all_sync(0xffffffffu, mbar_wait(&sm.bar[s], (done / kSymStages) & 1, wait_ns))) {
      if (ln == 0 && status) atomicExch(status, 4);
      break;
    }
    const int n = cc.P.n, m = cc.P.mode, I = cc.I, J = cc.J;
    const bool two = nz > 1 && m > 0, sym = cc.P.ncol == 0, trans = sym && J < I;
    const double scale = cc.P.scale;
    const T* A = reinterpret_cast<const T*>(sm.tile[s]);
    const double2* xs = sm.x[s];
    const int h = sym_rows(n, I);
    // output positions (the column this lane collects for the transposed
    // part, the row it collects where the tile row ends), loaded before the
    // products to overlap their latency
    const bool row_end = cc.row_last() || done + 1 == W.count;
    const int rrow = 4 * cq + rho;
    const int g_col = trans ? __ldg(cc.P.idx + kSymTile * J + col_of(cq, rho)) : 0;  // J < I: a full block
    const int g_row = (row_end && rrow < h) ? __ldg(cc.P.idx + kSymTile * I + rrow) : 0;
    double* Y0 = Y + static_cast<size_t>(2 * m) * rstride;
    double* Y1 = Y0 + rstride;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double2 xc[4];  // x of the lane's four columns (column block)
#pragma unroll
      for (int q = 0; q < 4; ++q) xc[q] = xs[col_of(cq, q) * NF + f];
      double w0[4], w1[4], tp0[4] = {0.0, 0.0, 0.0, 0.0}, tp1[4] = {0.0, 0.0, 0.0, 0.0};
      const bool h2 = ln & 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        // rows 4 i + rho and 16 + 4 i + rho, their direct partial sums
        // combined at once over lane bit 2 (the first halving exchange)
        double dp[2][2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int r = 16 * k + 4 * i + rho;
          double e[4];
          tile_row4(A + r * kSymLd, cq, r < h, e);
          dp[k][0] = fma(e[0], xc[0].x, fma(e[1], xc[1].x, fma(e[2], xc[2].x, e[3] * xc[3].x)));
          dp[k][1] = fma(e[0], xc[0].y, fma(e[1], xc[1].y, fma(e[2], xc[2].y, e[3] * xc[3].y)));
          if (trans) {
            const double2 xr = xs[(kSymTile + r) * NF + f];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              tp0[q] = fma(e[q], xr.x, tp0[q]);
              tp1[q] = fma(e[q], xr.y, tp1[q]);
            }
          }
        }
        w0[i] = (h2 ? dp[1][0] : dp[0][0]) + __shfl_xor_sync(0xffffffffu, h2 ? dp[0][0] : dp[1][0], 4);
        w1[i] = (h2 ? dp[1][1] : dp[0][1]) + __shfl_xor_sync(0xffffffffu, h2 ? dp[0][1] : dp[1][1], 4);
      }
      d0[f] += reduce_scatter4_low(w0, ln);
      d1[f] += reduce_scatter4_low(w1, ln);
      if (trans) {
        const double s0 = reduce_scatter4_high(tp0, ln), s1 = reduce_scatter4_high(tp1, ln);
        atomicAdd(&Y0[f * fstride + g_col], scale * s0);
        if (two) atomicAdd(&Y1[f * fstride + g_col], scale * s1);
      }
    }
    if (row_end) {
      if (rrow < h) {
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          atomicAdd(&Y0[f * fstride + g_row], scale * d0[f]);
          if (two) atomicAdd(&Y1[f * fstride + g_row], scale * d1[f]);
        }
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) d0[f] = d1[f] = 0.0;
    }
    __syncwarp();
    if (issued < W.count) issue(s);  // the buffer's reads are complete (syncwarp)
    cc.next(probs, done + 1 < W.count);
  }
  // leave no copy in flight (only after an expired wait; default bound)
  for (int k = done; k < issued; ++k) mbar_wait(&sm.bar[k % kSymStages], (k / kSymStages) & 1);
}

template <int CAP>
void configure_psymv_as() {
  raise_smem_limit(reinterpret_cast<const void*>(k_psymv<double, 1, CAP>), sym_smem<1>(kSymWarpsMax));
  raise_smem_limit(reinterpret_cast<const void*>(k_psymv<float, 1, CAP>), sym_smem<1>(kSymWarpsMax));
  raise_smem_limit(reinterpret_cast<const void*>(k_psymv<double, 2, CAP>), sym_smem<2>(kSymWarpsMax));
  raise_smem_limit(reinterpret_cast<const void*>(k_psymv<double, 3, CAP>), sym_smem<3>(kSymWarpsMax));
}

void configure_psymv() {
  configure_psymv_as<0>();
  configure_psymv_as<1>();
}

template <class T, int NF>
void launch_psymv_as(const T* pack, const SymProblem* probs, const SymWarp* warps, int nwarps, const double* X,
                     double* Y, int rstride, size_t fstride, int nz, int* status, unsigned long long wait_ns,
                     int wpb, int regcap, bool pdl, cudaStream_t st) {
  const int blocks = (nwarps + wpb - 1) / wpb;
  if (regcap)
    launch_ex(pdl, k_psymv<T, NF, 1>, dim3(blocks), dim3(32 * wpb), sym_smem<NF>(wpb), st, pack, probs, warps,
              nwarps, X, Y, rstride, fstride, nz, status, wait_ns);
  else
    launch_ex(pdl, k_psymv<T, NF, 0>, dim3(blocks), dim3(32 * wpb), sym_smem<NF>(wpb), st, pack, probs, warps,
              nwarps, X, Y, rstride, fstride, nz, status, wait_ns);
}

cudaError_t launch_psymv(const DevModal& S, const SymProblem* probs, const SymWarp* warps, int nwarps,
                         const double* X, double* Y, int rstride, int nz, bool fp32, cudaStream_t st, int nf = 1,
                         size_t fstride = 0) {
  if (nwarps <= 0) return cudaSuccess;
  configure_psymv();
  if (fp32)
    launch_psymv_as<float, 1>(S.l2_pack32, probs, warps, nwarps, X, Y, rstride, 0, nz, S.status, S.wait_ns, S.sym_warps, S.sym_regcap, S.pdl != 0, st);
  else if (nf == 3)
    launch_psymv_as<double, 3>(S.l2_pack, probs, warps, nwarps, X, Y, rstride, fstride, nz, S.status, S.wait_ns, S.sym_warps, S.sym_regcap, S.pdl != 0, st);
  else if (nf == 2)
    launch_psymv_as<double, 2>(S.l2_pack, probs, warps, nwarps, X, Y, rstride, fstride, nz, S.status, S.wait_ns, S.sym_warps, S.sym_regcap, S.pdl != 0, st);
  else
    launch_psymv_as<double, 1>(S.l2_pack, probs, warps, nwarps, X, Y, rstride, 0, nz, S.status, S.wait_ns, S.sym_warps, S.sym_regcap, S.pdl != 0, st);
  return cudaGetLastError();
}

}  // namespace

namespace {

__global__ void k_zero_ranges(ZeroRanges z, size_t total) {
  pdl_trigger();
  pdl_wait();
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    size_t j = i;
    int r = 0;
    while (r + 1 < z.count && j >= z.n[r]) j -= z.n[r++];
    z.p[r][j] = 0.0;
  }
}

}  // namespace

cudaError_t zero_ranges(bool pdl, const ZeroRanges& z, cudaStream_t st) {
  size_t n = 0;
  for (int r = 0; r < z.count; ++r) n += z.n[r];
  if (n == 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 148 * 8));
  return launch_ex(pdl, k_zero_ranges, dim3(blocks), dim3(256), 0, st, z, n);
}

cudaError_t zero_ranges(bool pdl, double* a, size_t na, double* b, size_t nb, cudaStream_t st) {
  ZeroRanges z;
  z.add(a, na);
  z.add(b, nb);
  return zero_ranges(pdl, z, st);
}

size_t twolevel_workspace_doubles(int rstride, int nz) { return static_cast<size_t>(rstride) * nz; }

cudaError_t twolevel_solve(const DevModal& S, const DevGeom& g, const DevNumbering& N, double* R, int rstride,
                           double* work, int nz, cudaStream_t st, cudaEvent_t mid, bool fp32, bool y_zeroed) {
  double* Yv = twolevel_solution(work, rstride, nz);  // y_I, then the whole skeleton solution
  // planes of the launch's modes
  const int k0 = nz > 1 ? 2 * S.mode0 : 0, k1 = nz > 1 ? std::min(nz, 2 * (S.mode0 + S.nmodes)) : 1;
  cudaError_t err = y_zeroed ? cudaSuccess
                             : zero_ranges(S.pdl != 0, Yv + static_cast<size_t>(rstride) * k0,
                                           static_cast<size_t>(rstride) * (k1 - k0), nullptr, 0, st);
  if (err != cudaSuccess) return err;
  // y_I = S_II^-1 R_I; r_B = R_B - S_BI y_I
  err = launch_psymv(S, S.prob_patch, S.warp_patch, S.nwarp_patch, R, Yv, rstride, nz, fp32, st);
  if (err != cudaSuccess) return err;
  element_schur_apply(0, g, N, S, Yv, R, rstride, st);
  // x_B = A^-1 r_B (into the interface positions of Y)
  err = launch_psymv(S, S.prob_iface, S.warp_iface, S.nwarp_iface, R, Yv, rstride, nz, fp32, st);
  if (err != cudaSuccess) return err;
  if (mid) cudaEventRecord(mid, st);
  // x_I = y_I - G x_B, G = S_II^-1 S_IB
  err = launch_psymv(S, S.prob_gen, S.warp_gen, S.nwarp_gen, Yv, Yv, rstride, nz, fp32, st);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

cudaError_t twolevel_solve_fields(const DevModal& S, const DevGeom& g, const DevNumbering& N, double* R,
                                  double* Y, size_t fstride, int nf, int rstride, int nz, cudaStream_t st,
                                  bool y_zeroed) {
  if (nf < 1 || nf > 3 || S.refine > 0 || S.l2_pack32) return cudaErrorInvalidValue;
  const int k0 = nz > 1 ? 2 * S.mode0 : 0, k1 = nz > 1 ? std::min(nz, 2 * (S.mode0 + S.nmodes)) : 1;
  cudaError_t err = cudaSuccess;
  if (!y_zeroed) {
    ZeroRanges z;
    for (int f = 0; f < nf; ++f)
      z.add(Y + f * fstride + static_cast<size_t>(rstride) * k0, static_cast<size_t>(rstride) * (k1 - k0));
    err = zero_ranges(S.pdl != 0, z, st);
  }
  if (err != cudaSuccess) return err;
  err = launch_psymv(S, S.prob_patch, S.warp_patch, S.nwarp_patch, R, Y, rstride, nz, false, st, nf, fstride);
  if (err != cudaSuccess) return err;
  for (int f = 0; f < nf; ++f) element_schur_apply(0, g, N, S, Y + f * fstride, R + f * fstride, rstride, st);
  err = launch_psymv(S, S.prob_iface, S.warp_iface, S.nwarp_iface, R, Y, rstride, nz, false, st, nf, fstride);
  if (err != cudaSuccess) return err;
  err = launch_psymv(S, S.prob_gen, S.warp_gen, S.nwarp_gen, Y, Y, rstride, nz, false, st, nf, fstride);
  if (err != cudaSuccess) return err;
  return cudaGetLastError();
}

int twolevel_launches(const DevModal& S) {
  return (S.nwarp_patch > 0 ? 1 : 0) + (S.nwarp_iface > 0 ? 1 : 0) + (S.nwarp_gen > 0 ? 1 : 0) + 1;
}

static int prob_ntiles(const SymProblem& P) { return P.ncol ? gen_ntiles(P.n, P.ncol) : sym_ntiles(P.n); }

std::vector<SymWarp> sym_schedule(const std::vector<SymProblem>& probs, int device, int wpb, int occ_pct,
                                  int regcap) {
  std::vector<SymWarp> out;
  long long total = 0;
  for (const auto& P : probs) total += prob_ntiles(P);
  if (total == 0) return out;
  int sms = 148, per_sm = 1;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  configure_psymv();
  const void* kern = regcap ? reinterpret_cast<const void*>(k_psymv<double, 1, 1>)
                            : reinterpret_cast<const void*>(k_psymv<double, 1, 0>);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * wpb, sym_smem<1>(wpb)) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  // warps of one full wave at the kernel's occupancy, times occ_pct / 100
  const long long wave = static_cast<long long>(sms) * per_sm * wpb;
  const long long nw = std::max<long long>(1, std::min<long long>(total, wave * occ_pct / 100));
  size_t p = 0;
  long long before = 0;  // tiles of problems [0, p)
  for (long long w = 0; w < nw; ++w) {
    const long long t0 = total * w / nw, t1 = total * (w + 1) / nw;
    while (before + prob_ntiles(probs[p]) <= t0) before += prob_ntiles(probs[p++]);
    out.push_back(SymWarp{static_cast<int>(p), static_cast<int>(t0 - before), static_cast<int>(t1 - t0)});
  }
  return out;
}

}  // namespace stx
