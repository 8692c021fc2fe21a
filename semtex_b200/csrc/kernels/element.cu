// Element kernels: one block per (chunk of up to chunk_max same-family
// elements, Fourier mode, row block of the family operator).  The forcing
// columns of the chunk (Re and Im planes of the mode; boundary-major node
// order for the condensation, natural order for the recovery, whose operator
// columns are permuted to match on the host) are assembled in shared memory;
// the family-mode operator slice is bulk-copied alongside; the product runs
// on the FP64 tensor cores (m8n8k4), one warp per 8-row by 32-column unit.
//
// Latency, not bandwidth, bounds this work (a few MB per launch), so every
// global -> shared transfer is asynchronous (8-byte cp.async, one bulk copy
// of the operator) and the index-dependent loads of a warp are issued for
// several columns at once.
#include "element.cuh"

#include <algorithm>

#include "launch.hpp"
#include "ptx.cuh"

namespace stx {

namespace {

constexpr int kColBatch = 4;  // columns per warp whose index loads are in flight together
constexpr int kMaxWarps = 32;
constexpr int kUnitTiles = 4;  // 8x8 tiles per warp unit of the product: 8 rows x 32 columns

struct ElemSmem {
  size_t a, b, d, q, flag, bits, idx, num, bytes;
};

// [mbarrier | A rows | B columns | D | Q4 / lift scratch | column flags |
//  override bits | pmap, emap, chunk elements | the chunk's btog, bmask]
__host__ __device__ inline ElemSmem elem_layout(int a_doubles, int cm, int ldb, int np, int nn, int next, bool lift) {
  ElemSmem L;
  L.a = 16;
  L.b = L.a + sizeof(double) * static_cast<size_t>(a_doubles);
  L.d = L.b + sizeof(double) * 2 * static_cast<size_t>(cm) * ldb;
  L.q = L.d + sizeof(double) * static_cast<size_t>(np) * np;
  const size_t q4 = static_cast<size_t>(cm) * nn, scratch = lift ? static_cast<size_t>(24) * nn : 0;
  const size_t qd = q4 > scratch ? q4 : scratch;
  L.flag = L.q + sizeof(double) * qd;
  L.bits = L.flag + sizeof(int) * 2 * static_cast<size_t>(cm);
  const int nwords = (next + 31) / 32;
  L.idx = L.bits + sizeof(unsigned) * 2 * static_cast<size_t>(cm) * nwords;
  L.num = L.idx + sizeof(int) * (static_cast<size_t>(nn) + nn + cm);
  L.bytes = (L.num + sizeof(int) * 2 * static_cast<size_t>(cm) * next + 15) / 16 * 16;
  return L;
}

// Small index tables in shared memory (the asynchronous copies stream
// through L1, so global index reads would go back to L2 every time), the
// chunk's numbering included: set-up data, loaded before the kernel waits
// for its predecessor.
struct ElemIdx {
  const int* pmap;   // [nn] boundary-major position of node t
  const int* emap;   // [nn] node at boundary-major position p
  const int* el;     // [cnt] the chunk's elements
  const int* btog;   // [cnt][next] global number of boundary node a of chunk element l
  const int* bmask;  // [cnt][next] its essential flag
};

__device__ __forceinline__ ElemIdx load_idx(const DevGeom& g, const DevNumbering& N, unsigned char* sraw,
                                            const ElemSmem& L, const int* el, int cnt) {
  int* sp = reinterpret_cast<int*>(sraw + L.idx);
  int* se = sp + g.npnp;
  int* sl = se + g.npnp;
  int* sb = reinterpret_cast<int*>(sraw + L.num);
  int* sm = sb + static_cast<size_t>(cnt) * g.next;
  for (int t = threadIdx.x; t < g.npnp; t += blockDim.x) {
    sp[t] = __ldg(g.pmap + t);
    se[t] = __ldg(g.emap + t);
  }
  for (int l = threadIdx.x; l < cnt; l += blockDim.x) sl[l] = __ldg(el + l);
  for (int q = threadIdx.x; q < cnt * g.next; q += blockDim.x) {
    const int l = q / g.next, a = q - l * g.next;
    const int e = __ldg(el + l);
    sb[q] = __ldg(N.btog + e * g.next + a);
    sm[q] = __ldg(N.bmask + e * g.next + a);
  }
  return ElemIdx{sp, se, sl, sb, sm};
}

// Row of node t of a column: natural node order or boundary-major order.
template <bool kNatural>
__device__ __forceinline__ int node_row(const ElemIdx& X, int t) {
  return kNatural ? t : X.pmap[t];
}

__device__ __forceinline__ void col_slot(int col, int cnt, int& slot, int& l) {
  slot = col >= cnt ? 1 : 0;  // at most two planes (Re, Im) per mode
  l = col - slot * cnt;
}

// Thread 0: initialise the mbarrier and start the bulk copy of the operator
// rows (bytes a multiple of 16, 16-byte aligned source).
__device__ __forceinline__ void stage_rows(uint64_t* bar, double* sA, const double* src, unsigned bytes) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(bar, bytes);
    const char* s = reinterpret_cast<const char*>(src);
    char* d = reinterpret_cast<char*>(sA);
    for (unsigned off = 0; off < bytes; off += 32768u) bulk_g2s(d + off, s + off, min(32768u, bytes - off), bar);
  }
}

// All threads: wait, bounded by `limit_ns`, for the operator rows; false
// (uniformly) when the bound expired, after the error is recorded and a
// second wait (bounded by the default 2 s) for the copy still in flight.
__device__ __forceinline__ bool rows_ready(uint64_t* bar, int* status, unsigned long long limit_ns) {
  const bool ok = __syncthreads_and(mbar_wait(bar, 0, limit_ns));
  if (!ok) {
    if (threadIdx.x == 0 && status) atomicExch(status, 3);
    mbar_wait(bar, 0);
  }
  return ok;
}

// Issue the asynchronous copies of the forcing columns, natural node order
// (f at the nodes whose boundary-major position p satisfies p >= pmin), and
// of the elements' Q4 at the same nodes; zero the padding rows [nn, ldb) of
// every column.  A warp's copies of a column are contiguous in both memories.
template <bool kNatural>
__device__ __forceinline__ void issue_forcing(const DevGeom& g, const double* __restrict__ F, const ElemIdx& X,
                                              int cnt, int m, int ncol, double* sB, int ldb, double* sQ, int pmin) {
  const int nn = g.npnp;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  for (int col = wp; col < ncol; col += nwp) {
    int slot, l;
    col_slot(col, cnt, slot, l);
    const int e = X.el[l];
    const double* f = F + static_cast<size_t>(2 * m + slot) * g.plane_size + static_cast<size_t>(e) * nn;
    const double* q4 = g.Q4 + static_cast<size_t>(e) * nn;
    double* b = sB + col * ldb;
    for (int t = ln; t < nn; t += 32) {
      if (X.pmap[t] < pmin) continue;
      cp_async8(b + node_row<kNatural>(X, t), f + t);
      if (slot == 0) cp_async8(sQ + l * nn + t, q4 + t);
    }
    for (int r = nn + ln; r < ldb; r += 32) b[r] = 0.0;
  }
}

// After the copies: forcing column entries become -Q4 f.
template <bool kNatural>
__device__ __forceinline__ void scale_forcing(const DevGeom& g, const ElemIdx& X, int cnt, int ncol, double* sB,
                                              int ldb, const double* sQ, int pmin) {
  const int nn = g.npnp;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  for (int col = wp; col < ncol; col += nwp) {
    int slot, l;
    col_slot(col, cnt, slot, l);
    double* b = sB + col * ldb;
    for (int t = ln; t < nn; t += 32)
      if (X.pmap[t] >= pmin) b[node_row<kNatural>(X, t)] *= -sQ[l * nn + t];
  }
}

// Boundary scan of the chunk's columns, index loads of kColBatch columns per
// warp in flight together.  For every column: flag = the element carries a
// nonzero essential value in this plane (its lift term is then formed).
// With `gather` (recovery): boundary rows of the column receive the solved
// skeleton values u_b (asynchronous copy; 0 at essential and pinned nodes),
// and essential values are written straight to U, with a bit per node
// telling the final write-out to leave them.
template <bool kGather>
__device__ void scan_boundary(const DevGeom& g, const DevNumbering& N, const double* __restrict__ G, int gstride,
                              const double* __restrict__ R, int rstride, double* __restrict__ U, int nsolve,
                              const ElemIdx& X, int cnt, int m, int ncol, double* sB, int ldb, int* sFlag,
                              unsigned* sBits) {
  const int next = g.next, nn = g.npnp;
  const int nwords = (next + 31) / 32;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  for (int c0 = wp; c0 < ncol; c0 += nwp * kColBatch) {
    bool nz[kColBatch];
#pragma unroll
    for (int j = 0; j < kColBatch; ++j) nz[j] = false;
    for (int a0 = 0; a0 < next; a0 += 64) {
      int gi[kColBatch][2], bm[kColBatch][2];
#pragma unroll
      for (int j = 0; j < kColBatch; ++j) {
        const int col = c0 + j * nwp;
        int slot, l;
        col_slot(min(col, ncol - 1), cnt, slot, l);
        const int eb = l * next;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int a = a0 + 32 * h + ln;
          const bool ok = col < ncol && a < next;
          gi[j][h] = ok ? X.btog[eb + a] : -1;
          bm[j][h] = (ok && G) ? X.bmask[eb + a] : 0;
        }
      }
      double gv[kColBatch][2];
#pragma unroll
      for (int j = 0; j < kColBatch; ++j) {
        const int col = c0 + j * nwp;
        const int k = 2 * m + (col >= cnt ? 1 : 0);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          gv[j][h] = bm[j][h] ? G[static_cast<size_t>(k) * gstride + gi[j][h]] : 0.0;
          if (kGather && gi[j][h] >= 0) {
            const int a = a0 + 32 * h + ln;
            const int t = X.emap[a];
            if (gi[j][h] < nsolve) cp_async8(sB + col * ldb + t, R + static_cast<size_t>(k) * rstride + gi[j][h]);
            else sB[col * ldb + t] = 0.0;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kColBatch; ++j) {
        const int col = c0 + j * nwp;
#pragma unroll
        for (int h = 0; h < 2; ++h) nz[j] = nz[j] || gv[j][h] != 0.0;
        if (kGather) {
          int slot, l;
          col_slot(min(col, ncol - 1), cnt, slot, l);
          const int e = X.el[l];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int a = a0 + 32 * h + ln;
            const bool ovr = bm[j][h] != 0;  // essential node: its value comes from G
            if (ovr && U)
              U[static_cast<size_t>(2 * m + slot) * g.plane_size + static_cast<size_t>(e) * nn + X.emap[a]] =
                  gv[j][h];
            const unsigned word = __ballot_sync(0xffffffffu, ovr);
            if (ln == 0 && col < ncol && (a0 + 32 * h) < next) sBits[col * nwords + (a0 + 32 * h) / 32] = word;
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kColBatch; ++j) {
      const int col = c0 + j * nwp;
      const bool any = __any_sync(0xffffffffu, nz[j]);
      if (ln == 0 && col < ncol) sFlag[col] = any;
    }
  }
}

// Lift term H g of the flagged columns, subtracted from their forcing (at
// all nodes, or only interior ones): one column per warp among the first 8
// warps, each with 3*nn doubles of scratch in wsc.
template <bool kNatural>
__device__ void lift_columns(const DevGeom& g, const DevNumbering& N, const double* __restrict__ G, int gstride,
                             double hcon, const ElemIdx& X, int cnt, int m, int ncol, double* sB, int ldb,
                             double* wsc, const double* sD, const int* sFlag, int pmin) {
  const int nn = g.npnp, np = g.np, next = g.next;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = min(8, static_cast<int>(blockDim.x >> 5));
  if (warp >= nwarp) return;
  double* su = wsc + static_cast<size_t>(warp) * 3 * nn;
  double* sR = su + nn;
  double* sS = sR + nn;
  for (int col = warp; col < ncol; col += nwarp) {
    if (!sFlag[col]) continue;
    int slot, l;
    col_slot(col, cnt, slot, l);
    const int e = X.el[l];
    const double* Gp = G + static_cast<size_t>(2 * m + slot) * gstride;
    for (int q = lane; q < nn; q += 32) su[q] = 0.0;
    __syncwarp();
    for (int q = lane; q < next; q += 32)
      if (X.bmask[l * next + q]) su[X.emap[q]] = Gp[X.btog[l * next + q]];
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
      if (X.pmap[q] < pmin) continue;
      const int i = q / np, j = q - (q / np) * np;
      double h = g.Q4[e * nn + q] * su[q] * hcon;
      for (int kk = 0; kk < np; ++kk) {
        h += sD[kk * np + i] * sS[kk * np + j];
        h += sR[i * np + kk] * sD[kk * np + j];
      }
      sB[col * ldb + node_row<kNatural>(X, q)] -= h;
    }
    __syncwarp();
  }
}

// acc[j] = tile j0+j (8x8) of the warp's 8-row strip: A[strip rows][0:K)
// B[tile columns][boff : boff + K), K a multiple of 4; rows and columns past
// the ends are clamped (their results are discarded).
__device__ __forceinline__ void unit_product(double (&acc)[kUnitTiles][2], const double* sA, int lda, int rows,
                                             int strip, const double* sB, int ldb, int ncol, int j0, int ntile,
                                             int boff, int K) {
  const int ln = threadIdx.x & 31, g8 = ln >> 2, t4 = ln & 3;
  const double* ap = sA + min(strip * 8 + g8, rows - 1) * lda + t4;
  const double* bp[kUnitTiles];
#pragma unroll
  for (int j = 0; j < kUnitTiles; ++j) bp[j] = sB + min((j0 + j) * 8 + g8, ncol - 1) * ldb + boff + t4;
#pragma unroll
  for (int j = 0; j < kUnitTiles; ++j) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll 4
  for (int k0 = 0; k0 < K; k0 += 4) {
    const double a = ap[k0];
#pragma unroll
    for (int j = 0; j < kUnitTiles; ++j)
      if (j0 + j < ntile) dmma_8x8x4(acc[j][0], acc[j][1], a, bp[j][k0]);
  }
}

__global__ void __launch_bounds__(32 * kMaxWarps, 1)
    k_elem_condense(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ F, const double* __restrict__ G,
                    int gstride, double* __restrict__ R, int rstride, int rb_rows) {
  extern __shared__ __align__(16) unsigned char sraw[];
  pdl_trigger();
  const int c = blockIdx.x, m = S.mode0 + blockIdx.y;
  const int nr = (g.nz > 1 && m > 0) ? 2 : 1;
  const int nn = g.npnp, next = g.next;
  const int4 cd = __ldg(g.chunk_desc + c);  // start, count, family
  const int cnt = cd.y;
  const int ncol = nr * cnt;
  const int* el = g.elem_sorted + cd.x;
  const int ldb = element_ld(nn), lda = S.eb_ld;
  const int r_lo = blockIdx.z * rb_rows, rows = min(rb_rows, next - r_lo);
  const ElemSmem L = elem_layout(rb_rows * lda, g.chunk_max, ldb, g.np, nn, next, G != nullptr);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sraw);
  double* sA = reinterpret_cast<double*>(sraw + L.a);
  double* sB = reinterpret_cast<double*>(sraw + L.b);
  double* sD = reinterpret_cast<double*>(sraw + L.d);
  double* sQ = reinterpret_cast<double*>(sraw + L.q);
  int* sFlag = reinterpret_cast<int*>(sraw + L.flag);
  const size_t fm = static_cast<size_t>(m) * S.nfamily + cd.z;
  stage_rows(bar, sA, S.eb + (fm * next + r_lo) * lda, static_cast<unsigned>(sizeof(double) * rows * lda));
  const ElemIdx X = load_idx(g, N, sraw, L, el, cnt);
  for (int w = threadIdx.x; w < g.np * g.np; w += blockDim.x) sD[w] = S.D[w];
  __syncthreads();
  pdl_wait();  // the operator rows are set-up data; F, G and R come from earlier kernels
  // boundary-major columns: the product takes the interior rows, F_b stays
  issue_forcing<false>(g, F, X, cnt, m, ncol, sB, ldb, sQ, 0);
  if (G)
    scan_boundary<false>(g, N, G, gstride, nullptr, 0, nullptr, 0, X, cnt, m, ncol, sB, ldb, sFlag, nullptr);
  cp_async_wait_all();
  __syncthreads();
  scale_forcing<false>(g, X, cnt, ncol, sB, ldb, sQ, 0);
  // lift terms only where some column carries a nonzero essential value
  if (__syncthreads_or(G && threadIdx.x < ncol && sFlag[threadIdx.x])) {
    lift_columns<false>(g, N, G, gstride, S.lambda2[m] + S.betak2[m], X, cnt, m, ncol, sB, ldb, sQ, sD, sFlag, 0);
    __syncthreads();
  }
  if (!rows_ready(bar, S.status, S.wait_ns)) return;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const int ntile = (ncol + 7) / 8, strips = (rows + 7) / 8;
  const int ncg = (ntile + kUnitTiles - 1) / kUnitTiles;
  const int K = (g.nint + 3) / 4 * 4;
  for (int unit = wp; unit < strips * ncg; unit += blockDim.x >> 5) {
    const int strip = unit / ncg, j0 = (unit - strip * ncg) * kUnitTiles;
    double acc[kUnitTiles][2];
    unit_product(acc, sA, lda, rows, strip, sB, ldb, ncol, j0, ntile, next, K);
    const int row = strip * 8 + (ln >> 2);
#pragma unroll
    for (int j = 0; j < kUnitTiles; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int col = (j0 + j) * 8 + 2 * (ln & 3) + i;
        if (j0 + j < ntile && row < rows && col < ncol) {
          int slot, l;
          col_slot(col, cnt, slot, l);
          const int b = r_lo + row;
          atomicAdd(&R[static_cast<size_t>(2 * m + slot) * rstride + X.btog[l * next + b]],
                    sB[col * ldb + b] - acc[j][i]);
        }
      }
  }
}

__global__ void __launch_bounds__(32 * kMaxWarps, 1)
    k_elem_recover(DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ F, const double* __restrict__ G,
                   int gstride, const double* __restrict__ R, int rstride, double* __restrict__ U, int rb_rows) {
  extern __shared__ __align__(16) unsigned char sraw[];
  pdl_trigger();
  const int c = blockIdx.x, m = S.mode0 + blockIdx.y;
  const int nr = (g.nz > 1 && m > 0) ? 2 : 1;
  const int nn = g.npnp, next = g.next, nint = g.nint;
  const int4 cd = __ldg(g.chunk_desc + c);  // start, count, family
  const int cnt = cd.y;
  const int ncol = nr * cnt;
  const int* el = g.elem_sorted + cd.x;
  const int ldb = element_ld(nn), lda = S.ew_ld;
  const int r_lo = blockIdx.z * rb_rows, rows = min(rb_rows, nint - r_lo);
  const ElemSmem L = elem_layout(rb_rows * lda, g.chunk_max, ldb, g.np, nn, next, G != nullptr);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sraw);
  double* sA = reinterpret_cast<double*>(sraw + L.a);
  double* sB = reinterpret_cast<double*>(sraw + L.b);
  double* sD = reinterpret_cast<double*>(sraw + L.d);
  double* sQ = reinterpret_cast<double*>(sraw + L.q);
  int* sFlag = reinterpret_cast<int*>(sraw + L.flag);
  unsigned* sBits = reinterpret_cast<unsigned*>(sraw + L.bits);
  const int nwords = (next + 31) / 32;
  const size_t fm = static_cast<size_t>(m) * S.nfamily + cd.z;
  stage_rows(bar, sA, S.ew + (fm * nint + r_lo) * lda, static_cast<unsigned>(sizeof(double) * rows * lda));
  const ElemIdx X = load_idx(g, N, sraw, L, el, cnt);
  for (int w = threadIdx.x; w < g.np * g.np; w += blockDim.x) sD[w] = S.D[w];
  __syncthreads();
  pdl_wait();  // F, G, R (and U's other writers) belong to earlier kernels
  // interior forcing only: the boundary rows carry u_b
  issue_forcing<true>(g, F, X, cnt, m, ncol, sB, ldb, sQ, next);
  const int nsolve = S.nsolve[m];
  // every row block gathers u_b (it enters every row's product); only row
  // block 0 writes the essential values
  scan_boundary<true>(g, N, G, gstride, R, rstride, blockIdx.z == 0 ? U : nullptr, nsolve, X, cnt, m, ncol, sB,
                      ldb, sFlag, sBits);
  cp_async_wait_all();
  __syncthreads();
  scale_forcing<true>(g, X, cnt, ncol, sB, ldb, sQ, next);
  // lift terms only where some column carries a nonzero essential value
  if (__syncthreads_or(G && threadIdx.x < ncol && sFlag[threadIdx.x])) {
    lift_columns<true>(g, N, G, gstride, S.lambda2[m] + S.betak2[m], X, cnt, m, ncol, sB, ldb, sQ, sD, sFlag, next);
    __syncthreads();
  }
  if (!rows_ready(bar, S.status, S.wait_ns)) return;
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  const int ntile = (ncol + 7) / 8, strips = (rows + 7) / 8;
  const int ncg = (ntile + kUnitTiles - 1) / kUnitTiles;
  const int K = (nn + 3) / 4 * 4;
  double acc[kUnitTiles][2];
  const bool active = wp < strips * ncg;  // the plan gives every unit its own warp
  const int strip = wp / ncg, j0 = (wp - strip * ncg) * kUnitTiles;
  if (active) unit_product(acc, sA, lda, rows, strip, sB, ldb, ncol, j0, ntile, 0, K);
  __syncthreads();  // every read of the columns is done
  if (active) {
    const int row = strip * 8 + (ln >> 2);
#pragma unroll
    for (int j = 0; j < kUnitTiles; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int col = (j0 + j) * 8 + 2 * (ln & 3) + i;
        if (j0 + j < ntile && row < rows && col < ncol) sB[col * ldb + X.emap[next + r_lo + row]] = acc[j][i];
      }
  }
  __syncthreads();
  for (int col = wp; col < ncol; col += nwp) {
    int slot, l;
    col_slot(col, cnt, slot, l);
    double* u_e = U + static_cast<size_t>(2 * m + slot) * g.plane_size + static_cast<size_t>(X.el[l]) * nn;
    const double* b = sB + col * ldb;
    const unsigned* bits = sBits + col * nwords;
    for (int t = ln; t < nn; t += 32) {
      const int p = X.pmap[t];
      const bool w = p >= next ? (p - next >= r_lo && p - next < r_lo + rows)
                               : (blockIdx.z == 0 && !((bits[p >> 5] >> (p & 31)) & 1u));
      if (w) u_e[t] = b[t];
    }
  }
}


// Element Schur complement products: one block per (chunk, mode).  The
// family-mode matrix S_e (rows padded) and the chunk's input columns (the
// source values at the element nodes of the taken class, zero elsewhere)
// in shared memory; out = S_e x on the tensor cores; the rows of the put
// class are subtracted from dst.  dir 0: patch-interior -> interface,
// 1: interface -> patch-interior, 2: every non-essential node both ways
// (dst -= S x, the skeleton residual).
__global__ void __launch_bounds__(256)
    k_elem_schur(int dir, DevGeom g, DevNumbering N, DevModal S, const double* __restrict__ src,
                 double* __restrict__ dst, int rstride) {
  extern __shared__ __align__(16) unsigned char sraw[];
  pdl_trigger();
  const int c = blockIdx.x, m = S.mode0 + blockIdx.y;
  const int nr = (g.nz > 1 && m > 0) ? 2 : 1;
  // this block's part of the chunk: elements [e0, e0 + cnt)
  const int4 cd = __ldg(g.chunk_desc + c);  // start, count, family
  const int e0 = cd.y * blockIdx.z / gridDim.z, cnt = cd.y * (blockIdx.z + 1) / gridDim.z - e0;
  const int next = g.next, ncol = nr * cnt;
  const int lda = S.l2_sc_ld, ldb = element_ld(next);
  double* sA = reinterpret_cast<double*>(sraw);               // [next][lda]
  double* sB = sA + next * lda;                               // [2 cm][ldb]
  int* sN = reinterpret_cast<int*>(sB + 2 * g.chunk_max * ldb);  // [cm][next] skeleton id << 2 | class
  const int take = dir == 0 ? 1 : 2, put = dir == 0 ? 2 : 1;
  const bool every = dir == 2;
  const double* A = S.l2_sc + (static_cast<size_t>(m) * S.nfamily + cd.z) * next * lda;
  for (int i = threadIdx.x; i < next * lda; i += blockDim.x) sA[i] = __ldg(A + i);
  const int wp = threadIdx.x >> 5, ln = threadIdx.x & 31, nwp = blockDim.x >> 5;
  const int* code = S.l2_ncode + static_cast<size_t>(cd.x + e0) * next;
  for (int i = threadIdx.x; i < cnt * next; i += blockDim.x) sN[i] = __ldg(code + i);
  __syncthreads();
  pdl_wait();  // S_e and the node codes are set-up data; src and dst are not
  // input columns, loads of kColBatch columns per warp in flight together
  for (int c0 = wp; c0 < ncol; c0 += nwp * kColBatch) {
    double v[kColBatch][2];
#pragma unroll
    for (int j = 0; j < kColBatch; ++j) {
      const int col = c0 + j * nwp;
      int slot, l;
      col_slot(min(col, ncol - 1), cnt, slot, l);
      const double* sp = src + static_cast<size_t>(2 * m + slot) * rstride;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int a = ln + 32 * h;
        const int code_v = (col < ncol && a < next) ? sN[l * next + a] : 0;
        v[j][h] = (every ? (code_v & 3) != 0 : (code_v & 3) == take) ? sp[code_v >> 2] : 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < kColBatch; ++j) {
      const int col = c0 + j * nwp;
      if (col >= ncol) continue;
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (ln + 32 * h < next) sB[col * ldb + ln + 32 * h] = v[j][h];
    }
  }
  __syncthreads();
  const int ntile = (ncol + 7) / 8, strips = (next + 7) / 8;
  const int ncg = (ntile + kUnitTiles - 1) / kUnitTiles;
  for (int unit = wp; unit < strips * ncg; unit += nwp) {
    const int strip = unit / ncg, j0 = (unit - strip * ncg) * kUnitTiles;
    double acc[kUnitTiles][2];
    unit_product(acc, sA, lda, next, strip, sB, ldb, ncol, j0, ntile, 0, next);
    const int row = strip * 8 + (ln >> 2);
#pragma unroll
    for (int j = 0; j < kUnitTiles; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int col = (j0 + j) * 8 + 2 * (ln & 3) + i;
        if (j0 + j < ntile && row < next && col < ncol) {
          int slot, l;
          col_slot(col, cnt, slot, l);
          const int code_v = sN[l * next + row];
          if (every ? (code_v & 3) != 0 : (code_v & 3) == put)
            atomicAdd(&dst[static_cast<size_t>(2 * m + slot) * rstride + (code_v >> 2)], -acc[j][i]);
        }
      }
  }
}
}  // namespace

ElementPlan element_plan(const DevGeom& g, const DevModal& S, bool lift) {
  ElementPlan P;
  if (g.nchunk <= 0 || !S.ew || !S.eb || S.ew_ld <= 0 || S.eb_ld <= 0 || g.nint <= 0) return P;
  const int ldb = element_ld(g.npnp);
  const int ncg = ((2 * g.chunk_max + 7) / 8 + kUnitTiles - 1) / kUnitTiles;
  // Two blocks of 16 warps per SM (<= 113 KB each), so that one block's
  // gathers overlap the other's product, when the whole operator fits;
  // otherwise one block of 32 warps per SM, operator rows split into
  // balanced row blocks where needed.
  auto fit = [&](int nrow, int ld, int warps, size_t cap, int& rows, int& nrb, int& threads, size_t& smem) {
    rows = std::min(nrow, 8 * (warps / ncg));  // one warp per product unit
    if (rows < nrow) rows -= rows % 8;
    for (;;) {
      smem = elem_layout(rows * ld, g.chunk_max, ldb, g.np, g.npnp, g.next, lift).bytes;
      if (smem <= cap) break;
      rows = rows % 8 ? rows - rows % 8 : rows - 8;
      if (rows < 8) return false;
    }
    nrb = (nrow + rows - 1) / rows;
    if (nrb > 1) {  // balance: equal row blocks, multiples of 8
      rows = ((nrow + nrb - 1) / nrb + 7) / 8 * 8;
      nrb = (nrow + rows - 1) / rows;
      smem = elem_layout(rows * ld, g.chunk_max, ldb, g.np, g.npnp, g.next, lift).bytes;
    }
    threads = 32 * warps;
    return (rows + 7) / 8 * ncg <= warps && smem <= cap;
  };
  // per kernel: the two-block tier only when it needs no row split, unless
  // S.elem_twoblock asks for it with row blocks (each gathers every column
  // of its chunk: more blocks and two per SM, for more gather traffic)
  auto choose = [&](int nrow, int ld, int& rows, int& nrb, int& threads, size_t& smem) {
    if (fit(nrow, ld, kMaxWarps / 2, 113 * 1024, rows, nrb, threads, smem) && (nrb == 1 || S.elem_twoblock))
      return true;
    return fit(nrow, ld, kMaxWarps, 227 * 1024, rows, nrb, threads, smem);
  };
  P.ok = choose(g.next, S.eb_ld, P.cond_rows, P.cond_rb, P.cond_threads, P.cond_smem) &&
         choose(g.nint, S.ew_ld, P.rec_rows, P.rec_rb, P.rec_threads, P.rec_smem);
  return P;
}

void element_condense(const ElementPlan& P, const DevGeom& g, const DevNumbering& N, const DevModal& S,
                      const double* F, const double* G, int gstride, double* R, int rstride, cudaStream_t st) {
  raise_smem_limit(reinterpret_cast<const void*>(k_elem_condense), P.cond_smem);
  launch_ex(S.pdl != 0, k_elem_condense, dim3(g.nchunk, S.nmodes, P.cond_rb), dim3(P.cond_threads), P.cond_smem, st,
            g, N, S, F, G, gstride, R, rstride, P.cond_rows);
}

void element_recover(const ElementPlan& P, const DevGeom& g, const DevNumbering& N, const DevModal& S,
                     const double* F, const double* G, int gstride, const double* R, int rstride, double* U,
                     cudaStream_t st) {
  raise_smem_limit(reinterpret_cast<const void*>(k_elem_recover), P.rec_smem);
  launch_ex(S.pdl != 0, k_elem_recover, dim3(g.nchunk, S.nmodes, P.rec_rb), dim3(P.rec_threads), P.rec_smem, st, g,
            N, S, F, G, gstride, R, rstride, U, P.rec_rows);
}

void element_schur_apply(int dir, const DevGeom& g, const DevNumbering& N, const DevModal& S, const double* src,
                         double* dst, int rstride, cudaStream_t st) {
  const size_t smem = sizeof(double) * (static_cast<size_t>(g.next) * S.l2_sc_ld +
                                        2 * static_cast<size_t>(g.chunk_max) * element_ld(g.next)) +
                      sizeof(int) * static_cast<size_t>(g.chunk_max) * g.next;
  raise_smem_limit(reinterpret_cast<const void*>(k_elem_schur), smem);
  // two blocks per chunk and mode: the work is latency-bound
  launch_ex(S.pdl != 0, k_elem_schur, dim3(g.nchunk, S.nmodes, 2), dim3(256), smem, st, dir, g, N, S, src, dst,
            rstride);
}

}  // namespace stx
