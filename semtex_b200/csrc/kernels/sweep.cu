// Batched block sweeps and the device assembly of the two-level systems
// (see sweep.cuh).  All FP64; every kernel's index arithmetic stays inside
// the n x n (or ld x ld) matrices it is given, n and ld multiples of 64.
#include "sweep.cuh"

#include <cmath>

#include "launch.hpp"
#include "symtile.hpp"

namespace stx {

namespace {

constexpr int kT = kSwBlk;          // tile order
constexpr int kTT = kT * kT;        // doubles per tile
constexpr int kThreads = 256;       // 16 x 16 threads, 4 x 4 outputs each

// Tile (i, j), i >= j, of the lower-triangle enumeration t = i (i + 1) / 2 + j.
__device__ __forceinline__ void tri_index(int t, int& i, int& j) {
  int r = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (r * (r + 1) / 2 > t) --r;
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  i = r;
  j = t - r * (r + 1) / 2;
}

// Invert the pivot block D = A[K, K] of every matrix by a scalar sweep in
// shared memory: Dv[b] = D^-1 (64 x 64, row-major).
__global__ void __launch_bounds__(kThreads) k_sweep_diag(const double* __restrict__ A, int n, long long stride,
                                                         int K, double* __restrict__ Dv, int* status) {
  extern __shared__ double sm[];
  double* M = sm;               // [64][65]
  double* cp = sm + kT * (kT + 1);  // pivot column
  const int b = blockIdx.x;
  const double* Ab = A + b * stride;
  const size_t k0 = static_cast<size_t>(K) * kT;
  for (int e = threadIdx.x; e < kTT; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    M[r * (kT + 1) + c] = r >= c ? Ab[(k0 + r) * n + k0 + c] : Ab[(k0 + c) * n + k0 + r];
  }
  bool bad = false;
  __syncthreads();
  for (int p = 0; p < kT; ++p) {
    if (threadIdx.x < kT) cp[threadIdx.x] = M[threadIdx.x * (kT + 1) + p];
    __syncthreads();
    double d = cp[p];
    if (!(d > 0.0)) {
      bad = true;
      d = 1.0;
    }
    const double inv = 1.0 / d;
    for (int e = threadIdx.x; e < kTT; e += blockDim.x) {
      const int r = e >> 6, c = e & 63;
      double v;
      if (r == p && c == p) v = -inv;
      else if (r == p) v = cp[c] * inv;
      else if (c == p) v = cp[r] * inv;
      else v = M[r * (kT + 1) + c] - cp[r] * cp[c] * inv;
      M[r * (kT + 1) + c] = v;
    }
    __syncthreads();
  }
  double* D = Dv + static_cast<size_t>(b) * kTT;
  for (int e = threadIdx.x; e < kTT; e += blockDim.x) D[e] = -M[(e >> 6) * (kT + 1) + (e & 63)];
  if (bad && threadIdx.x == 0) atomicExch(status, 1);
}

// Panel of pivot block K: for every tile row i != K, Q_i = A[i, K] (the
// original coupling, from the lower triangle) and P_i = Q_i D^-1, both stored
// transposed: QT[k][r] = Q_i[r][k], PT[k][r] = P_i[r][k].
__global__ void __launch_bounds__(kThreads) k_sweep_panel(const double* __restrict__ A, int n, long long stride,
                                                          int K, const double* __restrict__ Dv,
                                                          double* __restrict__ QT, double* __restrict__ PT) {
  extern __shared__ double sm[];
  double* Qs = sm;                  // [k][65]: Qs[k][r] = Q_i[r][k]
  double* Ds = sm + kT * (kT + 1);  // [k][65]: D^-1[k][c]
  const int i = blockIdx.x, b = blockIdx.y, nblk = gridDim.x;
  if (i == K) return;
  const double* Ab = A + b * stride;
  const size_t i0 = static_cast<size_t>(i) * kT, k0 = static_cast<size_t>(K) * kT;
  for (int e = threadIdx.x; e < kTT; e += blockDim.x) {
    const int hi = e >> 6, lo = e & 63;
    if (i > K)  // tile (i, K): rows of block i, coalesced along k
      Qs[lo * (kT + 1) + hi] = Ab[(i0 + hi) * n + k0 + lo];
    else        // tile (K, i) transposed, coalesced along r
      Qs[hi * (kT + 1) + lo] = Ab[(k0 + hi) * n + i0 + lo];
    Ds[hi * (kT + 1) + lo] = Dv[static_cast<size_t>(b) * kTT + e];
  }
  __syncthreads();
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double acc[4][4] = {};
  for (int k = 0; k < kT; ++k) {
    double q[4], d[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) q[a] = Qs[k * (kT + 1) + ty * 4 + a];
#pragma unroll
    for (int c = 0; c < 4; ++c) d[c] = Ds[k * (kT + 1) + tx * 4 + c];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = fma(q[a], d[c], acc[a][c]);
  }
  const size_t t0 = (static_cast<size_t>(b) * nblk + i) * kTT;
  for (int e = threadIdx.x; e < kTT; e += blockDim.x) QT[t0 + e] = Qs[(e >> 6) * (kT + 1) + (e & 63)];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) PT[t0 + static_cast<size_t>(tx * 4 + c) * kT + ty * 4 + a] = acc[a][c];
}

// Update of the lower tiles (i, j) for pivot block K:
//   i, j != K:  A_ij -= P_i Q_j^T
//   j == K:     A_iK  = P_i
//   i == K:     A_Kj  = P_j^T
//   i = j = K:  A_KK  = -D^-1
__global__ void __launch_bounds__(kThreads) k_sweep_update(double* __restrict__ A, int n, long long stride, int K,
                                                           const double* __restrict__ Dv,
                                                           const double* __restrict__ QT,
                                                           const double* __restrict__ PT, int nblk) {
  extern __shared__ __align__(16) double sm[];
  int i, j;
  tri_index(blockIdx.x, i, j);
  const int b = blockIdx.y;
  double* Ab = A + b * stride;
  const size_t i0 = static_cast<size_t>(i) * kT, j0 = static_cast<size_t>(j) * kT;
  const size_t pb = static_cast<size_t>(b) * nblk;
  if (i == K || j == K) {
    for (int e = threadIdx.x; e < kTT; e += blockDim.x) {
      const int r = e >> 6, c = e & 63;
      double v;
      if (i == K && j == K) v = -Dv[static_cast<size_t>(b) * kTT + e];
      else if (j == K) v = PT[(pb + i) * kTT + static_cast<size_t>(c) * kT + r];  // P_i[r][c]
      else v = PT[(pb + j) * kTT + static_cast<size_t>(r) * kT + c];              // P_j[c][r]
      Ab[(i0 + r) * n + j0 + c] = v;
    }
    return;
  }
  double* Ps = sm;        // [k][64] = P_i[r][k]
  double* Qs = sm + kTT;  // [k][64] = Q_j[c][k]
  const double2* pg = reinterpret_cast<const double2*>(PT + (pb + i) * kTT);
  const double2* qg = reinterpret_cast<const double2*>(QT + (pb + j) * kTT);
  for (int e = threadIdx.x; e < kTT / 2; e += blockDim.x) {
    reinterpret_cast<double2*>(Ps)[e] = pg[e];
    reinterpret_cast<double2*>(Qs)[e] = qg[e];
  }
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = Ab[(i0 + ty * 4 + a) * n + j0 + tx * 4 + c];
  __syncthreads();
  for (int k = 0; k < kT; ++k) {
    const double2 p0 = *reinterpret_cast<const double2*>(Ps + k * kT + ty * 4);
    const double2 p1 = *reinterpret_cast<const double2*>(Ps + k * kT + ty * 4 + 2);
    const double2 q0 = *reinterpret_cast<const double2*>(Qs + k * kT + tx * 4);
    const double2 q1 = *reinterpret_cast<const double2*>(Qs + k * kT + tx * 4 + 2);
    const double p[4] = {p0.x, p0.y, p1.x, p1.y}, q[4] = {q0.x, q0.y, q1.x, q1.y};
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = fma(-p[a], q[c], acc[a][c]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) Ab[(i0 + ty * 4 + a) * n + j0 + tx * 4 + c] = acc[a][c];
}

__global__ void k_patch_assemble(PatchAssembly p, double* __restrict__ A, long long stride) {
  const int m = blockIdx.x;
  double* Am = A + m * stride;
  const int ld = p.ld;
  for (int q = threadIdx.x; q < ld; q += blockDim.x)
    if ((q >= p.nI && q < p.pI) || q >= p.pI + p.nB) Am[static_cast<size_t>(q) * ld + q] = 1.0;
  const int nx = p.next, nn = nx * nx;
  for (int k = 0; k < p.nelem; ++k) {
    const double* h = p.hbb + (static_cast<size_t>(m) * p.nfamily + p.efam[k]) * nn;
    const int* loc = p.local + static_cast<size_t>(k) * nx;
    for (int e = threadIdx.x; e < nn; e += blockDim.x) {
      const int a = e / nx, c = e - a * nx;
      const int la = loc[a], lc = loc[c];
      if (la < 0 || lc < 0) continue;
      const int ra = la < p.nI ? la : p.pI + la - p.nI;
      const int rc = lc < p.nI ? lc : p.pI + lc - p.nI;
      // a periodic element may meet itself: two of its nodes can share a row
      atomicAdd(&Am[static_cast<size_t>(ra) * ld + rc], h[e]);
    }
    __syncthreads();
  }
  if (p.mixI)
    for (int q = threadIdx.x; q < p.nI; q += blockDim.x) Am[static_cast<size_t>(q) * ld + q] += p.mixI[q];
}

__global__ void k_iface_scatter(const double* __restrict__ T, long long tstride, int tld, int pI, int nB,
                                const int* __restrict__ iid, double* __restrict__ A, long long astride, int ald) {
  const int m = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nB * nB) return;
  const int a = e / nB, c = e - a * nB;
  const double* Tm = T + m * tstride;
  const size_t ra = static_cast<size_t>(pI) + a, rc = static_cast<size_t>(pI) + c;
  const double v = a >= c ? Tm[ra * tld + rc] : Tm[rc * tld + ra];
  // interface ids of one patch are distinct: no two threads share an entry
  A[m * astride + static_cast<size_t>(iid[a]) * ald + iid[c]] += v;
}

__global__ void k_iface_finish(double* __restrict__ A, long long stride, int ld, int ni,
                               const double* __restrict__ diag, const int* __restrict__ pin) {
  const int m = blockIdx.y;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ld) return;
  double* Am = A + m * stride;
  const int pn = pin ? pin[m] : -1;
  if (q >= ni) {
    Am[static_cast<size_t>(q) * ld + q] = 1.0;
    return;
  }
  if (diag) Am[static_cast<size_t>(q) * ld + q] += diag[q];
  if (pn >= 0) {
    // row and column pn become an identity: the pinned unknown is zero
    Am[static_cast<size_t>(pn) * ld + q] = q == pn ? 1.0 : 0.0;
    Am[static_cast<size_t>(q) * ld + pn] = q == pn ? 1.0 : 0.0;
  }
}

// Position of packed entry o of the symtile layout of order n.
__device__ __forceinline__ void sym_entry(int n, long long o, int& i, int& j, bool& pad) {
  const int T = sym_tiles(n);
  const long long full = static_cast<long long>(kSymTile) * kSymLd;
  const long long first = static_cast<long long>(T - 1) * T / 2 * full;
  int I, J;
  long long w;
  if (o < first) {
    const int q = static_cast<int>(o / full);
    tri_index(q, I, J);
    w = o - q * full;
  } else {
    const long long rows = sym_rows_stored(n, T - 1);
    const long long o2 = o - first;
    I = T - 1;
    J = static_cast<int>(o2 / (rows * kSymLd));
    w = o2 - J * rows * kSymLd;
  }
  int r, c;
  tile_rc(static_cast<int>(w), r, c);
  i = kSymTile * I + r;
  j = kSymTile * J + c;
  pad = c >= kSymTile || r >= sym_rows(n, I) || j >= n;
}

__global__ void k_pack_sym(const double* __restrict__ A, long long stride, int lda, int n, double sign,
                           double* __restrict__ out, const long long* __restrict__ off, long long total) {
  const int m = blockIdx.y;
  const long long o = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= total) return;
  int i, j;
  bool pad;
  sym_entry(n, o, i, j, pad);
  double v = 0.0;
  if (!pad) {
    const double* Am = A + m * stride;
    v = sign * (i >= j ? Am[static_cast<size_t>(i) * lda + j] : Am[static_cast<size_t>(j) * lda + i]);
  }
  out[off[m] + o] = v;
}

__global__ void k_pack_gen_t(const double* __restrict__ A, long long stride, int lda, int r0, int nr, int nc,
                             double* __restrict__ out, const long long* __restrict__ off, long long total) {
  const int m = blockIdx.y;
  const long long o = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (o >= total) return;
  const int Tr = sym_tiles(nr), Tc = sym_tiles(nc);
  const long long full = static_cast<long long>(kSymTile) * kSymLd;
  const long long first = static_cast<long long>(Tr - 1) * Tc * full;
  int I, J;
  long long w;
  if (o < first) {
    const long long q = o / full;
    I = static_cast<int>(q / Tc);
    J = static_cast<int>(q - static_cast<long long>(I) * Tc);
    w = o - q * full;
  } else {
    const long long rows = sym_rows_stored(nr, Tr - 1);
    const long long o2 = o - first;
    I = Tr - 1;
    J = static_cast<int>(o2 / (rows * kSymLd));
    w = o2 - J * rows * kSymLd;
  }
  int r, c;
  tile_rc(static_cast<int>(w), r, c);
  const int a = kSymTile * I + r, bcol = kSymTile * J + c;
  double v = 0.0;
  if (c < kSymTile && r < sym_rows(nr, I) && bcol < nc)
    v = A[m * stride + static_cast<size_t>(r0 + bcol) * lda + a];
  out[off[m] + o] = v;
}

__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = static_cast<float>(in[i]);
}

}  // namespace

size_t sweep_scratch_doubles(int n, int batch) {
  const size_t nblk = static_cast<size_t>(n) / kT;
  return static_cast<size_t>(batch) * kTT * (1 + 2 * nblk);
}

cudaError_t sym_sweep(double* A, int n, long long stride, int batch, int npiv, double* scratch, int* status,
                      cudaStream_t st) {
  if (n <= 0 || npiv <= 0 || batch <= 0) return cudaSuccess;
  if (n % kT || npiv % kT || npiv > n) return cudaErrorInvalidValue;
  const int nblk = n / kT;
  double* Dv = scratch;
  double* QT = Dv + static_cast<size_t>(batch) * kTT;
  double* PT = QT + static_cast<size_t>(batch) * nblk * kTT;
  const size_t sm_diag = sizeof(double) * (kT * (kT + 1) + kT);
  const size_t sm_panel = sizeof(double) * 2 * kT * (kT + 1);
  const size_t sm_upd = sizeof(double) * 2 * kTT;
  raise_smem_limit(reinterpret_cast<const void*>(k_sweep_diag), sm_diag);
  raise_smem_limit(reinterpret_cast<const void*>(k_sweep_panel), sm_panel);
  raise_smem_limit(reinterpret_cast<const void*>(k_sweep_update), sm_upd);
  const int ntri = nblk * (nblk + 1) / 2;
  for (int K = 0; K < npiv / kT; ++K) {
    k_sweep_diag<<<batch, kThreads, sm_diag, st>>>(A, n, stride, K, Dv, status);
    k_sweep_panel<<<dim3(nblk, batch), kThreads, sm_panel, st>>>(A, n, stride, K, Dv, QT, PT);
    k_sweep_update<<<dim3(ntri, batch), kThreads, sm_upd, st>>>(A, n, stride, K, Dv, QT, PT, nblk);
  }
  return cudaGetLastError();
}

cudaError_t patch_assemble(const PatchAssembly& p, double* A, long long stride, int nmodes, cudaStream_t st) {
  if (nmodes <= 0) return cudaSuccess;
  k_patch_assemble<<<nmodes, 256, 0, st>>>(p, A, stride);
  return cudaGetLastError();
}

cudaError_t interface_scatter(const double* T, long long tstride, int tld, int pI, int nB, const int* iid,
                              double* A, long long astride, int ald, int nmodes, cudaStream_t st) {
  if (nB <= 0 || nmodes <= 0) return cudaSuccess;
  k_iface_scatter<<<dim3((nB * nB + 255) / 256, nmodes), 256, 0, st>>>(T, tstride, tld, pI, nB, iid, A, astride,
                                                                       ald);
  return cudaGetLastError();
}

cudaError_t interface_finish(double* A, long long stride, int ld, int niface, const double* diag, const int* pin,
                             int nmodes, cudaStream_t st) {
  if (ld <= 0 || nmodes <= 0) return cudaSuccess;
  k_iface_finish<<<dim3((ld + 255) / 256, nmodes), 256, 0, st>>>(A, stride, ld, niface, diag, pin);
  return cudaGetLastError();
}

cudaError_t pack_sym(const double* A, long long stride, int lda, int n, double sign, double* out,
                     const long long* off, int nmodes, cudaStream_t st) {
  const long long total = sym_size(n);
  if (total <= 0 || nmodes <= 0) return cudaSuccess;
  k_pack_sym<<<dim3(static_cast<unsigned>((total + 255) / 256), nmodes), 256, 0, st>>>(A, stride, lda, n, sign,
                                                                                      out, off, total);
  return cudaGetLastError();
}

cudaError_t pack_gen_t(const double* A, long long stride, int lda, int r0, int nr, int nc, double* out,
                       const long long* off, int nmodes, cudaStream_t st) {
  const long long total = gen_size(nr, nc);
  if (total <= 0 || nmodes <= 0) return cudaSuccess;
  k_pack_gen_t<<<dim3(static_cast<unsigned>((total + 255) / 256), nmodes), 256, 0, st>>>(A, stride, lda, r0, nr,
                                                                                        nc, out, off, total);
  return cudaGetLastError();
}

cudaError_t to_float(const double* in, float* out, size_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_to_float<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(in, out, n);
  return cudaGetLastError();
}

}  // namespace stx
