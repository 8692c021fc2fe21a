// Two-level condensed solve of the skeleton system (all planes at once).
//
// After the element-level condensation has produced the skeleton right-hand
// side R (Element::local2globalSumSC, src/element.cpp:326-365), the reference
// solves the banded skeleton system with dpbtrs (src/field.cpp:693).  Here
// the same system is solved through patch-level condensation:
//   r_iface  = R[iface] - sum_patches G_p^T R[I_p]
//   x_iface  = A^{-1} r_iface                     (dense, per mode)
//   x_I      = S_II^{-1} R[I_p] - G_p x_iface      (per patch)
// Every step is a batched dense matrix-vector product; the Re and Im planes
// of a mode share each matrix read.
#include "twolevel.cuh"

namespace stx {

namespace {

// ri[k][i] = R[k][skel_of[i]], zero at a singular mode's pinned node.
__global__ void k_iface_gather(DevModal S, const double* __restrict__ R, int rstride, double* __restrict__ Ri,
                               int istride, int nz) {
  const int k = blockIdx.y;
  if (nz > 1 && k == 1) return;
  const int pin = S.pin[k >> 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.niface; i += gridDim.x * blockDim.x)
    Ri[static_cast<size_t>(k) * istride + i] = i == pin ? 0.0 : R[static_cast<size_t>(k) * rstride + S.skel_of[i]];
}

// Ri[k][B_p] -= G_p^T R[k][I_p]   (one block per patch and plane)
__global__ void k_l2_condense(DevModal S, const double* __restrict__ R, int rstride, double* __restrict__ Ri,
                              int istride, int nz) {
  extern __shared__ double sr[];
  const int p = blockIdx.x, k = blockIdx.y;
  if (nz > 1 && k == 1) return;
  const int m = k >> 1;
  const int nI = S.p_nI[p], nB = S.p_nB[p], f = S.p_family[p];
  const int* Ig = S.p_Igid + static_cast<size_t>(p) * S.nI_max;
  const int* Bi = S.p_Biid + static_cast<size_t>(p) * S.nB_max;
  for (int i = threadIdx.x; i < nI; i += blockDim.x) sr[i] = R[static_cast<size_t>(k) * rstride + Ig[i]];
  __syncthreads();
  const double* G = S.l2_g + (static_cast<size_t>(m) * S.pfam + f) * S.nI_max * S.nB_max;
  const int pin = S.pin[m];
  for (int b = threadIdx.x; b < nB; b += blockDim.x) {
    double v = 0.0, v2 = 0.0;
    int i = 0;
#pragma unroll 8
    for (; i + 1 < nI; i += 2) {
      v = fma(G[static_cast<size_t>(i) * S.nB_max + b], sr[i], v);
      v2 = fma(G[static_cast<size_t>(i + 1) * S.nB_max + b], sr[i + 1], v2);
    }
    if (i < nI) v = fma(G[static_cast<size_t>(i) * S.nB_max + b], sr[i], v);
    v += v2;
    const int iid = Bi[b];
    if (iid != pin) atomicAdd(&Ri[static_cast<size_t>(k) * istride + iid], -v);
  }
}

// Xi = A^{-1} Ri for the planes of each mode: a block computes 8 rows with a
// warp per row, lanes across columns, both planes per matrix read.
constexpr int kRowsPerBlock = 8;

__global__ void __launch_bounds__(32 * kRowsPerBlock) k_iface_gemv(DevModal S, const double* __restrict__ Ri,
                                                                   double* __restrict__ Xi, int istride, int nz) {
  extern __shared__ double sx[];  // [2][niface]
  const int m = blockIdx.y;
  const int n = S.niface;
  const int nr = (nz > 1 && m > 0) ? 2 : 1;
  const double* x0 = Ri + static_cast<size_t>(2 * m) * istride;
  const double* x1 = Ri + static_cast<size_t>(2 * m + 1) * istride;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sx[i] = x0[i];
    if (nr > 1) sx[n + i] = x1[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * kRowsPerBlock + warp;
  if (row >= n) return;
  const double* A = S.l2_ainv + static_cast<size_t>(m) * n * n + static_cast<size_t>(row) * n;
  double s0 = 0.0, s1 = 0.0;
  if (nr > 1) {
#pragma unroll 8
    for (int c = lane; c < n; c += 32) {
      const double a = __ldg(A + c);
      s0 = fma(a, sx[c], s0);
      s1 = fma(a, sx[n + c], s1);
    }
  } else {
#pragma unroll 8
    for (int c = lane; c < n; c += 32) s0 = fma(__ldg(A + c), sx[c], s0);
  }
  for (int o = 16; o; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (lane == 0) {
    Xi[static_cast<size_t>(2 * m) * istride + row] = s0;
    if (nr > 1) Xi[static_cast<size_t>(2 * m + 1) * istride + row] = s1;
  }
}

// R[k][I_p] = S_II^{-1} R[k][I_p] - G_p Xi[k][B_p]   (one block per patch and plane)
__global__ void k_l2_recover(DevModal S, double* __restrict__ R, int rstride, const double* __restrict__ Xi,
                             int istride, int nz) {
  extern __shared__ double sm[];
  const int p = blockIdx.x, k = blockIdx.y;
  if (nz > 1 && k == 1) return;
  const int m = k >> 1;
  const int nI = S.p_nI[p], nB = S.p_nB[p], f = S.p_family[p];
  const int* Ig = S.p_Igid + static_cast<size_t>(p) * S.nI_max;
  const int* Bi = S.p_Biid + static_cast<size_t>(p) * S.nB_max;
  double* sr = sm;
  double* sb = sm + S.nI_max;
  for (int i = threadIdx.x; i < nI; i += blockDim.x) sr[i] = R[static_cast<size_t>(k) * rstride + Ig[i]];
  for (int b = threadIdx.x; b < nB; b += blockDim.x) sb[b] = Xi[static_cast<size_t>(k) * istride + Bi[b]];
  __syncthreads();
  const size_t fm = static_cast<size_t>(m) * S.pfam + f;
  const double* Si = S.l2_sinv + fm * S.nI_max * S.nI_max;  // symmetric: read columns
  const double* GT = S.l2_gt + fm * S.nB_max * S.nI_max;
  for (int i = threadIdx.x; i < nI; i += blockDim.x) {
    double v = 0.0;
    for (int j = 0; j < nI; ++j) v = fma(Si[static_cast<size_t>(j) * S.nI_max + i], sr[j], v);
    for (int b = 0; b < nB; ++b) v = fma(-GT[static_cast<size_t>(b) * S.nI_max + i], sb[b], v);
    R[static_cast<size_t>(k) * rstride + Ig[i]] = v;
  }
}

// R[k][skel_of[i]] = Xi[k][i]
__global__ void k_iface_scatter(DevModal S, double* __restrict__ R, int rstride, const double* __restrict__ Xi,
                                int istride, int nz) {
  const int k = blockIdx.y;
  if (nz > 1 && k == 1) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.niface; i += gridDim.x * blockDim.x)
    R[static_cast<size_t>(k) * rstride + S.skel_of[i]] = Xi[static_cast<size_t>(k) * istride + i];
}

}  // namespace

size_t twolevel_workspace_doubles(const DevModal& S, int nz) {
  const size_t is = (static_cast<size_t>(S.niface) + 31) / 32 * 32;
  return 2 * is * nz;
}

cudaError_t twolevel_solve(const DevModal& S, double* R, int rstride, double* work, int nz, cudaStream_t st) {
  const int istride = (S.niface + 31) / 32 * 32;
  double* Ri = work;
  double* Xi = work + static_cast<size_t>(istride) * nz;
  const int ib = std::max(1, std::min(64, (S.niface + 255) / 256));
  if (S.niface) k_iface_gather<<<dim3(ib, nz), 256, 0, st>>>(S, R, rstride, Ri, istride, nz);
  const int pt = std::max(64, std::min(256, (std::max(S.nI_max, S.nB_max) + 31) / 32 * 32));
  if (S.niface)
    k_l2_condense<<<dim3(S.npatch, nz), pt, sizeof(double) * S.nI_max, st>>>(S, R, rstride, Ri, istride, nz);
  if (S.niface) {
    const size_t shm = sizeof(double) * 2 * S.niface;
    static size_t configured = 0;
    if (shm > 48 * 1024 && shm > configured) {
      cudaFuncSetAttribute(k_iface_gemv, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm));
      configured = shm;
    }
    k_iface_gemv<<<dim3((S.niface + kRowsPerBlock - 1) / kRowsPerBlock, S.nmodes), 32 * kRowsPerBlock, shm, st>>>(
        S, Ri, Xi, istride, nz);
  }
  k_l2_recover<<<dim3(S.npatch, nz), pt, sizeof(double) * (S.nI_max + S.nB_max), st>>>(S, R, rstride, Xi, istride,
                                                                                      nz);
  if (S.niface) k_iface_scatter<<<dim3(ib, nz), 256, 0, st>>>(S, R, rstride, Xi, istride, nz);
  return cudaGetLastError();
}

int twolevel_launches(const DevModal& S) { return S.niface ? 5 : 1; }

}  // namespace stx
