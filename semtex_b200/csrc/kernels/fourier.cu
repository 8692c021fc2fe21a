// z-direction real DFT of field planes (AuxField::transform,
// src/auxfield.cpp:1157-1194, contract of femlib/fourier.c:40-165).
//
// Forward (sign +1), scaled by 1/nz:  c_k = (1/nz) sum_n x_n exp(-2 pi i k n / nz),
// packed per point as [Re c_0, Re c_{nz/2}, Re c_1, Im c_1, Re c_2, ...].
// Inverse (sign -1):  x_n = c_0 + c_{nz/2} (-1)^n + 2 sum_k (Re c_k cos - Im c_k sin).
// nz == 2 follows the reference special case (forward zeroes plane 1,
// inverse copies plane 0 to plane 1).
//
// The reference layout keeps the z-lines strided by plane_size, so a block
// owns 32 consecutive points of every plane: loads and stores of each plane
// row are coalesced, and the transform runs out of shared memory.
#include "helmholtz.cuh"

namespace stx {

namespace {

constexpr int kTP = 32;  // points per block

__global__ void k_dft(double* __restrict__ data, int nz, int plane_size, int sign,
                      const double* __restrict__ twiddle) {
  extern __shared__ double sm[];
  double* x = sm;             // [nz][kTP]
  double* tw = sm + nz * kTP; // [2][nz]
  const int p0 = blockIdx.x * kTP;
  for (int t = threadIdx.x; t < 2 * nz; t += blockDim.x) tw[t] = twiddle[t];
  for (int t = threadIdx.x; t < nz * kTP; t += blockDim.x) {
    const int k = t / kTP, p = t - k * kTP;
    x[t] = (p0 + p < plane_size) ? data[static_cast<size_t>(k) * plane_size + p0 + p] : 0.0;
  }
  __syncthreads();
  const int half = nz >> 1;
  const double scale = 1.0 / nz;
  for (int t = threadIdx.x; t < nz * kTP; t += blockDim.x) {
    const int q = t / kTP, p = t - q * kTP;
    double v = 0.0;
    if (sign > 0) {
      const int kf = q == 0 ? 0 : (q == 1 ? half : q >> 1);
      const bool im = q >= 2 && (q & 1);
      int idx = 0;
      for (int n = 0; n < nz; ++n) {
        v += x[n * kTP + p] * (im ? -tw[nz + idx] : tw[idx]);
        idx += kf;
        if (idx >= nz) idx -= nz;
      }
      v *= scale;
    } else {
      const int n = q;
      v = x[p] + ((n & 1) ? -x[kTP + p] : x[kTP + p]);
      int idx = n, step = n;
      for (int k = 1; k < half; ++k) {
        v += 2.0 * (x[(2 * k) * kTP + p] * tw[idx] - x[(2 * k + 1) * kTP + p] * tw[nz + idx]);
        idx += step;
        if (idx >= nz) idx -= nz;
      }
    }
    sm[nz * kTP + 2 * nz + t] = v;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nz * kTP; t += blockDim.x) {
    const int k = t / kTP, p = t - k * kTP;
    if (p0 + p < plane_size)
      data[static_cast<size_t>(k) * plane_size + p0 + p] = sm[nz * kTP + 2 * nz + t];
  }
}

__global__ void k_nz2(double* data, int plane_size, int sign) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= plane_size) return;
  data[plane_size + p] = sign > 0 ? 0.0 : data[p];
}

}  // namespace

cudaError_t z_transform(double* data, int nz, int plane_size, int sign, const double* twiddle,
                        double* /*work*/, cudaStream_t st) {
  if (nz < 2) return cudaSuccess;
  if (nz == 2) {
    k_nz2<<<(plane_size + 255) / 256, 256, 0, st>>>(data, plane_size, sign);
    return cudaGetLastError();
  }
  const size_t shm = sizeof(double) * (2 * static_cast<size_t>(nz) * kTP + 2 * nz);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_dft, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  k_dft<<<(plane_size + kTP - 1) / kTP, 256, shm, st>>>(data, nz, plane_size, sign, twiddle);
  return cudaGetLastError();
}

}  // namespace stx
