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
#include "launch.hpp"
#include "ptx.cuh"

namespace stx {

namespace {

constexpr int kTP = 32;  // points per block

__global__ void k_dft(double* __restrict__ data, int nz, int plane_size, int sign,
                      const double* __restrict__ twiddle) {
  pdl_trigger();
  pdl_wait();
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

// ---------------------------------------------------------------------------
// Mixed-radix Stockham FFT (radices 4, 2, 3, 5) of the z-lines of TP
// consecutive points per block, complex arithmetic in shared memory
// ([n][p] layout, point index fastest, so global loads and stores of each
// plane row stay coalesced).  Forward: real lines in, packed spectrum out,
// scaled by 1/nz; inverse: packed spectrum expanded to its Hermitian form,
// real lines out.  Twiddles w^m = exp(-2 pi i m / nz) come from the same
// host-computed table as the DFT's.
// ---------------------------------------------------------------------------

// Radices of the stages, 4 bits each from the lowest (read with shifts: a
// kernel parameter indexed at run time would be copied to local memory).
struct FftPlan {
  int nf;
  unsigned long long radices;
  __device__ int dradix(int f) const { return static_cast<int>((radices >> (4 * f)) & 15u); }
};

__device__ __forceinline__ void cmul(double& ar, double& ai, double br, double bi) {
  const double r = ar * br - ai * bi;
  ai = ar * bi + ai * br;
  ar = r;
}

// In-place length-R DFT of (vr, vi) with exponent sign s (-1 forward).
template <int R>
__device__ __forceinline__ void small_dft(double* vr, double* vi, double s) {
  if (R == 2) {
    const double ar = vr[0], ai = vi[0];
    vr[0] = ar + vr[1];
    vi[0] = ai + vi[1];
    vr[1] = ar - vr[1];
    vi[1] = ai - vi[1];
  } else if (R == 4) {
    const double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
    const double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
    const double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
    const double t3r = vr[1] - vr[3], t3i = vi[1] - vi[3];
    // multiply t3 by s*i: (x + iy) * (s i) = -s y + i s x
    const double ur = -s * t3i, ui = s * t3r;
    vr[0] = t0r + t2r;
    vi[0] = t0i + t2i;
    vr[2] = t0r - t2r;
    vi[2] = t0i - t2i;
    vr[1] = t1r + ur;
    vi[1] = t1i + ui;
    vr[3] = t1r - ur;
    vi[3] = t1i - ui;
  } else if (R == 3) {
    const double c = -0.5, sn = s * 0.86602540378443864676;  // sin(2 pi / 3)
    const double sr = vr[1] + vr[2], si = vi[1] + vi[2];
    const double dr = vr[1] - vr[2], di = vi[1] - vi[2];
    const double ar = vr[0] + c * sr, ai = vi[0] + c * si;
    vr[0] += sr;
    vi[0] += si;
    // (dr + i di) * (i sn) = -sn di + i sn dr
    vr[1] = ar - sn * di;
    vi[1] = ai + sn * dr;
    vr[2] = ar + sn * di;
    vi[2] = ai - sn * dr;
  } else if (R == 5) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;   // cos(2pi/5), cos(4pi/5)
    const double s1 = s * 0.95105651629515357212, s2 = s * 0.58778525229247312917;  // sin(2pi/5), sin(4pi/5)
    const double a1r = vr[1] + vr[4], a1i = vi[1] + vi[4], b1r = vr[1] - vr[4], b1i = vi[1] - vi[4];
    const double a2r = vr[2] + vr[3], a2i = vi[2] + vi[3], b2r = vr[2] - vr[3], b2i = vi[2] - vi[3];
    const double x0r = vr[0], x0i = vi[0];
    const double p1r = x0r + c1 * a1r + c2 * a2r, p1i = x0i + c1 * a1i + c2 * a2i;
    const double p2r = x0r + c2 * a1r + c1 * a2r, p2i = x0i + c2 * a1i + c1 * a2i;
    // q = i * (s1 b1 + s2 b2), r = i * (s2 b1 - s1 b2)
    const double q1r = -(s1 * b1i + s2 * b2i), q1i = s1 * b1r + s2 * b2r;
    const double q2r = -(s2 * b1i - s1 * b2i), q2i = s2 * b1r - s1 * b2r;
    vr[0] = x0r + a1r + a2r;
    vi[0] = x0i + a1i + a2i;
    vr[1] = p1r + q1r;
    vi[1] = p1i + q1i;
    vr[4] = p1r - q1r;
    vi[4] = p1i - q1i;
    vr[2] = p2r + q2r;
    vi[2] = p2i + q2i;
    vr[3] = p2r - q2r;
    vi[3] = p2i - q2i;
  }
}

// One radix-R stage over TP complex lines whose rows are LD doubles apart.
template <int R, int TP, int LD>
__device__ __forceinline__ void stockham_stage(const double* xr, const double* xi, double* yr, double* yi, int N,
                                               int Ns, const double* tw, double s) {
  constexpr int tp = TP;
  const int nj = N / R;
  for (int w = threadIdx.x; w < nj * tp; w += blockDim.x) {
    const int j = w / tp, p = w - j * tp;
    const int k = j % Ns;
    double vr[R], vi[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      vr[r] = xr[(j + r * nj) * LD + p];
      vi[r] = xi[(j + r * nj) * LD + p];
    }
    // twiddle exp(s 2 pi i r k / (Ns R)) = table entry r*k*N/(Ns R) (< N)
    const int step = N / (Ns * R);
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const int m = r * k * step;
      cmul(vr[r], vi[r], tw[m], s * tw[N + m]);  // exp(s i theta) = cos + s i sin
    }
    small_dft<R>(vr, vi, s);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      yr[(base + r * Ns) * LD + p] = vr[r];
      yi[(base + r * Ns) * LD + p] = vi[r];
    }
  }
}

// Set when a bounded wait of k_fft for its bulk copies expired (the block
// then leaves its lines untransformed).
__device__ int g_fft_timeout = 0;

}  // namespace

int fft_timeout_flag() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_fft_timeout, sizeof(int)) != cudaSuccess) return -1;
  return v;
}

const int* fft_timeout_address() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_fft_timeout) != cudaSuccess) return nullptr;
  return static_cast<const int*>(p);
}

namespace {

// Real transforms of TPL z-lines per block as TPL/2 complex transforms: the
// block's rows [n][TPL] are read as complex lines z = x_p + i x_{p+TPL/2}
// (real part columns 0..TPL/2-1, imaginary part the rest); the two real
// spectra are separated afterwards through Hermitian symmetry (forward), or
// combined before the transform (inverse).  bulk != 0: the rows (16-byte
// aligned) arrive by bulk copies issued by one warp on one mbarrier.
template <int TPL>
__global__ void k_fft(double* __restrict__ data, int nz, int plane_size, int sign, const double* __restrict__ twiddle,
                      FftPlan plan, int bulk) {
  pdl_trigger();
  pdl_wait();
  constexpr int TPC = TPL / 2, LD = TPL;
  extern __shared__ __align__(16) double sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
  double* tw = sm + 2;                   // [2][nz]
  double* A = tw + 2 * nz;               // two [nz][LD] buffers
  double* B = A + nz * LD;
  const int p0 = blockIdx.x * TPL;
  const int cnt = min(TPL, plane_size - p0);
  const int N = nz, half = nz / 2;
  double* land = sign > 0 ? A : B;       // plane rows as stored: real lines, or the packed spectra
  if (bulk) {
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(bar, static_cast<unsigned>(sizeof(double) * nz * cnt));
    }
    __syncthreads();  // armed before any copy can complete
    if (threadIdx.x < 32)
      for (int n = threadIdx.x; n < nz; n += 32)
        bulk_g2s(land + n * LD, data + static_cast<size_t>(n) * plane_size + p0,
                 static_cast<unsigned>(sizeof(double) * cnt), bar);
  }
  for (int t = threadIdx.x; t < 2 * nz; t += blockDim.x) tw[t] = twiddle[t];
  if (bulk) {
    if (cnt < TPL)
      for (int t = threadIdx.x; t < nz * LD; t += blockDim.x)
        if (t % LD >= cnt) land[t] = 0.0;  // columns no copy writes
    const bool ok = __syncthreads_and(mbar_wait(bar, 0));
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(&g_fft_timeout, 1);
      mbar_wait(bar, 0);
      return;
    }
  } else {
    for (int t = threadIdx.x; t < nz * LD; t += blockDim.x) {
      const int n = t / LD, c = t - n * LD;
      land[t] = (c < cnt) ? data[static_cast<size_t>(n) * plane_size + p0 + c] : 0.0;
    }
    __syncthreads();
  }
  if (sign < 0) {
    // Z_k = X_k + i X'_k from the packed spectra of lines q and q + TPC
    // (B: plane 0 = Re X_0, 1 = Re X_{N/2}, 2k / 2k+1 = Re / Im X_k)
    for (int t = threadIdx.x; t < N * TPC; t += blockDim.x) {
      const int k = t / TPC, q = t - k * TPC;
      double xr[2], xi[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = q + h * TPC;
        if (k == 0) {
          xr[h] = B[c];
          xi[h] = 0.0;
        } else if (k == half) {
          xr[h] = B[LD + c];
          xi[h] = 0.0;
        } else if (k < half) {
          xr[h] = B[(2 * k) * LD + c];
          xi[h] = B[(2 * k + 1) * LD + c];
        } else {
          xr[h] = B[(2 * (N - k)) * LD + c];
          xi[h] = -B[(2 * (N - k) + 1) * LD + c];
        }
      }
      A[k * LD + q] = xr[0] - xi[1];
      A[k * LD + q + TPC] = xi[0] + xr[1];
    }
  }
  __syncthreads();
  const double s = sign > 0 ? -1.0 : 1.0;
  double *xb = A, *yb = B;
  int Ns = 1;
  for (int f = 0; f < plan.nf; ++f) {
    const int R = plan.dradix(f);
    if (R == 4) stockham_stage<4, TPC, LD>(xb, xb + TPC, yb, yb + TPC, N, Ns, tw, s);
    else if (R == 2) stockham_stage<2, TPC, LD>(xb, xb + TPC, yb, yb + TPC, N, Ns, tw, s);
    else if (R == 3) stockham_stage<3, TPC, LD>(xb, xb + TPC, yb, yb + TPC, N, Ns, tw, s);
    else stockham_stage<5, TPC, LD>(xb, xb + TPC, yb, yb + TPC, N, Ns, tw, s);
    Ns *= R;
    double* t0 = xb;
    xb = yb;
    yb = t0;
    __syncthreads();
  }
  if (sign < 0) {
    // z_n = x_n + i x'_n: the rows are the real lines again
    for (int t = threadIdx.x; t < nz * LD; t += blockDim.x) {
      const int n = t / LD, c = t - n * LD;
      if (c < cnt) data[static_cast<size_t>(n) * plane_size + p0 + c] = xb[t];
    }
    return;
  }
  // X_k = (Z_k + conj Z_{N-k}) / 2, X'_k = (Z_k - conj Z_{N-k}) / 2i, packed and scaled
  const double scale = 0.5 / nz;
  for (int t = threadIdx.x; t < nz * TPC; t += blockDim.x) {
    const int n = t / TPC, q = t - n * TPC;
    const int k = n == 0 ? 0 : (n == 1 ? half : n >> 1);
    const bool im = n >= 2 && (n & 1);
    const int kn = k == 0 ? 0 : N - k;
    const double zr = xb[k * LD + q], zi = xb[k * LD + q + TPC];
    const double wr = xb[kn * LD + q], wi = xb[kn * LD + q + TPC];
    const double v0 = im ? (zi - wi) : (zr + wr);   // line q
    const double v1 = im ? (wr - zr) : (zi + wi);   // line q + TPC
    const size_t row = static_cast<size_t>(n) * plane_size + p0;
    if (q < cnt) data[row + q] = v0 * scale;
    if (q + TPC < cnt) data[row + q + TPC] = v1 * scale;
  }
}

__global__ void k_nz2(double* data, int plane_size, int sign) {
  pdl_trigger();
  pdl_wait();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= plane_size) return;
  data[plane_size + p] = sign > 0 ? 0.0 : data[p];
}

}  // namespace

cudaError_t z_transform(double* data, int nz, int plane_size, int sign, const double* twiddle,
                        double* /*work*/, cudaStream_t st, bool pdl) {
  if (nz < 2) return cudaSuccess;
  if (nz == 2) {
    launch_ex(pdl, k_nz2, dim3((plane_size + 255) / 256), dim3(256), 0, st, data, plane_size, sign);
    return cudaGetLastError();
  }
  // Stockham FFT when nz factors into 2, 3, 5 (radix 4 first)
  FftPlan plan{};
  {
    int n = nz;
    auto add = [&](unsigned long long r) { plan.radices |= r << (4 * plan.nf++); };
    while (n % 4 == 0 && plan.nf < 16) { add(4); n /= 4; }
    while (n % 2 == 0 && plan.nf < 16) { add(2); n /= 2; }
    while (n % 3 == 0 && plan.nf < 16) { add(3); n /= 3; }
    while (n % 5 == 0 && plan.nf < 16) { add(5); n /= 5; }
    if (n != 1) plan.nf = 0;
  }
  raise_smem_limit(reinterpret_cast<const void*>(k_dft), 200 * 1024);
  raise_smem_limit(reinterpret_cast<const void*>(k_fft<32>), 200 * 1024);
  raise_smem_limit(reinterpret_cast<const void*>(k_fft<16>), 200 * 1024);
  raise_smem_limit(reinterpret_cast<const void*>(k_fft<8>), 200 * 1024);
  raise_smem_limit(reinterpret_cast<const void*>(k_fft<4>), 200 * 1024);
  if (plan.nf > 0) {
    int tp = 32;
    while (tp > 4 && sizeof(double) * (2 * static_cast<size_t>(nz) * tp + 2 * nz + 2) > 160 * 1024) tp /= 2;
    const size_t fshm = sizeof(double) * (2 * static_cast<size_t>(nz) * tp + 2 * nz + 2);
    // bulk row copies need 16-byte aligned rows: an aligned base and an even
    // plane size (tp is even)
    const int bulk = (reinterpret_cast<uintptr_t>(data) % 16 == 0 && plane_size % 2 == 0 && tp % 2 == 0) ? 1 : 0;
    if (fshm <= 200 * 1024) {
      const int nb = (plane_size + tp - 1) / tp;
      auto go = [&](auto kernel) {
        launch_ex(pdl, kernel, dim3(nb), dim3(256), fshm, st, data, nz, plane_size, sign, twiddle, plan, bulk);
      };
      if (tp == 32) go(k_fft<32>);
      else if (tp == 16) go(k_fft<16>);
      else if (tp == 8) go(k_fft<8>);
      else go(k_fft<4>);
      return cudaGetLastError();
    }
  }
  const size_t shm = sizeof(double) * (2 * static_cast<size_t>(nz) * kTP + 2 * nz);
  launch_ex(pdl, k_dft, dim3((plane_size + kTP - 1) / kTP), dim3(256), shm, st, data, nz, plane_size, sign, twiddle);
  return cudaGetLastError();
}

}  // namespace stx
