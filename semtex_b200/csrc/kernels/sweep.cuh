// Device-side setup of the two-level condensed systems (FP64): the dense
// linear algebra that the reference does per mode in MatrixSys
// (src/matrix.cpp:132-267: assembly of the condensed boundary system and its
// Cholesky factorisation, dpbtrf) runs here as batched kernels over modes.
//
// The tool is the block sweep (Gauss--Jordan elimination without pivoting,
// stable for symmetric positive-definite matrices).  Sweeping the pivot set
// I of a symmetric matrix [[S_II, S_IB], [S_BI, S_BB]] turns it into
//   [[-S_II^-1, S_II^-1 S_IB], [S_BI S_II^-1, S_BB - S_BI S_II^-1 S_IB]],
// so one partial sweep of a patch matrix gives the patch-interior inverse,
// G = S_II^-1 S_IB and the patch's interface Schur complement together, and
// a full sweep of the assembled interface system gives minus its inverse.
//
// Matrices are row-major with a leading dimension that is a multiple of 64,
// padded with identity rows and columns; only the lower triangle of 64 x 64
// tiles (tile row >= tile column) is read and written.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace stx {

constexpr int kSwBlk = 64;

inline int sweep_pad(int n) { return (n + kSwBlk - 1) / kSwBlk * kSwBlk; }

// Scratch doubles of sym_sweep for a batch of `batch` matrices of order n.
size_t sweep_scratch_doubles(int n, int batch);

// Sweep the pivots [0, npiv) (npiv and n multiples of 64) of `batch`
// symmetric n x n matrices A + b * stride.  *status (device int) is set to 1
// if a pivot is not positive (the matrix is not positive definite).
cudaError_t sym_sweep(double* A, int n, long long stride, int batch, int npiv, double* scratch, int* status,
                      cudaStream_t st);

// Patch matrices of one patch family for every mode, on the device:
// A[m] (order ld, zeroed by the caller) receives the assembled patch matrix
// sum_k local(hbb[m][family of element k]) over the patch's elements, with
// the interior nodes at rows [0, nI), the interface nodes at [pI, pI + nB)
// and identity on the padding; `mixI` (nI values or null) is added to the
// interior diagonal (mixed BCs).
struct PatchAssembly {
  const double* hbb;     // [nmodes][nfamily][next][next] element Schur complements
  int nfamily, next;
  const int* efam;       // [nelem] element family of each patch element
  const int* local;      // [nelem][next] local node index (-1: not an unknown)
  int nelem, nI, nB, pI, ld;
  const double* mixI;    // [nI] or null
};
cudaError_t patch_assemble(const PatchAssembly& p, double* A, long long stride, int nmodes, cudaStream_t st);

// Interface system of every mode: A[m] (order ld, zeroed by the caller)
// += T_m of each patch scattered by its interface ids; T_m is the swept
// patch matrix's [pI, pI + nB) block (lower triangle read).
cudaError_t interface_scatter(const double* T, long long tstride, int tld, int pI, int nB, const int* iid,
                              double* A, long long astride, int ald, int nmodes, cudaStream_t st);

// Finish the interface matrices: add `diag` (niface values, or null) to the
// diagonal, make row/column pin[m] (or none if < 0) an identity, and put
// identity on the padding rows [niface, ld).
cudaError_t interface_finish(double* A, long long stride, int ld, int niface, const double* diag, const int* pin,
                             int nmodes, cudaStream_t st);

// Pack sign * (symmetric n x n matrix at A + m*stride, lower triangle,
// leading dimension lda) into the symtile layout at out + off[m].
cudaError_t pack_sym(const double* A, long long stride, int lda, int n, double sign, double* out,
                     const long long* off, int nmodes, cudaStream_t st);

// Pack the nr x nc matrix G[a][b] = A[(r0 + b) * lda + a] (the transpose of
// a block below the diagonal) into the general tile layout at out + off[m].
cudaError_t pack_gen_t(const double* A, long long stride, int lda, int r0, int nr, int nc, double* out,
                       const long long* off, int nmodes, cudaStream_t st);

// out32[i] = (float) in[i], i < n.
cudaError_t to_float(const double* in, float* out, size_t n, cudaStream_t st);

}  // namespace stx
