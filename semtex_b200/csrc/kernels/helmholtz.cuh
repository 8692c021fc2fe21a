// Launchers of the hot-path kernels (all asynchronous on the given stream).
#pragma once

#include <cstddef>

#include "device.hpp"

namespace stx {

// Rows per block of the pipelined banded sweeps (and of the inverse
// diagonal blocks the host precomputes for them).
constexpr int kBandRows = 16;

// Doubles of scratch the direct solve needs: boundary RHS and essential
// values, one padded globally numbered vector each per plane.
size_t helmholtz_workspace_doubles(const DevGeom& g, const DevNumbering& N, const DevModal& S);

// Field::solve DIRECT over all planes: F (Fourier forcing, reference plane
// layout) -> U.  `lines` holds the Fourier-space BC values [nz][nline].
// U's Nyquist plane (k = 1) is left untouched, as in the reference.
// `phase_events` (optional, 5 events) are recorded on `st` before the
// element condensation, before the skeleton solve (two-level: patch and
// interface products; otherwise the forward banded sweep), between its two
// halves, before the element recovery and at the end.
cudaError_t helmholtz_direct_solve(const DevGeom& g, const DevNumbering& N, const DevModal& S,
                                   const double* F, double* U, const double* lines, int nline,
                                   double* work, cudaStream_t st,
                                   cudaEvent_t* phase_events = nullptr, cudaEvent_t after_condense = nullptr);

// The direct solve of nf (1..3) fields whose systems share S (the same
// matrices: equal constants and numbering; each field its own forcing, BC
// lines and DevNumbering): per-field condensation and recovery, one skeleton
// solve reading every matrix tile once for all fields.  Needs the two-level
// path with the element kernels and FP64 matrices
// (helmholtz_fields_supported); scratch helmholtz_fields_workspace_doubles.
bool helmholtz_fields_supported(const DevGeom& g, const DevNumbering& N, const DevModal& S);
size_t helmholtz_fields_workspace_doubles(const DevGeom& g, const DevNumbering& N, int nf);
cudaError_t helmholtz_direct_solve_fields(const DevGeom& g, const DevNumbering* const* N, const DevModal& S,
                                          const double* const* F, double* const* U, const double* const* lines,
                                          const int* nline, int nf, double* work, cudaStream_t st,
                                          cudaEvent_t after_condense = nullptr);

// Number of kernel launches one direct solve issues.
int helmholtz_direct_launches(const DevNumbering& N, const DevModal& S, int np);

// Field::solve JACPCG over all planes (src/field.cpp:711-805).  U holds the
// initial guess on entry.  Iterations per plane are written to `iters`
// (host array, nz entries, -1 for planes not solved).  Returns
// cudaErrorNotReady if a plane reached STEP_MAX, after finishing all planes.
size_t jacpcg_workspace_doubles(const DevGeom& g, const DevNumbering& N);
cudaError_t helmholtz_jacpcg_solve(const DevGeom& g, const DevNumbering& N, const DevModal& S,
                                   const double* F, double* U, const double* lines, int nline,
                                   double tol_rel, int step_max, double* work, int* iters,
                                   cudaStream_t st);

// Nonzero once a bounded wait in the z-FFT expired on the current device
// (read after the work has been synchronised; -1 if it cannot be read).
int fft_timeout_flag();
// Device address of that flag on the current device (null if unavailable).
const int* fft_timeout_address();

// AuxField::transform (src/auxfield.cpp:1157-1194, femlib/fourier.c:40-165)
// of nz planes in place: sign +1 forward (scaled by 1/nz), -1 inverse.
// `twiddle` holds cos/sin(2 pi m / nz), m < nz, as [2][nz].  pdl: launched
// programmatically dependent on the stream's previous kernel.
cudaError_t z_transform(double* data, int nz, int plane_size, int sign, const double* twiddle,
                        double* work, cudaStream_t st, bool pdl = false);

}  // namespace stx
