// Two-level (patch + interface) solve of the skeleton system.
#pragma once

#include <cstddef>
#include <vector>

#include "device.hpp"

namespace stx {

// Doubles of scratch twolevel_solve needs after R: one skeleton vector per
// plane (patch-interior products, then the solution).
size_t twolevel_workspace_doubles(int rstride, int nz);

// Skeleton vectors R[k][0..nglobal) of every solved plane hold the condensed
// right-hand sides on entry (R is overwritten); the skeleton solution is left
// in twolevel_solution(work, ...).  `mid` (optional) is recorded after the
// interface products.  fp32: the matrices are read from S.l2_pack32.
// y_zeroed: the caller has already zeroed the solution planes of the launch's
// modes (twolevel_solution(work, ...)).
cudaError_t twolevel_solve(const DevModal& S, const DevGeom& g, const DevNumbering& N, double* R, int rstride,
                           double* work, int nz, cudaStream_t st, cudaEvent_t mid = nullptr, bool fp32 = false,
                           bool y_zeroed = false);

inline double* twolevel_solution(double* work, int /*rstride*/, int /*nz*/) { return work; }

// The same solve for nf (1..3) fields that share the matrices (FP64 only):
// field f's right-hand sides at R + f fstride, its solution written to
// Y + f fstride; every tile is read once for all fields.
cudaError_t twolevel_solve_fields(const DevModal& S, const DevGeom& g, const DevNumbering& N, double* R,
                                  double* Y, size_t fstride, int nf, int rstride, int nz, cudaStream_t st,
                                  bool y_zeroed = false);

int twolevel_launches(const DevModal& S);

// Up to kZeroRanges ranges set to zero in one kernel, launched
// programmatically dependent when `pdl` is set (it waits for the previous
// kernel before writing).
constexpr int kZeroRanges = 9;
struct ZeroRanges {
  double* p[kZeroRanges];
  size_t n[kZeroRanges];
  int count = 0;
  void add(double* ptr, size_t len) {
    if (ptr && len && count < kZeroRanges) {
      p[count] = ptr;
      n[count++] = len;
    }
  }
};
cudaError_t zero_ranges(bool pdl, const ZeroRanges& z, cudaStream_t st);
// a[0..na) = 0 and b[0..nb) = 0 (b may be null)
cudaError_t zero_ranges(bool pdl, double* a, size_t na, double* b, size_t nb, cudaStream_t st);

// Split the tiles of `probs` (in order) into equal runs, one per warp of a
// grid of `wpb`-warp blocks that fills `device` occ_pct / 100 times at the
// product kernel's occupancy (100: one full wave).
std::vector<SymWarp> sym_schedule(const std::vector<SymProblem>& probs, int device, int wpb = 4,
                                  int occ_pct = 100, int regcap = 0);

}  // namespace stx
