// Element-level static condensation and interior recovery for all planes of
// a field (the per-element halves of Field::solve DIRECT,
// src/field.cpp:598-709): the forcing of each element is condensed onto its
// boundary nodes and summed into the skeleton right-hand side
// (Element::local2globalSumSC, src/element.cpp:326-365); after the skeleton
// solve the interior values are recovered (Element::global2localSC,
// src/element.cpp:368-407).
#pragma once

#include <cstddef>

#include "device.hpp"

namespace stx {

// Leading dimension used for the element operands: >= n, a multiple of 4 with
// an odd quotient, so that the 8 rows of an m8n8k4 fragment fall on distinct
// shared-memory bank groups.
__host__ __device__ inline int element_ld(int n) {
  int ld = (n + 3) / 4 * 4;
  if ((ld / 4) % 2 == 0) ld += 4;
  return ld;
}

struct ElementPlan {
  bool ok = false;
  int cond_rows = 0, cond_rb = 0, cond_threads = 0;
  int rec_rows = 0, rec_rb = 0, rec_threads = 0;
  size_t cond_smem = 0, rec_smem = 0;
};

// Block shapes and shared memory of the two kernels; ok = false when the
// element operands do not fit (the caller then uses the simple kernels).
ElementPlan element_plan(const DevGeom& g, const DevModal& S, bool lift);

// R[k][btog] += F_b - h_bi h_ii^-1 F_i for every element and solved plane,
// F = -(Q4 f + H g).  G (essential values, may be null) as in
// helmholtz_direct_solve.
void element_condense(const ElementPlan& P, const DevGeom& g, const DevNumbering& N, const DevModal& S,
                      const double* F, const double* G, int gstride, double* R, int rstride, cudaStream_t st);

// U = (boundary: solved skeleton values / essential values; interior:
// h_ii^-1 F_i - (h_ii^-1 h_ib) u_b) for every element and solved plane.
void element_recover(const ElementPlan& P, const DevGeom& g, const DevNumbering& N, const DevModal& S,
                     const double* F, const double* G, int gstride, const double* R, int rstride, double* U,
                     cudaStream_t st);

// Skeleton couplings through the element Schur complements S_e (two-level
// solve), for every element and solved plane, with I / B the element nodes
// that are patch-interior / patch-interface skeleton unknowns:
//   dir 0:  dst[B] -= S_BI src[I]        dir 1:  dst[I] -= S_IB src[B]
void element_schur_apply(int dir, const DevGeom& g, const DevNumbering& N, const DevModal& S, const double* src,
                         double* dst, int rstride, cudaStream_t st);

}  // namespace stx
