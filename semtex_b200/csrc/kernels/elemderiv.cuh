// Physical derivative at one node of an element held in shared memory
// (Element::grad, src/element.cpp:521-565, restated per node).
#pragma once

#include "device.hpp"
#include "ptx.cuh"

namespace stx {

// x (dir 0) or y (dir 1) derivative at node t of element e, whose np x np
// values su holds (row-major), D in sD.
__device__ __forceinline__ double elem_deriv(const DevGeom& g, const double* su, const double* sD, int e, int t,
                                             int dir) {
  const int np = g.np;
  const int i = t / np, j = t - (t / np) * np;
  double ur = 0.0, us = 0.0;
  for (int k = 0; k < np; ++k) {
    ur += su[i * np + k] * sD[j * np + k];  // (u D^T)[i][j] = du/dr
    us += sD[i * np + k] * su[k * np + j];  // (D u)[i][j]   = du/ds
  }
  const int q = e * g.npnp + t;
  return dir == 0 ? ur * g.drdx[q] + us * g.dsdx[q] : ur * g.drdy[q] + us * g.dsdy[q];
}

// Node of knot r of side `side` in the counter-clockwise traverse (row i =
// s, column j = r), as the BC lines order them.
__device__ __forceinline__ int side_node(int side, int r, int np) {
  int i, j;
  switch (side) {
    case 0: i = 0; j = r; break;
    case 1: i = r; j = np - 1; break;
    case 2: i = np - 1; j = np - 1 - r; break;
    default: i = np - 1 - r; j = 0; break;
  }
  return i * np + j;
}

}  // namespace stx

namespace stx {

// Element derivatives on the FP64 tensor cores (mma m8n8k4): the sum
// factorisation of Element::grad for one element plane U (np x np,
// row-major in shared memory), ur = U D^T and us = D U, as 8 x 8 result
// tiles (np padded to 8 MT), the k sums in KS steps of 4.  Lane l = 4 g + t
// holds the D fragment entries D[8 x + g][4 s + t] -- the same registers
// are the B operand of U D^T and the A operand of D U -- and receives
// C[g][2 t], C[g][2 t + 1] of every result tile: node (8 mi + g,
// 8 ni + 2 t + c).  The physical derivatives at a node are
// ur dr/dx + us ds/dx (x) and ur dr/dy + us ds/dy (y), as elem_deriv forms
// them.
template <int MT, int KS>
struct ElemMma {
  double df[MT][KS];
  __device__ __forceinline__ void load_d(const double* sD, int np) {
    const int ln = threadIdx.x & 31, g8 = ln >> 2, t4 = ln & 3;
#pragma unroll
    for (int x = 0; x < MT; ++x)
#pragma unroll
      for (int s = 0; s < KS; ++s) {
        const int r = 8 * x + g8, c = 4 * s + t4;
        df[x][s] = (r < np && c < np) ? sD[r * np + c] : 0.0;
      }
  }
  __device__ __forceinline__ void grad(const double* su, int np, double (&ur)[MT][MT][2],
                                       double (&us)[MT][MT][2]) const {
    const int ln = threadIdx.x & 31, g8 = ln >> 2, t4 = ln & 3;
    double ua[MT][KS], ub[KS][MT];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
      for (int s = 0; s < KS; ++s) {
        const int i = 8 * m + g8, k = 4 * s + t4;
        ua[m][s] = (i < np && k < np) ? su[i * np + k] : 0.0;  // U[i][k]
        const int kk = 4 * s + t4, j = 8 * m + g8;
        ub[s][m] = (kk < np && j < np) ? su[kk * np + j] : 0.0;  // U[k][j]
      }
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
      for (int n = 0; n < MT; ++n) {
        ur[m][n][0] = ur[m][n][1] = us[m][n][0] = us[m][n][1] = 0.0;
#pragma unroll
        for (int s = 0; s < KS; ++s) {
          dmma_8x8x4(ur[m][n][0], ur[m][n][1], ua[m][s], df[n][s]);
          dmma_8x8x4(us[m][n][0], us[m][n][1], df[m][s], ub[s][n]);
        }
      }
  }
};

// Tile counts of ElemMma for np nodes per direction: the launchers' choice
// of template instance (np <= 16).
inline int mma_tiles(int np) { return (np + 7) / 8; }
inline int mma_ksteps(int np) { return (np + 3) / 4; }

}  // namespace stx
