// Physical derivative at one node of an element held in shared memory
// (Element::grad, src/element.cpp:521-565, restated per node).
#pragma once

#include "device.hpp"

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
