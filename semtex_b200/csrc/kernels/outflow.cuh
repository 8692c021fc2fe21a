// Computed outflow boundary conditions <O> on the device (Dong, Karniadakis
// & Chryssostomidis 2014, as the reference implements them:
// BCmgr::maintainPhysical, src/bcmgr.cpp:998-1034; maintainFourier,
// :1203-1293; evaluateCEBCp, :1361-1465; evaluateCNBCu, :1516-1633).
//
// Per time step, on every outflow edge (element side, np nodes) of every
// plane:
//  - the physical edge velocities of the step are stored as a new level
//    (outflow_gather, from the nonlinear step's physical velocities);
//  - nu div u and nu n.grad(u).n of the Fourier velocity as new levels
//    (outflow_fourier; for the imaginary planes of the higher modes the
//    reference takes du/dx from the highest mode's imaginary plane, which its
//    loop leaves in place, and that is kept);
//  - KE* S0 = |u*|^2 / 2 (1 - tanh(u*.n / U0Delta)) / 2 of the extrapolated
//    edge velocities, Fourier-transformed along z (outflow_energy);
//  - the essential pressure: extrapolated nu n.grad(u).n - KE* S0
//    (outflow_plines), and after the pressure solve the natural u, v values
//    (KE* S0 / nu + p - extrapolated nu div u) n_x,y (outflow_ulines).
// Edge arrays are [plane][edge][node] with `ostride` doubles per plane.
#pragma once

#include <cuda_runtime.h>

#include "device.hpp"

namespace stx {

struct OutflowEdges {
  int no;             // outflow edges
  int ostride;        // doubles per plane of the edge arrays (>= no * np, even)
  const int* elmt;    // [no] element
  const int* side;    // [no] side
  const int* line;    // [no] edge number in the BC lines (the same for u, v, w, p)
  const double* nx;   // [no * np] unit outward normal
  const double* ny;
};

// lv[(c * nz + k) * ostride + e * np + r] = Up[c] at node r of edge e, plane k
// (c < ncom; component 2 zero when ncom < 3).
cudaError_t outflow_gather(const DevGeom& g, const OutflowEdges& E, const double* U, const double* V,
                           const double* W, double* lv, cudaStream_t st);

// New levels of nu div u and nu n.grad(u).n from the Fourier velocity.
cudaError_t outflow_fourier(const DevGeom& g, const OutflowEdges& E, const double* U, const double* V,
                            const double* W, double nu, double beta, double* divu, double* gradu, cudaStream_t st);

// fb (physical, nz planes) = KE* S0 of the edge velocities extrapolated over
// the levels lv[q] (coefficients ex[q], q < Jx); iuzd = 1 / U0Delta.
cudaError_t outflow_energy(const DevGeom& g, const OutflowEdges& E, const double* const* lv, const double* ex,
                           int Jx, double iuzd, double* fb, cudaStream_t st);

// Pressure lines of the outflow edges: sum_q ex[q] gradu[q] - fb.
cudaError_t outflow_plines(const DevGeom& g, const OutflowEdges& E, const double* const* gradu, const double* ex,
                           int Jx, const double* fb, double* lines, int nline, cudaStream_t st);

// Velocity lines (dir 0: u, 1: v) of the outflow edges from the new Fourier
// pressure p: (fb / nu + p - sum_q ex[q] divu[q]) n_dir.
cudaError_t outflow_ulines(const DevGeom& g, const OutflowEdges& E, const double* const* divu, const double* ex,
                           int Jx, const double* fb, const double* p, double nu, int dir, double* lines, int nline,
                           cudaStream_t st);

}  // namespace stx
