// Body forcing of the DNS nonlinear terms (<FORCE> section; FieldForce,
// dns/fieldforce.cpp:75-137 and the VirtualForce classes :240-822).
#pragma once

#include <cuda_runtime.h>

#include "exprprog.hpp"

namespace stx {

// Physical-space forcing of velocity component `com`, added to its
// nonlinear terms N on one z grid (nzl planes of plane_size doubles, nplane
// nodes each).  Every term present is summed into the force in the
// reference's class order -- sponge, Coriolis, steady, modulated,
// spatio-temporal, drag, selective frequency damping -- and the force added
// to N at the end (FieldForce::addPhysical).  Null pointers switch a term off.
struct ForceArgs {
  double* N;
  const double* U[3];  // physical velocity components (ncom of them)
  int ncom, com;
  int nzl, plane_size, nplane;
  double dz;           // z of plane k is k * dz
  double t;            // time the spatio-temporal programs see
  const double* x;     // [nplane] node coordinates
  const double* y;
  // SpongeForce (:516-578): force = (uref - u) mask
  const double* mask;
  const double* uref;
  // CoriolisForce (:631-756): 0 off, 1 steady, 2 unsteady
  int coriolis;
  double m2o[3];   // -2 Omega
  double dodt[3];  // -dOmega/dt (unsteady)
  double o[3];     // Omega (unsteady)
  double mo[3];    // -Omega (unsteady)
  // SteadyForce (:273-344), ModulatedForce (:387-460), SpatioTemporalForce
  // (:463-514)
  const double* steady;
  const double* moda;
  double alpha;
  const ExprOp* st;
  int nst;
  // DragForce (:581-628): force -= mask |u| u_com
  const double* drag;
  // SFDForce (:759-822): force += chi (qbar - u); qbar relaxes towards u
  double* qbar;
  double chi, rate;  // rate = D_T / SFD_DELTA
  int sfd_init;      // first call: qbar = u
};

cudaError_t dns_force_physical(const ForceArgs& a, cudaStream_t st);

// ConstForce::fourier (:262-270): v added to the nplane values of plane 0.
cudaError_t dns_force_const(double* N, int nplane, double v, cudaStream_t st);

// out = program(x, y, k dz, t) at the nplane nodes of nzl planes.
cudaError_t eval_program_field(const ExprOp* ops, int nops, double* out, int nzl, int plane_size, int nplane,
                               const double* x, const double* y, double dz, double t, cudaStream_t st);

}  // namespace stx
