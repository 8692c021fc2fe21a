// Per-Fourier-mode condensed Helmholtz systems (host-side setup, FP64).
//
// The role of MatrixSys (src/matrix.cpp:132-316) and Element::HelmholtzSC
// (src/element.cpp:131-214): for each geometry family, the elemental
// Helmholtz matrix (HelmholtzRow semantics, src/element.cpp:1411-1481) is
// permuted to boundary-major order and statically condensed:
//   hii <- hii^{-1},  hbi <- hbi hii^{-1},  hbb <- hbb - hbi hii^{-1} hib.
// The condensed boundary matrices are assembled into the banded global
// matrix over the first nsolve global nodes and Cholesky-factored (A = U^T U,
// the factorisation dpbtrf computes at src/matrix.cpp:252).  The factor is
// kept in two row-contiguous lower-band layouts for the device solves:
//   fwd[j*nband + t]  = U[j-kd+t][j]          (rows of U^T)
//   bwd[r*nband + t]  = U[i][i+kd-t], i=n-1-r (rows of the reversed U)
// with the diagonal entry (t = kd) stored as its reciprocal.
// For JACPCG the inverse of the assembled diagonal is kept instead
// (src/matrix.cpp:270-304).
#pragma once

#include <vector>

#include "mesh.hpp"
#include "patch.hpp"

namespace stx {

enum SolverKind { kDirect = 0, kJacPCG = 1 };

struct ModeSystem {
  double lambda2 = 0, betak2 = 0;
  int method = kDirect;
  int nsolve = 0, nglobal = 0, nband = 0;
  bool singular = false;
  std::vector<double> hbi;   // [nfamily][next][nint]  hbi hii^{-1}
  std::vector<double> hii;   // [nfamily][nint][nint]  hii^{-1}
  std::vector<double> fwd, bwd;  // [nsolve][nband]
  std::vector<double> pc;    // JACPCG: [nglobal + nel*nint] inverse diagonal
  // With a patching (two-level condensation) the patch matrices and the dense
  // inverse of the patch-interface Schur complement replace the band factor:
  std::vector<double> l2_sinv;  // [pfamily][nI_max][nI_max]  S_II^{-1}
  std::vector<double> l2_g;     // [pfamily][nI_max][nB_max]  S_II^{-1} S_IB
  std::vector<double> l2_ainv;  // [niface][niface] inverse of the interface system
  std::vector<double> hsc;      // [nfamily][next][next] element Schur complements h_bb - h_bi h_ii^-1 h_ib
  int pin_iid = -1;             // interface node fixed to zero (singular mode)
};

// Full elemental Helmholtz matrix of element e, row-major node order.
void element_helmholtz(const Mesh& M, int e, double lambda2, double betak2, double* H);

// `P` (may be null) selects the two-level condensation for DIRECT systems.
// l2_device: stop after the element level (hbi, hii, hsc, pin_iid): the
// patch and interface matrices are then formed on the device (l2setup.cu).
// In-place inverse of a symmetric positive-definite n x n matrix (Cholesky,
// triangular inverse, product) on `nthreads` host threads; throws if the
// matrix is not positive definite.
void spd_inverse(int n, double* A, int nthreads = 1);
ModeSystem build_mode_system(const Mesh& M, const Numbering& N, const Patching* P, double lambda2,
                             double betak2, int method, int nthreads = 1, bool l2_device = false);

}  // namespace stx
