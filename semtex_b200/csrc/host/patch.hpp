// Second level of static condensation (substructuring) of the boundary system.
//
// The reference solves the statically condensed element-boundary ("skeleton")
// system of every Fourier mode with one banded Cholesky factor
// (src/matrix.cpp:214-265, src/field.cpp:693).  Here elements are grouped into
// patches by recursive coordinate bisection; skeleton unknowns used only by the
// elements of one patch are condensed out patch by patch with dense matrices,
// and only the remaining patch-interface unknowns form a banded system.  The
// solution is the same linear-algebra solution; the banded factor and the
// sequential depth of its triangular solves shrink to the interface's.
//
// Patches whose elements belong to the same geometry families in the same
// arrangement and with the same node classification share their matrices
// (the Family::adopt idea of femlib/family.c applied one level up).
#pragma once

#include <vector>

#include "mesh.hpp"

namespace stx {

struct Patching {
  int npatch = 0, nfamily = 0;
  int nI_max = 0, nB_max = 0;
  std::vector<int> family;              // [npatch] patch family
  std::vector<int> family_rep;          // [nfamily] representative patch
  std::vector<int> nI, nB;              // [npatch] interior / interface node counts
  std::vector<int> I_gid;               // [npatch * nI_max] skeleton ids of interior nodes, -1 pad
  std::vector<int> B_iid;               // [npatch * nB_max] interface ids of boundary nodes, -1 pad
  std::vector<std::vector<int>> elems;  // [npatch] elements, canonical order
  std::vector<std::vector<int>> local;  // [npatch][pos*next + b] local node index, -1 = not an unknown
  int niface = 0;                       // interface unknowns
  int nband = 0;                        // band width of the interface system
  std::vector<int> iface_of;            // [nglobal] interface id or -1
  std::vector<int> skel_of;             // [niface] skeleton id of each interface unknown
  int pin_iid = -1;                     // interface id of the node a singular mode pins
};

// Build the patching of a numbering.  When the skeleton system has no
// essential nodes its k=0 problem may be singular: the skeleton node the
// reference pins (the highest-numbered solve node, src/matrix.cpp:160-162)
// is then kept on the interface (pin_iid), where a singular mode fixes it
// to zero with an identity row and column.
Patching build_patching(const Mesh& M, const Numbering& N, int max_patch_elems = 16, int rcm_roots = 32);

}  // namespace stx
