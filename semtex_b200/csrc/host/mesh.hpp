// Spectral-element mesh, geometry and global numbering (host-side setup).
//
// Element node placement follows Mesh::meshElmt (src/mesh.cpp:767-882),
// straight sides with a Coons patch; geometric factors follow
// Element::mapping (src/element.cpp:1253-1408); GLL operators restate
// femlib/polylib.c:312-575; the boundary-major element traverse restates
// femlib/mapping.c:46-132.  Numbering plays the role of the `.num`
// NumberSys (src/numbersys.h, src/bcmgr.cpp:586-826): btog, bmask, emask,
// nglobal / nsolve / nband and the inverse boundary mass (imass).  The
// ordering is this library's own reverse Cuthill--McKee, except for fields
// without essential nodes, which take the reference's `enumerate -O3`
// numbering (their singular k=0 system pins the highest-numbered node).
#pragma once

#include <array>
#include <string>
#include <vector>

#include "session.hpp"

namespace stx {

struct Quadrature {
  int np = 0;
  std::vector<double> z, w, D;  // D[i*np+j] = h_j'(z_i), row-major
};
Quadrature gll(int np);

// Spectral vanishing viscosity (src/svv.cpp).  svv_derivative: the
// SVV-modified derivative matrix MI diag(sqrt S) MF D (SVV::operators,
// :126-185; MF, MI the GLL Legendre transform pair of femlib/operators.c:
// 317-490), S_k = 1 + eps/nu exp(-((N-k)/(mN-k))^2) for k > mN (SVV::coeffs,
// :20-52); empty when SVV is off (mN outside [0, N) or eps <= EPSDP).
// svv_z: the factors of beta^2 k^2 for the viscous systems' num_modes
// Fourier modes (SVV::coeffs_z, :55-90; N = nMode - 1).
std::vector<double> svv_derivative(const Quadrature& q, double eps, int mN, double nu);
std::vector<double> svv_z(int nz, int num_modes, double eps, int mN, double nu);

struct Mesh {
  int np = 0, nel = 0, nz = 1;
  int npnp = 0, next = 0, nint = 0;
  int nplane = 0, plane_size = 0;   // nel*np*np and its even round-up
  Quadrature q;
  std::vector<int> emap, pmap;      // boundary-major permutation and inverse
  std::vector<double> x, y;         // [nel*npnp] node locations
  std::vector<double> Q1, Q2, Q3, Q4, drdx, drdy, dsdx, dsdy;  // [nel*npnp]
  std::vector<std::array<int, 2>> mate;  // [nel*4] (elmt, side) or (-1,-1)
  std::vector<char> group;               // [nel*4] boundary group or 0
  std::vector<int> family;               // element -> geometry family
  std::vector<int> family_rep;           // family -> representative element
  int nfamily = 0;
  std::vector<double> svv_D;             // SVV derivative of the viscous operators, or empty
  // Cylindrical coordinates (token CYLINDRICAL; x axial, y radial, z
  // azimuthal): Q1-Q4 carry the radius r = y in their quadrature, Q8 the
  // plain mass that weights forcing (src/element.cpp:1389-1399, 800-806).
  bool cyl = false;
  std::vector<double> Q8;                // [nel*npnp]

  // Row-major node indices of side s in CCW traverse (src/element.h:162-170).
  void side_nodes(int s, int* idx) const;
};

Mesh build_mesh(const Session& S);

// Lagrange interpolants of the GLL points q.z at x and their derivatives
// (the intmat_g / dermat_g vectors of intp, femlib/operators.c:250-300);
// either output may be null.
void gll_interpolants(const Quadrature& q, double x, double* h, double* dh);

// Element::locate (src/element.cpp:1061-1183) in element e: Newton's
// iteration for (r, s) with x(r, s) = (x, y), from the element node nearest
// the point (guess; false when the point is farther than the element's
// longer diagonal) or from the given (r, s); true when it converges
// (|F| <= tol within maxit steps) to |r|, |s| < 1 + tol.
bool element_locate(const Mesh& M, int e, double x, double y, double tol, int maxit, bool guess, double& r,
                    double& s);

// HistoryPoint::locate (src/history.cpp:45-63) with Element::locate
// (src/element.cpp:1061-1183): the first element, in order, where Newton's
// iteration from the nearest element node converges (|F| <= tol within
// maxit steps) to |r|, |s| < 1 + tol.  Returns the element, -1 when none.
int locate_point(const Mesh& M, double x, double y, double tol, int maxit, double& r, double& s);

struct BoundaryEdge {
  int elmt = 0, side = 0;
  char kind = 0;              // 'D', 'N', 'M' (mixed) or 'H' (pressure only); others rejected
  char group = 0;             // boundary group
  std::string expr;
  double mix_K = 0.0, mix_C = 0.0;  // 'M': dc/dn + K (c - C) = 0
  std::vector<double> area;   // np quadrature-weighted side lengths
  std::vector<double> x, y;   // np node locations along the side
  std::vector<double> nx, ny; // np unit outward normal components
};

struct Numbering {
  char field = 0;
  int nglobal = 0, nsolve = 0, nband = 0;
  std::vector<int> btog, bmask;  // [nel*next]
  std::vector<int> emask;        // [nel]
  std::vector<double> imass;     // [nglobal]
  std::vector<BoundaryEdge> edges;
  // Mixed BCs: K * (quadrature-weighted side length) summed into the
  // diagonal of the assembled boundary system at each edge node
  // (Mixed::augmentSC, src/condition.cpp:345-376); empty without <M> edges.
  std::vector<double> mixdiag;   // [nglobal]
  bool same_as(const Numbering& o) const {
    return nglobal == o.nglobal && nsolve == o.nsolve && btog == o.btog && mixdiag == o.mixdiag;
  }
};

// Mesh::buildMap (src/mesh.cpp:884-1030): the reference's initial global
// numbers of element-boundary nodes, [nel*next] in boundary-major order,
// with periodic vertices identified as Mesh::chooseNode does.
std::vector<int> reference_map(const Session& S, const Mesh& M);

// `enumerate -O3` (utility/enumerate.cpp:694-964) of a numbering without
// essential nodes: each node in turn as the SPARSPAK RCM root, the first of
// least global bandwidth kept; returns the renumbered map (the chosen root
// gets the highest number).
std::vector<int> enumerate_o3(const std::vector<int>& bmap, int nel, int next);

// Reverse Cuthill--McKee order of a graph given as adjacency lists (sorted
// and deduplicated in place); the best of rcm_roots trial roots by bandwidth.
std::vector<int> rcm_order(std::vector<std::vector<int>>& nbr, int rcm_roots);

// rcm_roots: number of trial roots for the reverse Cuthill--McKee search
// (the role of enumerate's optimisation levels, utility/enumerate.cpp:706-832).
// mclass: the Fourier mode class (0, 1, 2 = modes 2 and up) whose axis BCs
// apply (cylindrical coordinates, axis_kind); 0 when there is no axis.
Numbering build_numbering(const Session& S, const Mesh& M, char field, int rcm_roots = 48, int mclass = 0);

// An axis BC <A> as the homogeneous essential ('D') or natural ('N')
// condition of field `field` in Fourier mode class `mclass` (0, 1, 2+),
// as src/bcmgr.cpp:153-180 tabulates: u, p, c natural in mode 0 and
// essential above; v~ essential; w~ essential except natural in mode 1.
// Other kinds are returned unchanged.
char axis_kind(char kind, char field, int mclass);

}  // namespace stx
