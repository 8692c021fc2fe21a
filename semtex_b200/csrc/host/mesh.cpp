#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <queue>
#include <atomic>
#include <limits>
#include <stdexcept>
#include <thread>

namespace stx {

namespace {
constexpr double kEpsDP = 6.0e-14;  // veclib/cveclib.h:58

void legendre(int n, double x, double& pn, double& pn1) {
  double p0 = 1.0, p1 = x;
  if (n == 0) {
    pn = 1.0;
    pn1 = 0.0;
    return;
  }
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  pn = p1;
  pn1 = p0;
}
}  // namespace

Quadrature gll(int np) {
  if (np < 2) throw std::runtime_error("need > 2 knots for element edges");
  Quadrature Q;
  Q.np = np;
  const int N = np - 1;
  Q.z.resize(np);
  Q.w.resize(np);
  Q.D.assign(np * np, 0.0);
  // Lobatto nodes: Newton iteration on (x P_N - P_{N-1}) from the
  // Chebyshev--Gauss--Lobatto points (roots of (1-x^2) P_N'(x)).
  for (int j = 0; j < np; ++j) {
    double x = -std::cos(M_PI * j / N);
    for (int it = 0; it < 100; ++it) {
      double pn, pn1;
      legendre(N, x, pn, pn1);
      double dx = (x * pn - pn1) / (np * pn);
      x -= dx;
      if (std::fabs(dx) < 1e-17) break;
    }
    Q.z[j] = x;
  }
  Q.z[0] = -1.0;
  Q.z[N] = 1.0;
  std::vector<double> PN(np);
  for (int j = 0; j < np; ++j) {
    double pn, pn1;
    legendre(N, Q.z[j], pn, pn1);
    PN[j] = pn;
    Q.w[j] = 2.0 / (N * (N + 1) * pn * pn);
  }
  for (int i = 0; i < np; ++i)
    for (int j = 0; j < np; ++j)
      if (i != j) Q.D[i * np + j] = PN[i] / (PN[j] * (Q.z[i] - Q.z[j]));
  Q.D[0] = -N * (N + 1) / 4.0;
  Q.D[N * np + N] = N * (N + 1) / 4.0;
  return Q;
}

namespace {
constexpr double kEpsDp = 6.0e-14;  // EPSDP, veclib/cveclib.h:58
}

std::vector<double> svv_derivative(const Quadrature& q, double eps, int mN, double nu) {
  const int np = q.np, N = np - 1;
  if (!(mN >= 0 && mN < N && eps > kEpsDp)) return {};
  std::vector<double> S(np, 0.0), L(static_cast<size_t>(np) * np);
  for (int k = mN + 1; k < np; ++k) {
    const double r = (N - k) / (1.0 * mN - k);
    S[k] = std::exp(-r * r);
  }
  for (int k = 0; k < np; ++k) S[k] = 1.0 + eps / nu * S[k];
  // L[k][j] = P_k(z_j); forward transform MF[k][j] = C_k w_j L[k][j] with
  // C_k = 1/gamma_k of the discrete GLL norms; inverse MI[j][k] = L[k][j]
  for (int j = 0; j < np; ++j) {
    double p0 = 1.0, p1 = q.z[j];
    L[j] = 1.0;
    if (np > 1) L[np + j] = p1;
    for (int k = 2; k < np; ++k) {
      const double p2 = ((2 * k - 1) * q.z[j] * p1 - (k - 1) * p0) / k;
      L[static_cast<size_t>(k) * np + j] = p2;
      p0 = p1;
      p1 = p2;
    }
  }
  std::vector<double> dv(static_cast<size_t>(np) * np), dt(static_cast<size_t>(np) * np),
      out(static_cast<size_t>(np) * np, 0.0);
  for (int k = 0; k < np; ++k) {
    const double ck = k < N ? 0.5 * (k + k + 1) : 0.5 * N;
    const double sk = std::sqrt(S[k]);
    for (int j = 0; j < np; ++j) dv[k * np + j] = sk * (ck * q.w[j] * L[k * np + j]);
  }
  for (int i = 0; i < np; ++i)  // dt = MI dv
    for (int j = 0; j < np; ++j) {
      double v = 0.0;
      for (int k = 0; k < np; ++k) v += L[k * np + i] * dv[k * np + j];
      dt[i * np + j] = v;
    }
  for (int i = 0; i < np; ++i)  // out = dt D
    for (int j = 0; j < np; ++j) {
      double v = 0.0;
      for (int k = 0; k < np; ++k) v += dt[i * np + k] * q.D[k * np + j];
      out[i * np + j] = v;
    }
  return out;
}

std::vector<double> svv_z(int nz, int num_modes, double eps, int mN, double nu) {
  std::vector<double> S(num_modes, 0.0);
  const int N = (nz + 1) / 2 - 1;
  if (mN >= 0 && mN < N && eps > kEpsDp) {
    for (int i = 0; i < num_modes; ++i)
      if (i > mN) {
        const double r = (N - i) / (1.0 * mN - i);
        S[i] = std::exp(-r * r);
      }
    for (auto& v : S) v = 1.0 + eps / nu * v;
  } else {
    for (auto& v : S) v = 1.0;
  }
  return S;
}

void Mesh::side_nodes(int s, int* idx) const {
  const int n = np;
  for (int t = 0; t < n; ++t) {
    switch (s) {
      case 0: idx[t] = t; break;
      case 1: idx[t] = t * n + n - 1; break;
      case 2: idx[t] = (n - 1) * n + (n - 1 - t); break;
      default: idx[t] = (n - 1 - t) * n; break;
    }
  }
}

Mesh build_mesh(const Session& S) {
  if (S.has_curves) throw std::runtime_error("curved element sides are not supported");
  Mesh M;
  M.np = S.tokens.ivalue("N_P");
  M.nz = S.tokens.ivalue("N_Z");
  if (M.nz > 1 && (M.nz & 1)) throw std::runtime_error("N_Z must be even");
  M.nel = static_cast<int>(S.elements.size());
  if (M.nel < 1) throw std::runtime_error("at least 1 element needed");
  const int n = M.np, nel = M.nel;
  M.npnp = n * n;
  M.next = 4 * (n - 1);
  M.nint = (n - 2) * (n - 2);
  M.nplane = nel * M.npnp;
  M.plane_size = M.nplane + (M.nplane % 2);  // src/geometry.cpp:105-108
  M.q = gll(n);
  if (S.tokens.value("SVV_EPSN") > kEpsDp) {
    if (S.tokens.value("SVV_MN") > n)  // dns/drive.cpp:244-245
      throw std::runtime_error("SVV_MN exceeds N_P");
    M.svv_D = svv_derivative(M.q, S.tokens.value("SVV_EPSN"), static_cast<int>(S.tokens.value("SVV_MN")),
                             S.tokens.value("KINVIS"));
  }
  const auto& z = M.q.z;
  const auto& w = M.q.w;
  const auto& D = M.q.D;

  // -- boundary-major traverse (femlib/mapping.c:97-115)
  M.emap.resize(M.npnp);
  M.pmap.resize(M.npnp);
  {
    int k = 0, v = 0;
    M.emap[0] = 0;
    for (int i = 1; i < n; ++i) M.emap[++k] = v += 1;
    for (int i = 1; i < n; ++i) M.emap[++k] = v += n;
    for (int i = 1; i < n; ++i) M.emap[++k] = v -= 1;
    for (int i = 1; i < n - 1; ++i) M.emap[++k] = v -= n;
    ++k;
    for (int i = 1; i < n - 1; ++i)
      for (int j = 1; j < n - 1; ++j) M.emap[k++] = i * n + j;
    for (int i = 0; i < M.npnp; ++i) M.pmap[M.emap[i]] = i;
  }

  // -- node locations: bilinear (Coons patch of straight sides)
  const double xs = S.tokens.value("X_SHIFT"), ys = S.tokens.value("Y_SHIFT");
  const double xc = S.tokens.value("X_SCALE"), yc = S.tokens.value("Y_SCALE");
  M.x.resize(M.nplane);
  M.y.resize(M.nplane);
  for (int e = 0; e < nel; ++e) {
    const auto& v = S.elements[e];
    double P[4][2];
    for (int c = 0; c < 4; ++c) {
      P[c][0] = S.nodes[v[c]][0];
      P[c][1] = S.nodes[v[c]][1];
    }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double r = z[j], s = z[i];
        const double a = (1 - r) * (1 - s), b = (1 + r) * (1 - s), c = (1 + r) * (1 + s),
                     d = (1 - r) * (1 + s);
        double X = 0.25 * (a * P[0][0] + b * P[1][0] + c * P[2][0] + d * P[3][0]);
        double Y = 0.25 * (a * P[0][1] + b * P[1][1] + c * P[2][1] + d * P[3][1]);
        if (std::fabs(xs) > kEpsDP) X += xs;
        if (std::fabs(ys) > kEpsDP) Y += ys;
        if (std::fabs(xc - 1.0) > kEpsDP) X *= xc;
        if (std::fabs(yc - 1.0) > kEpsDP) Y *= yc;
        M.x[e * M.npnp + i * n + j] = X;
        M.y[e * M.npnp + i * n + j] = Y;
      }
  }

  // -- geometric factors (src/element.cpp:1307-1407)
  M.cyl = S.tokens.ivalue("CYLINDRICAL") != 0;
  for (auto* v : {&M.Q1, &M.Q2, &M.Q3, &M.Q4, &M.Q8, &M.drdx, &M.drdy, &M.dsdx, &M.dsdy})
    v->assign(M.nplane, 0.0);
  for (int e = 0; e < nel; ++e) {
    const double* X = &M.x[e * M.npnp];
    const double* Y = &M.y[e * M.npnp];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double xr = 0, xs_ = 0, yr = 0, ys_ = 0;
        for (int k = 0; k < n; ++k) {
          xr += X[i * n + k] * D[j * n + k];
          yr += Y[i * n + k] * D[j * n + k];
          xs_ += D[i * n + k] * X[k * n + j];
          ys_ += D[i * n + k] * Y[k * n + j];
        }
        const double jac = xr * ys_ - xs_ * yr;
        if (jac < 4 * kEpsDP)
          throw std::runtime_error("Jacobian of element " + std::to_string(e + 1) + " nonpositive");
        const double WW = w[i] * w[j];
        const int ij = e * M.npnp + i * n + j;
        M.Q1[ij] = (xs_ * xs_ + ys_ * ys_) / jac * WW;
        M.Q2[ij] = (xr * xr + yr * yr) / jac * WW;
        M.Q3[ij] = (-yr * ys_ - xr * xs_) / jac * WW;
        M.Q4[ij] = jac * WW;
        M.drdx[ij] = ys_ / jac;
        M.drdy[ij] = -xs_ / jac;
        M.dsdx[ij] = -yr / jac;
        M.dsdy[ij] = xr / jac;
      }
    // the plain mass, then r premultiplied into the quadrature
    for (int k = 0; k < M.npnp; ++k) M.Q8[e * M.npnp + k] = M.Q4[e * M.npnp + k];
    if (M.cyl)
      for (int k = e * M.npnp; k < (e + 1) * M.npnp; ++k) {
        M.Q1[k] *= M.y[k];
        M.Q2[k] *= M.y[k];
        M.Q3[k] *= M.y[k];
        M.Q4[k] *= M.y[k];
      }
    // null-mapping: vectors below 4*EPSDP in 2-norm are exactly zero
    for (auto* v : {&M.drdx, &M.drdy, &M.dsdx, &M.dsdy, &M.Q3}) {
      double s = 0;
      for (int k = 0; k < M.npnp; ++k) s += (*v)[e * M.npnp + k] * (*v)[e * M.npnp + k];
      if (std::sqrt(s) < 4 * kEpsDP)
        std::fill(v->begin() + e * M.npnp, v->begin() + (e + 1) * M.npnp, 0.0);
    }
  }

  // -- side connectivity: shared vertex pairs, then <P> periodic mates
  M.mate.assign(nel * 4, {-1, -1});
  M.group.assign(nel * 4, 0);
  std::map<std::pair<int, int>, std::vector<int>> sides;
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s)
      sides[{S.elements[e][s], S.elements[e][(s + 1) % 4]}].push_back(e * 4 + s);
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      auto it = sides.find({S.elements[e][(s + 1) % 4], S.elements[e][s]});
      if (it != sides.end()) {
        int o = it->second.front();
        M.mate[e * 4 + s] = {o / 4, o % 4};
      }
    }
  for (const auto& sf : S.surfaces) {
    if (sf.elmt < 0 || sf.elmt >= nel || sf.side < 0 || sf.side > 3)
      throw std::runtime_error("surface element/side out of range");
    if (sf.kind == 'B') {
      M.group[sf.elmt * 4 + sf.side] = sf.group;
    } else {
      if (sf.mate_elmt < 0 || sf.mate_elmt >= nel || sf.mate_side < 0 || sf.mate_side > 3)
        throw std::runtime_error("periodic mate out of range");
      M.mate[sf.elmt * 4 + sf.side] = {sf.mate_elmt, sf.mate_side};
      M.mate[sf.mate_elmt * 4 + sf.mate_side] = {sf.elmt, sf.side};
    }
  }

  // -- geometry families: elements whose Q1..Q4 agree to EPSDP share
  //    condensed matrices (the role of Family::adopt, femlib/family.c:185).
  M.family.assign(nel, -1);
  for (int e = 0; e < nel; ++e) {
    for (int f = 0; f < M.nfamily && M.family[e] < 0; ++f) {
      const int r = M.family_rep[f];
      bool same = true;
      for (const auto* v : {&M.Q1, &M.Q2, &M.Q3, &M.Q4}) {
        for (int k = 0; k < M.npnp && same; ++k)
          same = std::fabs((*v)[e * M.npnp + k] - (*v)[r * M.npnp + k]) <= kEpsDP;
        if (!same) break;
      }
      if (same) M.family[e] = f;
    }
    if (M.family[e] < 0) {
      M.family[e] = M.nfamily++;
      M.family_rep.push_back(e);
    }
  }
  return M;
}

namespace {

// Reverse Cuthill--McKee from `root` over a symmetric adjacency (CSR).
void rcm_from(int root, const std::vector<int>& xadj, const std::vector<int>& adj,
              const std::vector<int>& deg, std::vector<int>& order, std::vector<char>& seen) {
  std::queue<int> Qu;
  Qu.push(root);
  seen[root] = 1;
  std::vector<int> nb;
  while (!Qu.empty()) {
    int v = Qu.front();
    Qu.pop();
    order.push_back(v);
    nb.clear();
    for (int k = xadj[v]; k < xadj[v + 1]; ++k)
      if (!seen[adj[k]]) {
        nb.push_back(adj[k]);
        seen[adj[k]] = 1;
      }
    std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
    for (int u : nb) Qu.push(u);
  }
}

int bfs_far(int root, const std::vector<int>& xadj, const std::vector<int>& adj,
            const std::vector<int>& deg, int& depth) {
  const int n = static_cast<int>(deg.size());
  std::vector<int> lev(n, -1);
  std::queue<int> Qu;
  Qu.push(root);
  lev[root] = 0;
  int last = root;
  while (!Qu.empty()) {
    int v = Qu.front();
    Qu.pop();
    if (lev[v] > lev[last] || (lev[v] == lev[last] && deg[v] < deg[last])) last = v;
    for (int k = xadj[v]; k < xadj[v + 1]; ++k)
      if (lev[adj[k]] < 0) {
        lev[adj[k]] = lev[v] + 1;
        Qu.push(adj[k]);
      }
  }
  depth = lev[last];
  return last;
}

}  // namespace

std::vector<int> rcm_order(std::vector<std::vector<int>>& nbr, int rcm_roots) {
  const int ns = static_cast<int>(nbr.size());
  std::vector<int> order;
  if (ns == 0) return order;
  std::vector<int> xadj(ns + 1, 0), adj, deg(ns);
  for (int a = 0; a < ns; ++a) {
    auto& v = nbr[a];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    deg[a] = static_cast<int>(v.size());
    xadj[a + 1] = xadj[a] + deg[a];
    adj.insert(adj.end(), v.begin(), v.end());
  }
  // candidate roots: a pseudo-peripheral node plus a spread of others
  std::vector<int> cand;
  {
    int depth = 0;
    int r = bfs_far(0, xadj, adj, deg, depth);
    for (int it = 0; it < 4; ++it) {
      int d2 = 0;
      int r2 = bfs_far(r, xadj, adj, deg, d2);
      if (d2 <= depth) break;
      depth = d2;
      r = r2;
    }
    cand.push_back(r);
    for (int k = 1; k < rcm_roots; ++k) cand.push_back(static_cast<int>((static_cast<long>(k) * ns) / rcm_roots));
  }
  auto bandwidth = [&](const std::vector<int>& ord) {
    std::vector<int> pos(ns);
    for (int k = 0; k < ns; ++k) pos[ord[k]] = k;
    int bw = 0;
    for (int a = 0; a < ns; ++a)
      for (int k = xadj[a]; k < xadj[a + 1]; ++k) bw = std::max(bw, std::abs(pos[a] - pos[adj[k]]));
    return bw;
  };
  int best_bw = -1;
  for (int root : cand) {
    std::vector<int> ord;
    std::vector<char> seen(ns, 0);
    rcm_from(root, xadj, adj, deg, ord, seen);
    for (int a = 0; a < ns; ++a)
      if (!seen[a]) rcm_from(a, xadj, adj, deg, ord, seen);
    int bw = bandwidth(ord);
    if (best_bw < 0 || bw < best_bw) {
      best_bw = bw;
      order.assign(ord.rbegin(), ord.rend());
    }
  }
  return order;
}

namespace {

// Mesh::chooseNode (src/mesh.cpp:479-531): the periodic representative of a
// vertex pair is the lower node id among the alternatives; per[v] = -1 when
// unset.  (fixPeriodic, :538-554, changes nothing.)
void choose_node(std::vector<int>& per, int n1, int n2) {
  const int p1 = per[n1], p2 = per[n2];
  int pn;
  if (p1 < 0) {
    if (p2 < 0) {
      pn = std::min(n1, n2);
      per[n1] = per[n2] = pn;
    } else if (p2 != n2) {
      pn = n1 < p2 ? n1 : p2;
      per[n1] = per[n2] = pn;
      per[p2] = pn;
    } else {
      pn = std::min(n1, n2);
      per[n1] = per[n2] = pn;
    }
  } else if (p1 != n1) {
    if (p2 < 0) {
      pn = p1 < n2 ? p1 : n2;
      per[n2] = per[n1] = pn;
      per[p1] = pn;
    } else if (p2 != n2) {
      pn = p1 < p2 ? p1 : p2;
      per[n1] = per[n2] = pn;
      per[p1] = pn;
      per[p2] = pn;
    } else {
      pn = p1 < n2 ? p1 : n2;
      per[n2] = per[n1] = pn;
      per[p1] = pn;
    }
  } else {
    if (p2 < 0) {
      pn = std::min(n1, n2);
      per[n1] = per[n2] = pn;
    } else if (p2 != n2) {
      pn = n1 < p2 ? n1 : n2;
      per[n2] = per[n1] = pn;
      per[p1] = pn;
    } else {
      pn = std::min(n1, n2);
      per[n1] = per[n2] = pn;
    }
  }
}

// One SPARSPAK RCM ordering (George & Liu; RCM and DEGREE as in
// femlib/netlib.f:1678-1890) of a connected graph from `root`, in Cuthill--
// McKee order (not yet reversed): breadth-first levels, each node's
// unnumbered neighbours in adjacency order, stably sorted by degree.  While
// numbering, the element spans (positions max - min over an element's
// nodes) are tracked; the walk stops early, returning -1, once a span
// exceeds `limit`.  Otherwise returns the largest span.
int cm_walk(int root, const std::vector<int>& xadj, const std::vector<int>& adj, const std::vector<int>& deg,
            const std::vector<int>& xel, const std::vector<int>& nel_of, int limit,
            std::vector<int>& perm, std::vector<int>& pos, std::vector<int>& first) {
  const int n = static_cast<int>(xadj.size()) - 1;
  perm.clear();
  std::fill(pos.begin(), pos.end(), -1);
  std::fill(first.begin(), first.end(), -1);
  int span = 0;
  auto place = [&](int v) {
    const int p = static_cast<int>(perm.size());
    pos[v] = p;
    perm.push_back(v);
    for (int k = xel[v]; k < xel[v + 1]; ++k) {
      const int e = nel_of[k];
      if (first[e] < 0) first[e] = p;
      span = std::max(span, p - first[e]);
    }
  };
  place(root);
  int lvlend = 0;
  while (true) {
    const int lbegin = lvlend;
    lvlend = static_cast<int>(perm.size());
    for (int i = lbegin; i < lvlend; ++i) {
      const int node = perm[i];
      const size_t fnbr = perm.size();
      for (int k = xadj[node]; k < xadj[node + 1]; ++k) {
        const int nb = adj[k];
        if (pos[nb] < 0) {
          pos[nb] = -2;  // taken; position assigned after the sort
          perm.push_back(nb);
        }
      }
      if (perm.size() - fnbr > 1)
        std::stable_sort(perm.begin() + fnbr, perm.end(), [&](int a, int b) { return deg[a] < deg[b]; });
      const std::vector<int> fresh(perm.begin() + fnbr, perm.end());
      perm.resize(fnbr);
      for (int v : fresh) place(v);
      if (span > limit) return -1;
    }
    if (static_cast<int>(perm.size()) <= lvlend) break;
  }
  if (static_cast<int>(perm.size()) != n) throw std::runtime_error("numbering graph is not connected");
  return span;
}

}  // namespace

std::vector<int> reference_map(const Session& S, const Mesh& M) {
  const int n = M.np, nel = M.nel, nm = n - 1, ni = n - 2, next = M.next;
  std::vector<int> per(S.nodes.size(), -1);
  for (const Surface& f : S.surfaces)
    if (f.kind == 'P') {
      choose_node(per, S.elements[f.elmt][f.side], S.elements[f.mate_elmt][(f.mate_side + 1) % 4]);
      choose_node(per, S.elements[f.elmt][(f.side + 1) % 4], S.elements[f.mate_elmt][f.mate_side]);
    }
  std::vector<int> vg(S.nodes.size(), -1);
  std::vector<std::vector<int>> sg(nel * 4);
  int nxt = 0;
  auto vertex = [&](int v) {
    const int p = per[v];
    if (p >= 0) {
      if (vg[p] < 0) vg[p] = nxt++;
      if (vg[v] < 0) vg[v] = vg[p];
    }
    if (vg[v] < 0) vg[v] = nxt++;
  };
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      vertex(S.elements[e][s]);
      if (ni) {
        const auto m = M.mate[e * 4 + s];
        std::vector<int>& g = sg[e * 4 + s];
        if (m[0] >= 0 && !sg[m[0] * 4 + m[1]].empty()) {
          const std::vector<int>& o = sg[m[0] * 4 + m[1]];
          g.assign(o.rbegin(), o.rend());
        } else {
          for (int t = 0; t < ni; ++t) g.push_back(nxt++);
        }
      }
      vertex(S.elements[e][(s + 1) % 4]);
    }
  std::vector<int> map(nel * next);
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      map[e * next + s * nm] = vg[S.elements[e][s]];
      for (int t = 0; t < ni; ++t) map[e * next + s * nm + 1 + t] = sg[e * 4 + s][t];
    }
  return map;
}

std::vector<int> enumerate_o3(const std::vector<int>& bmap, int nel, int next) {
  const int n = *std::max_element(bmap.begin(), bmap.end()) + 1;
  // -- Nsys::buildAdjncy / connectivSC (utility/enumerate.cpp:832-920):
  //    neighbours in order of first appearance, element by element
  std::vector<std::vector<int>> lists(n);
  for (int e = 0; e < nel; ++e) {
    const int* row = &bmap[e * next];
    for (int i = 0; i < next; ++i) {
      std::vector<int>& a = lists[row[i]];
      for (int j = 0; j < next; ++j)
        if (i != j && std::find(a.begin(), a.end(), row[j]) == a.end()) a.push_back(row[j]);
    }
  }
  std::vector<int> xadj(n + 1, 0), adj, deg(n);
  for (int v = 0; v < n; ++v) {
    deg[v] = static_cast<int>(lists[v].size());
    xadj[v + 1] = xadj[v] + deg[v];
    adj.insert(adj.end(), lists[v].begin(), lists[v].end());
  }
  // elements of each node (distinct), for the span bookkeeping
  std::vector<int> xel(n + 1, 0), nel_of;
  {
    std::vector<std::vector<int>> els(n);
    for (int e = 0; e < nel; ++e)
      for (int i = 0; i < next; ++i) {
        std::vector<int>& l = els[bmap[e * next + i]];
        if (l.empty() || l.back() != e) l.push_back(e);
      }
    for (int v = 0; v < n; ++v) {
      xel[v + 1] = xel[v] + static_cast<int>(els[v].size());
      nel_of.insert(nel_of.end(), els[v].begin(), els[v].end());
    }
  }
  // -- Nsys::renumber level 3 (utility/enumerate.cpp:694-831): every node
  //    as the root, the first of least global bandwidth (max element span
  //    + 1, globalBandwidth :923-964) wins.  Spans of reversed and forward
  //    orders are equal.  Roots are shared among threads; a walk stops once
  //    its span exceeds the best found so far (ties run to completion, so
  //    the lowest root among equals is kept).
  std::vector<int> span(n, -1);
  std::atomic<int> best{std::numeric_limits<int>::max()};
  std::atomic<int> next_root{0};
  const int nthr = std::max(1, std::min(16, static_cast<int>(std::thread::hardware_concurrency())));
  auto work = [&] {
    std::vector<int> perm, pos(n), first(nel);
    perm.reserve(n);
    for (int r; (r = next_root.fetch_add(1)) < n;) {
      const int sp = cm_walk(r, xadj, adj, deg, xel, nel_of, best.load(), perm, pos, first);
      span[r] = sp;
      if (sp >= 0) {
        int b = best.load();
        while (sp < b && !best.compare_exchange_weak(b, sp)) {
        }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthr; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  int root = -1;
  for (int r = 0; r < n; ++r)
    if (span[r] >= 0 && (root < 0 || span[r] < span[root])) root = r;
  std::vector<int> perm, pos(n), first(nel);
  cm_walk(root, xadj, adj, deg, xel, nel_of, std::numeric_limits<int>::max(), perm, pos, first);
  // reversed: CM position p -> number n - 1 - p (the root gets n - 1)
  std::vector<int> inv(n);
  for (int p = 0; p < n; ++p) inv[perm[p]] = n - 1 - p;
  std::vector<int> out(bmap.size());
  for (size_t k = 0; k < bmap.size(); ++k) out[k] = inv[bmap[k]];
  return out;
}

char axis_kind(char kind, char field, int mclass) {
  if (kind != 'A') return kind;
  if (field == 'u' || field == 'p' || field == 'c') return mclass == 0 ? 'N' : 'D';
  if (field == 'v') return 'D';
  if (field == 'w') return mclass == 1 ? 'N' : 'D';
  throw std::runtime_error(std::string("axis BC for unknown field ") + field);
}

Numbering build_numbering(const Session& S, const Mesh& M, char field, int rcm_roots, int mclass) {
  const int n = M.np, nel = M.nel, nm = n - 1, next = M.next;
  Numbering N;
  N.field = field;
  // -- vertex identification: union of periodic vertex pairs
  std::vector<int> parent(S.nodes.size());
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int a) {
    while (parent[a] != a) a = parent[a] = parent[parent[a]];
    return a;
  };
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      auto m = M.mate[e * 4 + s];
      if (m[0] < 0) continue;
      int a = S.elements[e][s], b = S.elements[e][(s + 1) % 4];
      int c = S.elements[m[0]][m[1]], d = S.elements[m[0]][(m[1] + 1) % 4];
      for (auto pr : {std::make_pair(a, d), std::make_pair(b, c)}) {
        int ru = find(pr.first), rv = find(pr.second);
        if (ru != rv) parent[std::max(ru, rv)] = std::min(ru, rv);
      }
    }
  std::vector<int> gid(nel * next, -1);
  std::map<int, int> vid;
  int nxt = 0;
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      int r = find(S.elements[e][s]);
      auto it = vid.find(r);
      if (it == vid.end()) it = vid.emplace(r, nxt++).first;
      gid[e * next + s * nm] = it->second;
    }
  std::vector<int> edge_first(nel * 4, -1);
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      const int es = e * 4 + s;
      int base;
      bool reversed = false;
      auto m = M.mate[es];
      if (edge_first[es] >= 0) {
        base = edge_first[es];
        reversed = true;
      } else {
        base = nxt;
        nxt += nm - 1;
        if (m[0] >= 0) edge_first[m[0] * 4 + m[1]] = base;
      }
      for (int t = 1; t < nm; ++t)
        gid[e * next + s * nm + t] = reversed ? base + (nm - 1 - t) : base + (t - 1);
    }
  const int nglobal = nxt;
  // -- essential nodes (Mesh::buildMask semantics, src/mesh.cpp:1226-1326),
  //    applied to every copy of a global node.
  std::vector<char> ess(nglobal, 0);
  for (int e = 0; e < nel; ++e)
    for (int s = 0; s < 4; ++s) {
      const int es = e * 4 + s;
      if (M.mate[es][0] >= 0) continue;
      char g = M.group[es];
      if (!g) continue;
      auto gi = S.bcs.find(g);
      if (gi == S.bcs.end()) throw std::runtime_error(std::string("no BCs for group ") + g);
      auto bi = gi->second.find(field);
      if (bi == gi->second.end())
        throw std::runtime_error(std::string("no BC for field ") + field + " in group " + g);
      BCSpec bc = bi->second;
      if (bc.kind == 'A') {  // axis: on y = 0, cylindrical only (BCmgr::buildsurf, src/bcmgr.cpp:872-890)
        if (!M.cyl) throw std::runtime_error("axis BCs disallowed in Cartesian coords");
        std::vector<int> idx(n);
        M.side_nodes(s, idx.data());
        for (int t = 0; t < n; ++t)
          if (std::fabs(M.y[e * M.npnp + idx[t]]) > kEpsDP)
            throw std::runtime_error("y value too large on axis BC");
        bc.kind = axis_kind('A', field, mclass);
        bc.expr = "0.0";
      }
      if (bc.kind == 'O') {  // computed outflow (src/bcmgr.cpp:416-431): p essential, u v natural, w c zero natural
        auto gd = S.groups.find(g);
        if (gd == S.groups.end() || gd->second.find("outflow") == std::string::npos)
          throw std::runtime_error("type 'O' BC must belong to group \"outflow\"");
        if (field != 'u' && field != 'v' && field != 'w' && field != 'p' && field != 'c')
          throw std::runtime_error(std::string("field name '") + field + "' for outflow BC not in 'uvwpc'");
        if (field == 'w' || field == 'c') {
          bc.kind = 'N';
          bc.expr = "0.0";
        }
      }
      if (bc.kind == 'D' || (bc.kind == 'O' && field == 'p')) {
        for (int t = 0; t <= nm; ++t) ess[gid[e * next + (s * nm + t) % next]] = 1;
      } else if (bc.kind == 'H') {
        if (field != 'p')
          throw std::runtime_error(std::string("high-order BC <H> given for field ") + field + ", not pressure");
      } else if (bc.kind != 'N' && bc.kind != 'M' && bc.kind != 'O') {
        throw std::runtime_error(std::string("boundary condition kind <") + bc.kind +
                                 "> is not supported");
      }
      BoundaryEdge E;
      E.elmt = e;
      E.side = s;
      E.kind = bc.kind;
      E.group = g;
      E.expr = bc.expr;
      if (bc.kind == 'M') {  // "K;C" or "K,C" (Mixed::Mixed, src/condition.cpp:295-312)
        const size_t cut = bc.expr.find_first_of(";,");
        if (cut == std::string::npos)
          throw std::runtime_error("mixed BC needs two values separated by ';' or ','");
        E.mix_K = S.tokens.eval(bc.expr.substr(0, cut), nullptr);
        E.mix_C = S.tokens.eval(bc.expr.substr(cut + 1), nullptr);
      }
      std::vector<int> idx(n);
      M.side_nodes(s, idx.data());
      E.x.resize(n);
      E.y.resize(n);
      for (int t = 0; t < n; ++t) {
        E.x[t] = M.x[e * M.npnp + idx[t]];
        E.y[t] = M.y[e * M.npnp + idx[t]];
      }
      // unit outward normal from the mapping partials at the side's nodes
      // (Element::sideGeom, src/element.cpp:1625-1747)
      E.nx.resize(n);
      E.ny.resize(n);
      for (int t = 0; t < n; ++t) {
        const int k = e * M.npnp + idx[t];
        double ax, ay;
        switch (s) {
          case 0: ax = -M.dsdx[k]; ay = -M.dsdy[k]; break;
          case 1: ax = M.drdx[k]; ay = M.drdy[k]; break;
          case 2: ax = M.dsdx[k]; ay = M.dsdy[k]; break;
          default: ax = -M.drdx[k]; ay = -M.drdy[k]; break;
        }
        const double len = std::hypot(ax, ay);
        E.nx[t] = ax / len;
        E.ny[t] = ay / len;
      }
      const double L = std::hypot(E.x[n - 1] - E.x[0], E.y[n - 1] - E.y[0]);
      E.area.resize(n);
      for (int t = 0; t < n; ++t) E.area[t] = 0.5 * L * M.q.w[t];
      N.edges.push_back(E);
    }
  // -- solve nodes first, RCM-ordered; essential nodes last
  std::vector<int> loc(nglobal, -1), solve_nodes;
  for (int g = 0; g < nglobal; ++g)
    if (!ess[g]) {
      loc[g] = static_cast<int>(solve_nodes.size());
      solve_nodes.push_back(g);
    }
  const int ns = static_cast<int>(solve_nodes.size());
  std::vector<int> order;
  if (ns > 1) {
    std::vector<std::vector<int>> nbr(ns);
    for (int e = 0; e < nel; ++e) {
      std::vector<int> v;
      for (int i = 0; i < next; ++i)
        if (loc[gid[e * next + i]] >= 0) v.push_back(loc[gid[e * next + i]]);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      for (int a : v)
        for (int b : v)
          if (a != b) nbr[a].push_back(b);
    }
    order = rcm_order(nbr, rcm_roots);
  } else if (ns == 1) {
    order.push_back(0);
  }
  std::vector<int> newid(nglobal);
  for (int k = 0; k < ns; ++k) newid[solve_nodes[order[k]]] = k;
  int ne = ns;
  for (int g = 0; g < nglobal; ++g)
    if (ess[g]) newid[g] = ne++;
  N.nglobal = nglobal;
  N.nsolve = ns;
  N.btog.resize(nel * next);
  N.bmask.resize(nel * next);
  N.emask.assign(nel, 0);
  for (int k = 0; k < nel * next; ++k) {
    N.btog[k] = newid[gid[k]];
    N.bmask[k] = ess[gid[k]];
    if (N.bmask[k]) N.emask[k / next] = 1;
  }
  if (ns == nglobal && ns > 1) {
    // No essential nodes: the k=0 system is singular and its pinned node, the
    // highest number, decides the solution (with high-order pressure BCs
    // the discrete Neumann data are not compatible, so more than a constant).
    // Such fields take the reference's own `enumerate -O3` numbering.
    N.btog = enumerate_o3(reference_map(S, M), nel, next);
  }
  for (const BoundaryEdge& E : N.edges)
    if (E.kind == 'M') {
      if (N.mixdiag.empty()) N.mixdiag.assign(nglobal, 0.0);
      for (int t = 0; t < n; ++t)
        N.mixdiag[N.btog[E.elmt * next + (E.side * nm + t) % next]] += E.mix_K * E.area[t];
    }
  int bw = 0;
  for (int e = 0; e < nel; ++e) {
    int lo = nglobal, hi = -1;
    for (int i = 0; i < next; ++i) {
      int g = N.btog[e * next + i];
      if (g < ns) {
        lo = std::min(lo, g);
        hi = std::max(hi, g);
      }
    }
    if (hi >= 0) bw = std::max(bw, hi - lo);
  }
  N.nband = bw + 1;
  // -- inverse boundary mass (src/bcmgr.cpp:813-825)
  N.imass.assign(nglobal, 0.0);
  for (int e = 0; e < nel; ++e)
    for (int i = 0; i < next; ++i)
    {
      // Element::bndryDsSum weights (src/element.cpp:433-463): in cylindrical
      // coordinates 1 where the r-weighted mass vanishes (on the axis)
      const double w = M.Q4[e * M.npnp + M.emap[i]];
      N.imass[N.btog[e * next + i]] += M.cyl && !(w > kEpsDP) ? 1.0 : w;
    }
  for (auto& v : N.imass) v = 1.0 / v;
  return N;
}

void gll_interpolants(const Quadrature& q, double x, double* h, double* dh) {
  const int n = q.np;
  const double* z = q.z.data();
  for (int j = 0; j < n; ++j) {
    // h_j(x) = prod_{m != j} (x - z_m) / (z_j - z_m); its derivative the
    // sum over l != j of the same product with factor l replaced by
    // 1 / (z_j - z_l)
    double v = 1.0, d = 0.0;
    for (int m = 0; m < n; ++m) {
      if (m == j) continue;
      const double f = (x - z[m]) / (z[j] - z[m]);
      d = d * f + v / (z[j] - z[m]);
      v *= f;
    }
    if (h) h[j] = v;
    if (dh) dh[j] = d;
  }
}

bool element_locate(const Mesh& M, int e, double x, double y, double tol, int maxit, bool guess, double& r,
                    double& s) {
  const int np = M.np, nn = M.npnp;
  const double kDiverge = 20.0;
  std::vector<double> ir(np), is(np), dr(np), ds(np), tp(np);
  const double* X = M.x.data() + static_cast<size_t>(e) * nn;
  const double* Y = M.y.data() + static_cast<size_t>(e) * nn;
  if (guess) {
    // initial guess: the element node nearest (x, y), if within the
    // element's longer diagonal
    const double diag = std::max(std::hypot(X[nn - 1] - X[0], Y[nn - 1] - Y[0]),
                                 std::hypot(X[np * (np - 1)] - X[np - 1], Y[np * (np - 1)] - Y[np - 1]));
    int best = 0;
    double dmin = 0.0;
    for (int t = 0; t < nn; ++t) {
      const double dx = x - X[t], dy = y - Y[t];
      const double d2 = dx * dx + dy * dy;
      if (t == 0 || d2 < dmin) {
        dmin = d2;
        best = t;
      }
    }
    if (dmin - diag * diag > 0.0) return false;
    r = M.q.z[best % np];
    s = M.q.z[best / np];
  }
  int it = 0;
  double F0, F1;
  do {
    gll_interpolants(M.q, r, ir.data(), dr.data());
    gll_interpolants(M.q, s, is.data(), ds.data());
    // x(r, s) = is^T X ir and its partials
    auto form = [&](const double* A, const double* w, const double* v) {
      for (int i = 0; i < np; ++i) {
        double a = 0.0;
        for (int j = 0; j < np; ++j) a += A[i * np + j] * w[j];
        tp[i] = a;
      }
      double a = 0.0;
      for (int i = 0; i < np; ++i) a += v[i] * tp[i];
      return a;
    };
    F0 = x - form(X, ir.data(), is.data());
    F1 = y - form(Y, ir.data(), is.data());
    const double J2 = form(X, ir.data(), ds.data()), J3 = form(Y, ir.data(), ds.data());
    const double J0 = form(X, dr.data(), is.data()), J1 = form(Y, dr.data(), is.data());
    double idet = J0 * J3 - J1 * J2;
    idet = std::fabs(idet) < kEpsDP ? 1.0 / kEpsDP : 1.0 / idet;
    r += (F0 * J3 - F1 * J2) * idet;
    s += (F1 * J0 - F0 * J1) * idet;
    if (std::fabs(r) > kDiverge && std::fabs(s) > kDiverge) return false;
  } while (++it < maxit && (std::fabs(F0) > tol || std::fabs(F1) > tol));
  return it < maxit && std::fabs(r) < 1.0 + tol && std::fabs(s) < 1.0 + tol;
}

int locate_point(const Mesh& M, double x, double y, double tol, int maxit, double& r, double& s) {
  for (int e = 0; e < M.nel; ++e) {
    r = s = 0.0;
    if (element_locate(M, e, x, y, tol, maxit, true, r, s)) return e;
  }
  return -1;
}

}  // namespace stx
