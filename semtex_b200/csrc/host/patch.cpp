#include "patch.hpp"

#include <cstring>

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <stdexcept>

namespace stx {

namespace {

// Recursive coordinate bisection of element centroids into groups of at
// most `cap` elements, splitting the longer extent at the median.
void bisect(std::vector<int>& ids, size_t lo, size_t hi, const std::vector<double>& cx,
            const std::vector<double>& cy, int cap, std::vector<std::vector<int>>& out) {
  if (hi - lo <= static_cast<size_t>(cap)) {
    out.emplace_back(ids.begin() + lo, ids.begin() + hi);
    return;
  }
  double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
  for (size_t i = lo; i < hi; ++i) {
    x0 = std::min(x0, cx[ids[i]]);
    x1 = std::max(x1, cx[ids[i]]);
    y0 = std::min(y0, cy[ids[i]]);
    y1 = std::max(y1, cy[ids[i]]);
  }
  const bool byx = (x1 - x0) >= (y1 - y0);
  auto key = [&](int e) { return byx ? std::make_pair(cx[e], cy[e]) : std::make_pair(cy[e], cx[e]); };
  std::sort(ids.begin() + lo, ids.begin() + hi, [&](int a, int b) { return key(a) < key(b); });
  const size_t mid = lo + (hi - lo) / 2;
  bisect(ids, lo, mid, cx, cy, cap, out);
  bisect(ids, mid, hi, cx, cy, cap, out);
}

}  // namespace

Patching build_patching(const Mesh& M, const Numbering& N, int max_patch_elems, int rcm_roots) {
  Patching P;
  const int nel = M.nel, next = M.next, ng = N.nglobal, ns = N.nsolve;
  std::vector<double> cx(nel, 0.0), cy(nel, 0.0);
  double ext = 0.0;
  for (int e = 0; e < nel; ++e) {
    for (int k = 0; k < M.npnp; ++k) {
      cx[e] += M.x[e * M.npnp + k];
      cy[e] += M.y[e * M.npnp + k];
    }
    cx[e] /= M.npnp;
    cy[e] /= M.npnp;
    ext = std::max({ext, std::fabs(cx[e]), std::fabs(cy[e])});
  }
  std::vector<int> ids(nel);
  std::iota(ids.begin(), ids.begin() + nel, 0);
  bisect(ids, 0, nel, cx, cy, std::max(1, max_patch_elems), P.elems);
  P.npatch = static_cast<int>(P.elems.size());
  std::vector<int> epatch(nel);
  for (int p = 0; p < P.npatch; ++p)
    for (int e : P.elems[p]) epatch[e] = p;

  // -- classify skeleton solve nodes: interior to one patch, or interface
  const bool maybe_singular = ng == ns;  // no essential nodes: k=0 may be pinned
  const int pin = maybe_singular ? ns - 1 : -1;
  std::vector<int> owner(ng, -1);  // patch, or -2 when shared
  for (int e = 0; e < nel; ++e)
    for (int i = 0; i < next; ++i) {
      const int g = N.btog[e * next + i];
      if (owner[g] == -1) owner[g] = epatch[e];
      else if (owner[g] != epatch[e]) owner[g] = -2;
    }
  P.iface_of.assign(ng, -1);
  std::vector<int> iface_nodes;
  for (int g = 0; g < ns; ++g)
    if (owner[g] == -2 || g == pin) iface_nodes.push_back(g);
  // -- interface numbering: RCM over "shares a patch"
  {
    std::vector<int> loc(ng, -1);
    std::vector<int> cand;
    for (int g : iface_nodes) {
      loc[g] = static_cast<int>(cand.size());
      cand.push_back(g);
    }
    std::vector<std::vector<int>> nbr(cand.size());
    for (int p = 0; p < P.npatch; ++p) {
      std::vector<int> v;
      for (int e : P.elems[p])
        for (int i = 0; i < next; ++i) {
          const int l = loc[N.btog[e * next + i]];
          if (l >= 0) v.push_back(l);
        }
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      for (int a : v)
        for (int b : v)
          if (a != b) nbr[a].push_back(b);
    }
    std::vector<int> order = rcm_order(nbr, rcm_roots);
    for (size_t k = 0; k < order.size(); ++k) {
      P.iface_of[cand[order[k]]] = static_cast<int>(k);
      P.skel_of.push_back(cand[order[k]]);
    }
    P.niface = static_cast<int>(P.skel_of.size());
    P.pin_iid = pin >= 0 ? P.iface_of[pin] : -1;
  }

  // -- per patch: canonical element order, local node indices (I first)
  std::map<std::vector<long long>, int> fam_of;
  P.local.resize(P.npatch);
  std::vector<std::vector<int>> Ig(P.npatch), Bi(P.npatch);
  const double q = 1e-9 * std::max(ext, 1.0);
  for (int p = 0; p < P.npatch; ++p) {
    auto& E = P.elems[p];
    double x0 = 1e300, y0 = 1e300;
    for (int e : E) {
      x0 = std::min(x0, cx[e]);
      y0 = std::min(y0, cy[e]);
    }
    std::sort(E.begin(), E.end(), [&](int a, int b) {
      const long long ya = std::llround((cy[a] - y0) / q), yb = std::llround((cy[b] - y0) / q);
      if (ya != yb) return ya < yb;
      return std::llround((cx[a] - x0) / q) < std::llround((cx[b] - x0) / q);
    });
    std::map<int, int> li;  // skeleton id -> provisional local id within class
    std::vector<int> Ilist, Blist;
    for (int e : E)
      for (int i = 0; i < next; ++i) {
        const int g = N.btog[e * next + i];
        if (g >= ns || li.count(g)) continue;
        if (P.iface_of[g] >= 0) {
          li[g] = -1 - static_cast<int>(Blist.size());
          Blist.push_back(g);
        } else {
          li[g] = static_cast<int>(Ilist.size());
          Ilist.push_back(g);
        }
      }
    const int nI = static_cast<int>(Ilist.size());
    auto& Lc = P.local[p];
    Lc.assign(E.size() * next, -1);
    std::vector<long long> sig;
    sig.push_back(nI);
    sig.push_back(static_cast<long long>(Blist.size()));
    for (size_t k = 0; k < E.size(); ++k) {
      sig.push_back(M.family[E[k]]);
      sig.push_back(std::llround((cx[E[k]] - x0) / q));
      sig.push_back(std::llround((cy[E[k]] - y0) / q));
      for (int i = 0; i < next; ++i) {
        const int g = N.btog[E[k] * next + i];
        int l = -1;
        if (g < ns) {
          const int v = li[g];
          l = v >= 0 ? v : nI + (-1 - v);
        }
        Lc[k * next + i] = l;
        sig.push_back(l);
      }
    }
    // mixed-BC diagonal entries of the interior nodes (bit patterns): patches
    // sharing matrices must agree on them
    if (!N.mixdiag.empty())
      for (int g : Ilist) {
        long long bits;
        std::memcpy(&bits, &N.mixdiag[g], sizeof(bits));
        sig.push_back(bits);
      }
    auto it = fam_of.find(sig);
    if (it == fam_of.end()) {
      it = fam_of.emplace(sig, P.nfamily++).first;
      P.family_rep.push_back(p);
    }
    P.family.push_back(it->second);
    Ig[p] = Ilist;
    for (int g : Blist) Bi[p].push_back(P.iface_of[g]);
    P.nI.push_back(nI);
    P.nB.push_back(static_cast<int>(Blist.size()));
    P.nI_max = std::max(P.nI_max, nI);
    P.nB_max = std::max(P.nB_max, static_cast<int>(Blist.size()));
  }
  P.nI_max = std::max(1, P.nI_max);
  P.nB_max = std::max(1, P.nB_max);
  P.I_gid.assign(static_cast<size_t>(P.npatch) * P.nI_max, -1);
  P.B_iid.assign(static_cast<size_t>(P.npatch) * P.nB_max, -1);
  for (int p = 0; p < P.npatch; ++p) {
    std::copy(Ig[p].begin(), Ig[p].end(), P.I_gid.begin() + static_cast<size_t>(p) * P.nI_max);
    std::copy(Bi[p].begin(), Bi[p].end(), P.B_iid.begin() + static_cast<size_t>(p) * P.nB_max);
  }
  // -- interface band width
  int bw = 0;
  for (int p = 0; p < P.npatch; ++p) {
    int lo = P.niface, hi = -1;
    for (int b = 0; b < P.nB[p]; ++b) {
      const int v = P.B_iid[static_cast<size_t>(p) * P.nB_max + b];
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
    if (hi >= 0) bw = std::max(bw, hi - lo);
  }
  P.nband = bw + 1;
  return P;
}

}  // namespace stx
