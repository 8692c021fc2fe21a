#include "helmsys.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <thread>

namespace stx {

namespace {
constexpr double kEpsSP = 6.0e-7;

// In-place inverse of a dense n x n matrix by Gauss--Jordan with partial
// pivoting (the role of getrf + getri at src/element.cpp:197-211).
void invert(int n, double* A) {
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  std::vector<double> B(static_cast<size_t>(n) * 2 * n, 0.0);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) B[i * 2 * n + j] = A[i * n + j];
    B[i * 2 * n + n + i] = 1.0;
  }
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(B[r * 2 * n + c]) > std::fabs(B[p * 2 * n + c])) p = r;
    if (B[p * 2 * n + c] == 0.0) throw std::runtime_error("matrix hii is singular");
    if (p != c)
      for (int j = 0; j < 2 * n; ++j) std::swap(B[p * 2 * n + j], B[c * 2 * n + j]);
    const double d = 1.0 / B[c * 2 * n + c];
    for (int j = 0; j < 2 * n; ++j) B[c * 2 * n + j] *= d;
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = B[r * 2 * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; ++j) B[r * 2 * n + j] -= f * B[c * 2 * n + j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) A[i * n + j] = B[i * 2 * n + n + j];
}
// f(lo, hi) over [0, n) split into contiguous ranges on `nthreads` threads.
template <class F>
void parallel_ranges(int n, int nthreads, F&& f) {
  const int t = std::max(1, std::min(nthreads, n / 16));
  if (t <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int w = 0; w < t; ++w) {
    const int lo = static_cast<int>(static_cast<long long>(n) * w / t);
    const int hi = static_cast<int>(static_cast<long long>(n) * (w + 1) / t);
    pool.emplace_back([&f, lo, hi] { f(lo, hi); });
  }
  for (auto& th : pool) th.join();
}

// Same, with rows interleaved (for triangular work whose cost grows with the row).
template <class F>
void parallel_rows(int n, int nthreads, F&& f) {
  const int t = std::max(1, std::min(nthreads, n / 16));
  if (t <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  for (int w = 0; w < t; ++w)
    pool.emplace_back([&f, w, t, n] {
      for (int i = w; i < n; i += t) f(i);
    });
  for (auto& th : pool) th.join();
}
}  // namespace

void element_helmholtz(const Mesh& M, int e, double lambda2, double betak2, double* H) {
  const int n = M.np, nn = M.npnp;
  // viscous systems take the SVV-stabilised derivative (src/element.cpp:1454-1455)
  const double* D = lambda2 > 6.0e-14 && !M.svv_D.empty() ? M.svv_D.data() : M.q.D.data();
  const double* Q1 = &M.Q1[e * nn];
  const double* Q2 = &M.Q2[e * nn];
  const double* Q3 = &M.Q3[e * nn];
  const double* Q4 = &M.Q4[e * nn];
  const double hcon = lambda2 + betak2;
  for (int k = 0; k < nn * nn; ++k) H[k] = 0.0;
  // row (i,j), column (m,n) -- HelmholtzRow (src/element.cpp:1443-1480)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double* row = H + (i * n + j) * nn;
      for (int c = 0; c < n; ++c) {
        double s = 0;
        for (int q = 0; q < n; ++q) s += Q1[i * n + q] * D[q * n + j] * D[q * n + c];
        row[i * n + c] += s;
      }
      for (int m = 0; m < n; ++m) {
        double s = 0;
        for (int p = 0; p < n; ++p) s += Q2[p * n + j] * D[p * n + i] * D[p * n + m];
        row[m * n + j] += s;
      }
      for (int m = 0; m < n; ++m)
        for (int c = 0; c < n; ++c) {
          row[m * n + c] += Q3[i * n + c] * D[c * n + j] * D[i * n + m];
          row[m * n + c] += Q3[m * n + j] * D[j * n + c] * D[m * n + i];
        }
      // cylindrical: betak2 / r^2 + lambda2, zero on the axis (src/element.cpp:1450)
      const double r2 = M.cyl ? M.y[e * nn + i * n + j] * M.y[e * nn + i * n + j] : 1.0;
      row[i * n + j] += Q4[i * n + j] * (M.cyl ? (r2 > 6.0e-14 ? betak2 / r2 + lambda2 : 0.0) : hcon);
    }
}

namespace {

// Banded Cholesky A = U^T U in place, A[j*nb + t] = A(j-kd+t, j) (dpbtrf "U"),
// then the two row layouts the device sweeps read.
void factor_band(std::vector<double>& A, int ns, int nb, ModeSystem& S) {
  const int kd = nb - 1;
  for (int j = 0; j < ns; ++j) {
    double* cj = &A[static_cast<size_t>(j) * nb];
    const int i0 = std::max(0, j - kd);
    for (int i = i0; i < j; ++i) {
      const double* ci = &A[static_cast<size_t>(i) * nb];
      double s = cj[kd - (j - i)];
      const int k0 = std::max(i0, i - kd);
      for (int k = k0; k < i; ++k) s -= ci[kd - (i - k)] * cj[kd - (j - k)];
      cj[kd - (j - i)] = s / ci[kd];
    }
    double d = cj[kd];
    for (int k = i0; k < j; ++k) d -= cj[kd - (j - k)] * cj[kd - (j - k)];
    if (!(d > 0.0))
      throw std::runtime_error("failed to factor Helmholtz matrix (not positive definite)");
    cj[kd] = std::sqrt(d);
  }
  S.fwd.assign(static_cast<size_t>(ns) * nb, 0.0);
  S.bwd.assign(static_cast<size_t>(ns) * nb, 0.0);
  for (int j = 0; j < ns; ++j)
    for (int t = 0; t < nb; ++t) {
      double v = A[static_cast<size_t>(j) * nb + t];
      if (j - kd + t < 0) v = 0.0;
      S.fwd[static_cast<size_t>(j) * nb + t] = (t == kd) ? 1.0 / v : v;
    }
  for (int r = 0; r < ns; ++r) {
    const int i = ns - 1 - r;
    for (int t = 0; t < nb; ++t) {
      const int c = i + kd - t;
      double v = 0.0;
      if (c < ns) v = A[static_cast<size_t>(c) * nb + kd - (c - i)];
      S.bwd[static_cast<size_t>(r) * nb + t] = (t == kd) ? 1.0 / v : v;
    }
  }
}

}  // namespace

void spd_inverse(int n, double* A, int nthreads) {
  // A = L L^T, lower triangle in place, in column blocks of kb: the diagonal
  // block serially, then the rows below it in parallel (row i of the block
  // needs only its own earlier columns and the block's rows).
  constexpr int kb = 48;
  for (int j0 = 0; j0 < n; j0 += kb) {
    const int j1 = std::min(n, j0 + kb);
    for (int j = j0; j < j1; ++j) {
      double* aj = A + static_cast<size_t>(j) * n;
      double d = aj[j];
      for (int k = 0; k < j; ++k) d -= aj[k] * aj[k];
      if (!(d > 0.0)) throw std::runtime_error("failed to factor Helmholtz matrix (not positive definite)");
      aj[j] = std::sqrt(d);
      for (int i = j + 1; i < j1; ++i) {
        double* ai = A + static_cast<size_t>(i) * n;
        double v = ai[j];
        for (int k = 0; k < j; ++k) v -= ai[k] * aj[k];
        ai[j] = v / aj[j];
      }
    }
    parallel_ranges(n - j1, nthreads, [&](int lo, int hi) {
      for (int i = j1 + lo; i < j1 + hi; ++i) {
        double* ai = A + static_cast<size_t>(i) * n;
        for (int j = j0; j < j1; ++j) {
          const double* aj = A + static_cast<size_t>(j) * n;
          double v = ai[j];
          for (int k = 0; k < j; ++k) v -= ai[k] * aj[k];
          ai[j] = v / aj[j];
        }
      }
    });
  }
  // W = L^{-1}: column c of W solves L w = e_c (forward substitution over
  // rows i >= c); stored as row c of WT (WT[c][i] = W[i][c]).
  std::vector<double> WT(static_cast<size_t>(n) * n, 0.0);
  parallel_rows(n, nthreads, [&](int c) {
    double* w = &WT[static_cast<size_t>(c) * n];
    w[c] = 1.0 / A[static_cast<size_t>(c) * n + c];
    for (int i = c + 1; i < n; ++i) {
      const double* ai = A + static_cast<size_t>(i) * n;
      double v = 0.0;
      for (int k = c; k < i; ++k) v -= ai[k] * w[k];
      w[i] = v / ai[i];
    }
  });
  // A^{-1} = W^T W: (i, j) = sum_{k >= max(i, j)} WT[i][k] WT[j][k]
  parallel_rows(n, nthreads, [&](int i) {
    const double* ti = &WT[static_cast<size_t>(i) * n];
    for (int j = i; j < n; ++j) {
      const double* tj = &WT[static_cast<size_t>(j) * n];
      double v = 0.0;
      for (int k = j; k < n; ++k) v += ti[k] * tj[k];
      A[static_cast<size_t>(i) * n + j] = v;
    }
  });
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < i; ++j) A[static_cast<size_t>(i) * n + j] = A[static_cast<size_t>(j) * n + i];
}

ModeSystem build_mode_system(const Mesh& M, const Numbering& N, const Patching* P, double lambda2,
                             double betak2, int method, int nthreads, bool l2_device) {
  ModeSystem S;
  S.lambda2 = lambda2;
  S.betak2 = betak2;
  S.method = method;
  S.nglobal = N.nglobal;
  S.singular = (lambda2 + betak2) < kEpsSP && N.nglobal == N.nsolve && N.mixdiag.empty();
  S.nsolve = S.singular ? N.nsolve - 1 : N.nsolve;
  S.nband = N.nband;
  const int nn = M.npnp, next = M.next, nint = M.nint, nel = M.nel;
  std::vector<double> H(static_cast<size_t>(nn) * nn);

  if (method == kJacPCG) {
    S.pc.assign(N.nglobal + static_cast<size_t>(nel) * nint, 0.0);
    for (int e = 0; e < nel; ++e) {
      element_helmholtz(M, e, lambda2, betak2, H.data());
      for (int i = 0; i < next; ++i)
        S.pc[N.btog[e * next + i]] += H[static_cast<size_t>(M.emap[i]) * nn + M.emap[i]];
      for (int i = 0; i < nint; ++i) {
        const int r = M.emap[next + i];
        S.pc[N.nglobal + static_cast<size_t>(e) * nint + i] = H[static_cast<size_t>(r) * nn + r];
      }
    }
    for (size_t g = 0; g < N.mixdiag.size(); ++g) S.pc[g] += N.mixdiag[g];  // Mixed::augmentDg
    for (auto& v : S.pc) v = 1.0 / v;
    return S;
  }

  // -- per-family static condensation (Element::HelmholtzSC)
  const int nf = M.nfamily;
  S.hbi.assign(static_cast<size_t>(nf) * next * nint, 0.0);
  S.hii.assign(static_cast<size_t>(nf) * nint * nint, 0.0);
  std::vector<double> hbb_all(static_cast<size_t>(nf) * next * next);
  for (int f = 0; f < nf; ++f) {
    element_helmholtz(M, M.family_rep[f], lambda2, betak2, H.data());
    double* hbb = &hbb_all[static_cast<size_t>(f) * next * next];
    double* hbi = &S.hbi[static_cast<size_t>(f) * next * nint];
    double* hii = &S.hii[static_cast<size_t>(f) * nint * nint];
    std::vector<double> bi(static_cast<size_t>(next) * nint);
    for (int a = 0; a < next; ++a)
      for (int b = 0; b < next; ++b)
        hbb[a * next + b] = H[static_cast<size_t>(M.emap[a]) * nn + M.emap[b]];
    for (int a = 0; a < next; ++a)
      for (int b = 0; b < nint; ++b)
        bi[static_cast<size_t>(a) * nint + b] = H[static_cast<size_t>(M.emap[a]) * nn + M.emap[next + b]];
    for (int a = 0; a < nint; ++a)
      for (int b = 0; b < nint; ++b)
        hii[a * nint + b] = H[static_cast<size_t>(M.emap[next + a]) * nn + M.emap[next + b]];
    if (nint) {
      invert(nint, hii);
      for (int a = 0; a < next; ++a)
        for (int b = 0; b < nint; ++b) {
          double s = 0;
          for (int k = 0; k < nint; ++k) s += bi[static_cast<size_t>(a) * nint + k] * hii[k * nint + b];
          hbi[static_cast<size_t>(a) * nint + b] = s;
        }
      for (int a = 0; a < next; ++a)
        for (int b = 0; b < next; ++b) {
          double s = 0;
          for (int k = 0; k < nint; ++k)
            s += hbi[static_cast<size_t>(a) * nint + k] * bi[static_cast<size_t>(b) * nint + k];
          hbb[a * next + b] -= s;
        }
    }
  }

  if (P && l2_device) {
    S.hsc = hbb_all;
    S.pin_iid = S.singular ? P->pin_iid : -1;
    S.nsolve = P->niface;
    S.nband = 0;
    return S;
  }
  if (P) {
    // -- second level: per patch family, condense the patch-interior
    //    skeleton nodes; assemble the interface Schur complements.
    const int nI_max = std::max(1, P->nI_max), nB_max = std::max(1, P->nB_max);
    S.l2_sinv.assign(static_cast<size_t>(P->nfamily) * nI_max * nI_max, 0.0);
    S.l2_g.assign(static_cast<size_t>(P->nfamily) * nI_max * nB_max, 0.0);
    std::vector<std::vector<double>> T(P->nfamily);
    for (int f = 0; f < P->nfamily; ++f) {
      const int p = P->family_rep[f];
      const int nI = P->nI[p], nB = P->nB[p], nl = nI + nB;
      std::vector<double> Sp(static_cast<size_t>(nl) * nl, 0.0);
      const auto& E = P->elems[p];
      for (size_t k = 0; k < E.size(); ++k) {
        const double* hbb = &hbb_all[static_cast<size_t>(M.family[E[k]]) * next * next];
        for (int a = 0; a < next; ++a) {
          const int la = P->local[p][k * next + a];
          if (la < 0) continue;
          for (int b = 0; b < next; ++b) {
            const int lb = P->local[p][k * next + b];
            if (lb >= 0) Sp[static_cast<size_t>(la) * nl + lb] += hbb[a * next + b];
          }
        }
      }
      double* Si = &S.l2_sinv[static_cast<size_t>(f) * nI_max * nI_max];
      double* G = &S.l2_g[static_cast<size_t>(f) * nI_max * nB_max];
      std::vector<double> II(static_cast<size_t>(nI) * nI);
      for (int a = 0; a < nI; ++a)
        for (int b = 0; b < nI; ++b) II[static_cast<size_t>(a) * nI + b] = Sp[static_cast<size_t>(a) * nl + b];
      // mixed-BC diagonal of the patch-interior nodes (the family's patches
      // agree on it: it is part of the family signature)
      if (!N.mixdiag.empty())
        for (int a = 0; a < nI; ++a)
          II[static_cast<size_t>(a) * nI + a] += N.mixdiag[P->I_gid[static_cast<size_t>(p) * P->nI_max + a]];
      if (nI) spd_inverse(nI, II.data(), nthreads);  // S_II is symmetric positive definite
      for (int a = 0; a < nI; ++a)
        for (int b = 0; b < nI; ++b) Si[static_cast<size_t>(a) * nI_max + b] = II[static_cast<size_t>(a) * nI + b];
      // S_BI rows (= S_IB columns, contiguous): SB[b][c] = Sp[nI + b][c]
      std::vector<double> SB(static_cast<size_t>(nB) * std::max(nI, 1));
      for (int b = 0; b < nB; ++b)
        for (int c = 0; c < nI; ++c) SB[static_cast<size_t>(b) * nI + c] = Sp[static_cast<size_t>(nI + b) * nl + c];
      // G = S_II^-1 S_IB, GT[b][a] = G[a][b] kept for the Schur update
      std::vector<double> GT(static_cast<size_t>(nB) * std::max(nI, 1));
      parallel_ranges(nI, nthreads, [&](int lo, int hi) {
        for (int a = lo; a < hi; ++a) {
          const double* ia = &II[static_cast<size_t>(a) * nI];
          for (int b = 0; b < nB; ++b) {
            const double* sb = &SB[static_cast<size_t>(b) * nI];
            double v = 0;
            for (int c = 0; c < nI; ++c) v += ia[c] * sb[c];
            G[static_cast<size_t>(a) * nB_max + b] = v;
            GT[static_cast<size_t>(b) * nI + a] = v;
          }
        }
      });
      auto& Tf = T[f];
      Tf.assign(static_cast<size_t>(nB) * nB, 0.0);
      parallel_ranges(nB, nthreads, [&](int lo, int hi) {
        for (int a = lo; a < hi; ++a) {
          const double* sa = &SB[static_cast<size_t>(a) * nI];
          for (int b = 0; b < nB; ++b) {
            const double* gb = &GT[static_cast<size_t>(b) * nI];
            double v = Sp[static_cast<size_t>(nI + a) * nl + nI + b];
            for (int c = 0; c < nI; ++c) v -= sa[c] * gb[c];
            Tf[static_cast<size_t>(a) * nB + b] = v;
          }
        }
      });
    }
    const int ni = P->niface;
    S.hsc = hbb_all;
    std::vector<double>& A = S.l2_ainv;
    A.assign(static_cast<size_t>(ni) * ni, 0.0);
    for (int p = 0; p < P->npatch; ++p) {
      const auto& Tf = T[P->family[p]];
      const int nB = P->nB[p];
      const int* iid = &P->B_iid[static_cast<size_t>(p) * P->nB_max];
      for (int a = 0; a < nB; ++a)
        for (int b = 0; b < nB; ++b) A[static_cast<size_t>(iid[a]) * ni + iid[b]] += Tf[static_cast<size_t>(a) * nB + b];
    }
    // mixed-BC diagonal of the interface nodes (Mixed::augmentSC)
    if (!N.mixdiag.empty())
      for (int q = 0; q < ni; ++q) A[static_cast<size_t>(q) * ni + q] += N.mixdiag[P->skel_of[q]];
    if (S.singular) {
      // the pinned node is known (zero): identity row and column
      const int q = P->pin_iid;
      for (int t = 0; t < ni; ++t) {
        A[static_cast<size_t>(q) * ni + t] = 0.0;
        A[static_cast<size_t>(t) * ni + q] = 0.0;
      }
      A[static_cast<size_t>(q) * ni + q] = 1.0;
      S.pin_iid = q;
    }
    if (ni) spd_inverse(ni, A.data(), nthreads);
    S.nsolve = ni;
    S.nband = 0;
    return S;
  }

  // -- banded assembly over the first nsolve global nodes (src/matrix.cpp:218-232)
  const int ns = S.nsolve, nb = S.nband, kd = nb - 1;
  std::vector<double> A(static_cast<size_t>(ns) * nb, 0.0);  // A[j*nb + t] = A(j-kd+t, j)
  for (int e = 0; e < nel; ++e) {
    const double* hbb = &hbb_all[static_cast<size_t>(M.family[e]) * next * next];
    for (int a = 0; a < next; ++a) {
      const int m = N.btog[e * next + a];
      if (m >= ns) continue;
      for (int b = 0; b < next; ++b) {
        const int c = N.btog[e * next + b];
        if (c < ns && c >= m) {
          if (c - m > kd) throw std::runtime_error("numbering bandwidth exceeded");
          A[static_cast<size_t>(c) * nb + kd - (c - m)] += hbb[a * next + b];
        }
      }
    }
  }
  for (int j = 0; j < ns && j < static_cast<int>(N.mixdiag.size()); ++j)  // Mixed::augmentSC
    A[static_cast<size_t>(j) * nb + kd] += N.mixdiag[j];
  factor_band(A, ns, nb, S);
  return S;
}

}  // namespace stx
