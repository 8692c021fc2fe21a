// C ABI of the library: context, modal systems, solves, transforms.
//
// Host code here owns the session, mesh and numbering (FP64 setup on the
// host cores) and the device copies the kernels read.  Errors are reported
// as status codes with a thread-local message instead of the reference's
// print-and-exit (veclib/util.c:24-46).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/semtex_b200.h"
#include "host/helmsys.hpp"
#include "host/mesh.hpp"
#include "host/session.hpp"
#include "kernels/helmholtz.cuh"
#include "kernels/ptx.cuh"
#include "kernels/sweep.cuh"
#include "l2setup.hpp"
#include "kernels/element.cuh"
#include "kernels/symtile.hpp"
#include "kernels/twolevel.cuh"
#include "stx_internal.hpp"

namespace {

thread_local std::string g_last_error;

struct StxError : std::runtime_error {
  int code;
  StxError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw StxError(STX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return STX_OK;
  } catch (const StxError& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    const std::string m = e.what();
    if (m.find("positive definite") != std::string::npos || m.find("singular") != std::string::npos)
      return STX_ENUMERIC;
    if (m.find("not supported") != std::string::npos) return STX_EUNSUPPORTED;
    return STX_ESESSION;
  }
}

// An expression of x, y, z, t evaluated at many points: the compiled
// program (equal to the interpreter bit for bit), or the interpreter for
// the forms the compiler does not take (assignments inside the expression).
struct PointEvaluator {
  const stx::TokenTable& T;
  std::string expr;
  bool compiled = false;
  stx::ExprProgram P;
  std::map<std::string, double> vars;
  PointEvaluator(const stx::TokenTable& tab, const std::string& e) : T(tab), expr(e) {
    try {
      P = T.compile(e);
      compiled = true;
    } catch (const std::exception&) {
      compiled = false;
    }
  }
  double operator()(double x, double y, double z, double t) {
    if (compiled) return P.run(x, y, z, t);
    vars["x"] = x;
    vars["y"] = y;
    vars["z"] = z;
    vars["t"] = t;
    return T.eval(expr, &vars);
  }
};

}  // namespace

namespace stx {

void set_last_error(const std::string& msg) { g_last_error = msg; }

void* DeviceArena::alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 8;
  cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
  ptrs.push_back(p);
  return p;
}

DeviceArena::~DeviceArena() {
  for (void* p : ptrs) cudaFree(p);
}

void host_dft_forward(std::vector<double>& a, int nz, int n) {
  // Same contract as the device z_transform, for short BC lines.
  if (nz < 2) return;
  if (nz == 2) {
    for (int i = 0; i < n; ++i) a[n + i] = 0.0;
    return;
  }
  std::vector<double> out(a.size(), 0.0);
  const int half = nz / 2;
  for (int i = 0; i < n; ++i)
    for (int q = 0; q < nz; ++q) {
      const int kf = q == 0 ? 0 : (q == 1 ? half : q / 2);
      const bool im = q >= 2 && (q & 1);
      double v = 0;
      for (int k = 0; k < nz; ++k) {
        const double th = 2.0 * M_PI * ((static_cast<long>(kf) * k) % nz) / nz;
        v += a[static_cast<size_t>(k) * n + i] * (im ? -std::sin(th) : std::cos(th));
      }
      out[static_cast<size_t>(q) * n + i] = v / nz;
    }
  a.swap(out);
}

// Inverses of the kBandRows x kBandRows diagonal blocks of a lower-triangular
// band factor stored as rows L[j*nb + t] (column j-kd+t, 1/diagonal at t=kd).
// Block b covers rows [16b, 16b+16); rows past n are identity.
void band_block_inverses(const std::vector<double>& L, int n, int nb, double* out) {
  const int B = kBandRows, kd = nb - 1;
  for (int j0 = 0, b = 0; j0 < n; j0 += B, ++b) {
    double T[kBandRows][kBandRows] = {};
    for (int r = 0; r < B; ++r) {
      const int j = j0 + r;
      if (j >= n) {
        T[r][r] = 1.0;
        continue;
      }
      for (int s2 = 0; s2 < r; ++s2)
        if (r - s2 <= kd) T[r][s2] = L[static_cast<size_t>(j) * nb + kd - r + s2];
      T[r][r] = 1.0 / L[static_cast<size_t>(j) * nb + kd];
    }
    double* Y = out + static_cast<size_t>(b) * B * B;  // Y = T^{-1}, lower triangular
    for (int c = 0; c < B; ++c)
      for (int r = 0; r < B; ++r) {
        if (r < c) {
          Y[r * B + c] = 0.0;
          continue;
        }
        double v = (r == c) ? 1.0 : 0.0;
        for (int s2 = c; s2 < r; ++s2) v -= T[r][s2] * Y[s2 * B + c];
        Y[r * B + c] = v / T[r][r];
      }
  }
}

}  // namespace stx

using namespace stx;

// Device status word of a DIRECT system: nonzero if a bounded wait for a
// copy expired (1 banded sweep, 3 element kernels, 4 packed skeleton
// products); every wait is bounded, so the kernels return and the context
// stays usable, but the solution is not valid.  Read after synchronising.
static int status_word(const stx_modal* sys) {
  const int* st = sys->store ? sys->store->dm.status : nullptr;
  if (!st) return 0;
  int v = 0;
  cuda_check(cudaMemcpy(&v, st, sizeof(int), cudaMemcpyDeviceToHost), "status read");
  return v;
}

static void check_sweep_status(const stx_modal* sys) {
  const int v = status_word(sys);
  if (!v) return;
  const char* where = v == 1 ? "banded sweep" : v == 3 ? "element kernel" : v == 4 ? "packed skeleton product" : "solve";
  throw StxError(STX_ECUDA, std::string(where) + ": a bounded wait for a bulk copy expired");
}

// Planes between host and device: one linear copy when both sides are
// packed (plane size = points per plane), else a pitched copy.
static cudaError_t copy_planes(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows,
                               cudaMemcpyKind kind, cudaStream_t st) {
  if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * rows, kind, st);
  return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, st);
}

template <class T>
static T* upload(DeviceArena& A, const std::vector<T>& v) {
  T* p = static_cast<T*>(A.alloc(sizeof(T) * v.size()));
  if (!v.empty()) cuda_check(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
  return p;
}

extern "C" {

const char* stx_last_error(void) { return g_last_error.c_str(); }

int stx_context_create(const char* session_path, const char* overrides, int device, void* stream,
                       stx_context** out) {
  return guarded([&] {
    if (!session_path || !out) throw StxError(STX_EINVAL, "null argument");
    *out = nullptr;
    auto ctx = std::make_unique<stx_context>();
    ctx->S = read_session(session_path, overrides ? overrides : "");
    if (ctx->S.tokens.ivalue("CYLINDRICAL"))
      throw StxError(STX_EUNSUPPORTED, "cylindrical coordinates are not supported");
    ctx->M = build_mesh(ctx->S);
    ctx->device = device;
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    if (stream) {
      ctx->stream = static_cast<cudaStream_t>(stream);
      ctx->own_stream = false;
    } else {
      cuda_check(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
      ctx->own_stream = true;
    }
    const Mesh& M = ctx->M;
    DeviceArena& A = ctx->arena;
    DevGeom& g = ctx->dg;
    g.np = M.np;
    g.nel = M.nel;
    g.nz = M.nz;
    g.npnp = M.npnp;
    g.next = M.next;
    g.nint = M.nint;
    g.plane_size = M.plane_size;
    // the DNS step's own kernels launch programmatically dependent only on
    // request (token STX_PDL_STEP = 1; measured slower on the 24x24x96
    // Taylor-Green step); the solves' kernels do by default (STX_PDL)
    g.pdl = ctx->S.tokens.has("STX_PDL_STEP") && ctx->S.tokens.ivalue("STX_PDL_STEP") != 0;
    g.D = upload(A, M.q.D);
    g.Q1 = upload(A, M.Q1);
    g.Q2 = upload(A, M.Q2);
    g.Q3 = upload(A, M.Q3);
    g.Q4 = upload(A, M.Q4);
    g.drdx = upload(A, M.drdx);
    g.drdy = upload(A, M.drdy);
    g.dsdx = upload(A, M.dsdx);
    g.dsdy = upload(A, M.dsdy);
    g.emap = upload(A, M.emap);
    g.pmap = upload(A, M.pmap);
    g.family = upload(A, M.family);
    {
      // chunks of up to 32 same-family elements (fewer when the recovery
      // kernel's shared-memory plan would exceed 200 KB; token STX_CHUNK
      // caps the count, the autotuner's element-chunk choice)
      int cm = 32;
      if (ctx->S.tokens.has("STX_CHUNK")) {
        const int want = ctx->S.tokens.ivalue("STX_CHUNK");
        if (want < 1 || want > 32) throw StxError(STX_EINVAL, "STX_CHUNK must be in 1..32");
        cm = want;
      }
      auto need = [&](int c) {  // shared memory of the batched recovery kernel
        return sizeof(double) * (2 * static_cast<size_t>(c) * (M.npnp | 1) + 2 * static_cast<size_t>(c) * (M.next | 1) +
                                 24 * M.npnp + M.np * M.np);
      };
      while (cm > 1 && need(cm) > 200 * 1024) cm /= 2;
      std::vector<int> sorted(M.nel);
      for (int e = 0; e < M.nel; ++e) sorted[e] = e;
      std::stable_sort(sorted.begin(), sorted.end(), [&](int a, int b) { return M.family[a] < M.family[b]; });
      std::vector<int> cstart, ccount;
      for (int i = 0; i < M.nel;) {
        int j = i;
        while (j < M.nel && j - i < cm && M.family[sorted[j]] == M.family[sorted[i]]) ++j;
        cstart.push_back(i);
        ccount.push_back(j - i);
        i = j;
      }
      g.nchunk = static_cast<int>(cstart.size());
      g.chunk_max = cm;
      g.chunk_start = upload(A, cstart);
      g.chunk_count = upload(A, ccount);
      g.elem_sorted = upload(A, sorted);
      ctx->elem_sorted = sorted;
      std::vector<int4> desc(cstart.size());
      for (size_t k = 0; k < cstart.size(); ++k)
        desc[k] = make_int4(cstart[k], ccount[k], M.family[sorted[cstart[k]]], 0);
      g.chunk_desc = upload(A, desc);
    }
    std::vector<double> tw(2 * std::max(1, M.nz));
    for (int m = 0; m < M.nz; ++m) {
      tw[m] = std::cos(2.0 * M_PI * m / M.nz);
      tw[M.nz + m] = std::sin(2.0 * M_PI * m / M.nz);
    }
    ctx->d_twiddle = upload(A, tw);
    for (char c : ctx->S.fields) {
      FieldDev& F = ctx->fields[c];
      F.N = build_numbering(ctx->S, M, c);
      const Numbering& N = F.N;
      DevNumbering& d = F.dn;
      d.nglobal = N.nglobal;
      d.nsolve = N.nsolve;
      d.nband = N.nband;
      d.btog = upload(A, N.btog);
      d.bmask = upload(A, N.bmask);
      d.emask = upload(A, N.emask);
      d.imass = upload(A, N.imass);
      d.nedge = static_cast<int>(N.edges.size());
      std::vector<int> gid, kind;
      std::vector<double> area;
      for (const auto& E : N.edges) {
        for (int t = 0; t < M.np; ++t) {
          gid.push_back(N.btog[E.elmt * M.next + (E.side * (M.np - 1) + t) % M.next]);
          area.push_back(E.area[t]);
        }
        // NaturalCBCp::sum is Natural::sum (src/condition.cpp:470-495); Mixed::sum
        // adds K C w, the line value of an 'M' edge (:315-343); a computed
        // outflow edge is essential for the pressure (EssentialCBCp) and
        // natural for the velocities (NaturalCBCu), its values computed per
        // step (src/bcmgr.cpp:416-431)
        char k = E.kind;
        if (k == 'H' || k == 'M') k = 'N';
        if (k == 'O') k = c == 'p' ? 'D' : 'N';
        kind.push_back(k);
      }
      d.ness = static_cast<int>(std::count(kind.begin(), kind.end(), static_cast<int>('D')));
      d.nnat = static_cast<int>(std::count(kind.begin(), kind.end(), static_cast<int>('N')));
      d.edge_gid = upload(A, gid);
      d.edge_kind = upload(A, kind);
      d.mixdiag = F.N.mixdiag.empty() ? nullptr : upload(A, F.N.mixdiag);
      d.edge_area = upload(A, area);
      F.nline = d.nedge * M.np;
      F.d_lines = static_cast<double*>(A.alloc(sizeof(double) * std::max(1, F.nline) * M.nz));
      cuda_check(cudaMemset(F.d_lines, 0, sizeof(double) * std::max(1, F.nline) * M.nz), "memset");
    }
    *out = ctx.release();
    for (char c : (*out)->S.fields) stx_field_bc_evaluate(*out, c, 0.0);
    if (!g_last_error.empty()) {
      std::string m = g_last_error;
      stx_context_destroy(*out);
      *out = nullptr;
      throw StxError(STX_ESESSION, m);
    }
  });
}

int stx_context_destroy(stx_context* ctx) {
  return guarded([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto* m : ctx->modals) delete m;
    ctx->modals.clear();
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
  });
}

int stx_context_geometry(const stx_context* ctx, int* np, int* nz, int* nel, int* plane_size) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    if (np) *np = ctx->M.np;
    if (nz) *nz = ctx->M.nz;
    if (nel) *nel = ctx->M.nel;
    if (plane_size) *plane_size = ctx->M.plane_size;
  });
}

int stx_context_fields(const stx_context* ctx, char* buf, int len) {
  return guarded([&] {
    if (!ctx || !buf) throw StxError(STX_EINVAL, "null argument");
    if (static_cast<int>(ctx->S.fields.size()) + 1 > len) throw StxError(STX_EINVAL, "buffer too small");
    std::strcpy(buf, ctx->S.fields.c_str());
  });
}

int stx_token(const stx_context* ctx, const char* expr, double* value) {
  return guarded([&] {
    if (!ctx || !expr || !value) throw StxError(STX_EINVAL, "null argument");
    *value = ctx->S.tokens.value(expr);
  });
}

int stx_numbering(const stx_context* ctx, char field, int* nglobal, int* nsolve, int* nband) {
  return guarded([&] {
    auto it = ctx->fields.find(field);
    if (it == ctx->fields.end()) throw StxError(STX_EINVAL, std::string("no field ") + field);
    if (nglobal) *nglobal = it->second.N.nglobal;
    if (nsolve) *nsolve = it->second.N.nsolve;
    if (nband) *nband = it->second.N.nband;
  });
}

int stx_numbering_host(const char* session_path, const char* overrides, char field, int* nel, int* next,
                       int* nglobal, int* nsolve, int* nband, int* h_btog, int* h_bmask) {
  return stx_numbering_host_mode(session_path, overrides, field, 0, nel, next, nglobal, nsolve, nband, h_btog,
                                 h_bmask);
}

int stx_numbering_host_mode(const char* session_path, const char* overrides, char field, int mode, int* nel,
                            int* next, int* nglobal, int* nsolve, int* nband, int* h_btog, int* h_bmask) {
  return guarded([&] {
    if (!session_path || mode < 0) throw StxError(STX_EINVAL, "bad argument");
    const Session S = read_session(session_path, overrides ? overrides : "");
    if (S.fields.find(field) == std::string::npos) throw StxError(STX_EINVAL, std::string("no field ") + field);
    const Mesh M = build_mesh(S);
    bool axis = false;
    for (const auto& g : S.bcs)
      for (const auto& f : g.second) axis = axis || f.second.kind == 'A';
    const int mclass = M.cyl && M.nz > 1 && axis ? std::min(mode, 2) : 0;
    const Numbering N = build_numbering(S, M, field, 48, mclass);
    if (nel) *nel = M.nel;
    if (next) *next = M.next;
    if (nglobal) *nglobal = N.nglobal;
    if (nsolve) *nsolve = N.nsolve;
    if (nband) *nband = N.nband;
    if (h_btog) std::memcpy(h_btog, N.btog.data(), sizeof(int) * N.btog.size());
    if (h_bmask) std::memcpy(h_bmask, N.bmask.data(), sizeof(int) * N.bmask.size());
  });
}

int stx_element_matrix_host(const char* session_path, const char* overrides, int elmt, double lambda2,
                            double betak2, int* np, double* h_matrix) {
  return guarded([&] {
    if (!session_path) throw StxError(STX_EINVAL, "null argument");
    const Session S = read_session(session_path, overrides ? overrides : "");
    const Mesh M = build_mesh(S);
    if (elmt < 0 || elmt >= M.nel) throw StxError(STX_EINVAL, "element out of range");
    if (np) *np = M.np;
    if (h_matrix) element_helmholtz(M, elmt, lambda2, betak2, h_matrix);
  });
}

int stx_mesh_coords(const stx_context* ctx, double* h_x, double* h_y) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    if (h_x) std::memcpy(h_x, ctx->M.x.data(), sizeof(double) * ctx->M.x.size());
    if (h_y) std::memcpy(h_y, ctx->M.y.data(), sizeof(double) * ctx->M.y.size());
  });
}

int stx_mesh_mass(const stx_context* ctx, double* h_q4) {
  return guarded([&] {
    if (!ctx || !h_q4) throw StxError(STX_EINVAL, "null argument");
    std::memcpy(h_q4, ctx->M.Q4.data(), sizeof(double) * ctx->M.Q4.size());
  });
}

namespace {

void locate_points(const Session& S, const Mesh& M, int npts, const double* xy, int* h_elmt, double* h_rs) {
  if (npts < 0 || (npts > 0 && (!xy || !h_elmt || !h_rs))) throw StxError(STX_EINVAL, "null argument");
  const double tol = S.tokens.value("TOL_POS");
  const int maxit = S.tokens.ivalue("NR_MAX");
  for (int i = 0; i < npts; ++i) {
    double r = 0.0, s = 0.0;
    h_elmt[i] = locate_point(M, xy[2 * i], xy[2 * i + 1], tol, maxit, r, s);
    h_rs[2 * i] = h_elmt[i] >= 0 ? r : 0.0;
    h_rs[2 * i + 1] = h_elmt[i] >= 0 ? s : 0.0;
  }
}

// FluidParticle::integrate's search (src/particle.cpp:155-175): Newton's
// iteration in the point's element from its (r, s), else the full search.
void relocate_points(const Session& S, const Mesh& M, int npts, const double* xy, int* h_elmt, double* h_rs) {
  if (npts < 0 || (npts > 0 && (!xy || !h_elmt || !h_rs))) throw StxError(STX_EINVAL, "null argument");
  const double tol = S.tokens.value("TOL_POS");
  const int maxit = S.tokens.ivalue("NR_MAX");
  for (int i = 0; i < npts; ++i) {
    const int e = h_elmt[i];
    if (e >= M.nel) throw StxError(STX_EINVAL, "element out of range");
    double r = h_rs[2 * i], s = h_rs[2 * i + 1];
    if (e >= 0 && element_locate(M, e, xy[2 * i], xy[2 * i + 1], tol, maxit, false, r, s)) {
      h_rs[2 * i] = r;
      h_rs[2 * i + 1] = s;
      continue;
    }
    h_elmt[i] = locate_point(M, xy[2 * i], xy[2 * i + 1], tol, maxit, r, s);
    h_rs[2 * i] = h_elmt[i] >= 0 ? r : 0.0;
    h_rs[2 * i + 1] = h_elmt[i] >= 0 ? s : 0.0;
  }
}

}  // namespace

int stx_mesh_relocate(const stx_context* ctx, int npts, const double* xy, int* h_elmt, double* h_rs) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    relocate_points(ctx->S, ctx->M, npts, xy, h_elmt, h_rs);
  });
}

int stx_mesh_relocate_host(const char* session_path, const char* overrides, int npts, const double* xy,
                           int* h_elmt, double* h_rs) {
  return guarded([&] {
    if (!session_path) throw StxError(STX_EINVAL, "null argument");
    const Session S = read_session(session_path, overrides ? overrides : "");
    relocate_points(S, build_mesh(S), npts, xy, h_elmt, h_rs);
  });
}

int stx_mesh_locate(const stx_context* ctx, int npts, const double* xy, int* h_elmt, double* h_rs) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    locate_points(ctx->S, ctx->M, npts, xy, h_elmt, h_rs);
  });
}

int stx_mesh_locate_host(const char* session_path, const char* overrides, int npts, const double* xy, int* h_elmt,
                         double* h_rs) {
  return guarded([&] {
    if (!session_path) throw StxError(STX_EINVAL, "null argument");
    const Session S = read_session(session_path, overrides ? overrides : "");
    locate_points(S, build_mesh(S), npts, xy, h_elmt, h_rs);
  });
}

int stx_mesh_families(const stx_context* ctx, int* nfamily) {
  return guarded([&] {
    if (!ctx || !nfamily) throw StxError(STX_EINVAL, "null argument");
    *nfamily = ctx->M.nfamily;
  });
}


int stx_field_evaluate(const stx_context* ctx, const char* expr, double t, double* h_out) {
  return guarded([&] {
    if (!ctx || !expr || !h_out) throw StxError(STX_EINVAL, "null argument");
    const Mesh& M = ctx->M;
    const double dz = 2.0 * M_PI / ctx->S.tokens.value("BETA") / M.nz;
    PointEvaluator f(ctx->S.tokens, expr);
    for (int k = 0; k < M.nz; ++k)
      for (int i = 0; i < M.nplane; ++i)
        h_out[static_cast<size_t>(k) * M.nplane + i] = f(M.x[i], M.y[i], k * dz, t);
  });
}

int stx_expression_eval(const char* expr, const char* assignments, int compiled, int n, const double* x,
                        const double* y, const double* z, double t, double* out, int* nops) {
  return guarded([&] {
    if (!expr || n < 0 || (n > 0 && (!x || !y || !z || !out))) throw StxError(STX_EINVAL, "bad argument");
    TokenTable T;
    if (assignments) {
      std::string all(assignments), item;
      for (size_t a = 0; a <= all.size();) {
        size_t b = all.find(';', a);
        if (b == std::string::npos) b = all.size();
        item = all.substr(a, b - a);
        if (item.find_first_not_of(" \t") != std::string::npos) T.assign(item);
        a = b + 1;
      }
    }
    if (compiled) {
      const ExprProgram P = T.compile(expr);
      if (nops) *nops = static_cast<int>(P.ops.size());
      for (int i = 0; i < n; ++i) out[i] = P.run(x[i], y[i], z[i], t);
    } else {
      if (nops) *nops = 0;
      std::map<std::string, double> vars;
      vars["t"] = t;
      for (int i = 0; i < n; ++i) {
        vars["x"] = x[i];
        vars["y"] = y[i];
        vars["z"] = z[i];
        out[i] = T.eval(expr, &vars);
      }
    }
  });
}

int stx_session_force_value(const char* session_path, const char* token, char* buf, int len, int* found) {
  return guarded([&] {
    if (!session_path || !token || !buf || len < 1 || !found) throw StxError(STX_EINVAL, "bad argument");
    const Session S = read_session(session_path, "");
    std::string v;
    *found = S.force_value(token, v) ? 1 : 0;
    if (!*found) v.clear();
    if (static_cast<int>(v.size()) >= len) throw StxError(STX_EINVAL, "buffer too short");
    std::memcpy(buf, v.c_str(), v.size() + 1);
  });
}

int stx_svv(int np, double eps_n, int m_n, int nz, double eps_z, int m_z, double kinvis, double* d_matrix,
            double* z_factors) {
  return guarded([&] {
    if (np < 2 || nz < 1 || !(kinvis > 0.0)) throw StxError(STX_EINVAL, "bad argument");
    if (d_matrix) {
      const Quadrature q = gll(np);
      std::vector<double> D = svv_derivative(q, eps_n, m_n, kinvis);
      if (D.empty()) D = q.D;
      std::copy(D.begin(), D.end(), d_matrix);
    }
    if (z_factors) {
      const std::vector<double> S = svv_z(nz, (nz + 1) / 2, eps_z, m_z, kinvis);
      std::copy(S.begin(), S.end(), z_factors);
    }
  });
}

int stx_field_bc_evaluate(stx_context* ctx, char field, double t) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    auto it = ctx->fields.find(field);
    if (it == ctx->fields.end()) throw StxError(STX_EINVAL, std::string("no field ") + field);
    FieldDev& F = it->second;
    const Mesh& M = ctx->M;
    const int nz = M.nz, np = M.np;
    if (F.nline == 0) return;
    const double dz = 2.0 * M_PI / ctx->S.tokens.value("BETA") / nz;
    std::vector<double> line(static_cast<size_t>(F.nline) * nz, 0.0);
    std::map<std::string, PointEvaluator> evals;  // one per distinct expression
    for (int k = 0; k < nz; ++k) {
      for (size_t b = 0; b < F.N.edges.size(); ++b) {
        const BoundaryEdge& E = F.N.edges[b];
        // high-order pressure values are computed on the device each step
        if (E.kind == 'H' || E.kind == 'M') continue;
        auto it = evals.find(E.expr);
        if (it == evals.end()) it = evals.emplace(E.expr, PointEvaluator(ctx->S.tokens, E.expr)).first;
        for (int q = 0; q < np; ++q)
          line[static_cast<size_t>(k) * F.nline + b * np + q] = it->second(E.x[q], E.y[q], k * dz, t);
      }
    }
    host_dft_forward(line, nz, F.nline);
    // Mixed::sum adds K C <1, w> on every plane (src/condition.cpp:315-343)
    for (size_t b = 0; b < F.N.edges.size(); ++b) {
      const BoundaryEdge& E = F.N.edges[b];
      if (E.kind != 'M') continue;
      for (int k = 0; k < nz; ++k)
        for (int q = 0; q < np; ++q) line[static_cast<size_t>(k) * F.nline + b * np + q] = E.mix_K * E.mix_C;
    }
    cuda_check(cudaMemcpyAsync(F.d_lines, line.data(), sizeof(double) * line.size(),
                               cudaMemcpyHostToDevice, ctx->stream),
               "bc upload");
    cuda_check(cudaStreamSynchronize(ctx->stream), "bc sync");
  });
}

int stx_modal_create(stx_context* ctx, char field, double lambda2, double beta, int base_mode,
                     int num_modes, int method, stx_modal** out) {
  return guarded([&] {
    if (!ctx || !out) throw StxError(STX_EINVAL, "null argument");
    *out = nullptr;
    auto it = ctx->fields.find(field);
    if (it == ctx->fields.end()) throw StxError(STX_EINVAL, std::string("no field ") + field);
    if (method != STX_DIRECT && method != STX_JACPCG && method != STX_MIXED)
      throw StxError(STX_EINVAL, "unknown method");
    const bool direct = method != STX_JACPCG;  // DIRECT, or DIRECT with FP32 skeleton matrices
    const int nmode_total = (ctx->M.nz + 1) / 2;
    if (base_mode != 0 || num_modes != nmode_total)
      throw StxError(STX_EINVAL, "a single-device context holds all modes: base 0, nz/2 modes");
    cudaSetDevice(ctx->device);
    const Numbering& N = it->second.N;
    auto sys = std::make_unique<stx_modal>();
    sys->ctx = ctx;
    sys->field = field;
    sys->method = method;
    // -- share storage with an existing system of equal constants/numbering
    for (auto* o : ctx->modals)
      if (o->method == method && std::fabs(o->lambda2 - lambda2) < 6e-14 &&
          std::fabs(o->beta - beta) < 6e-14 && ctx->fields.at(o->field).N.same_as(N)) {
        sys->store = o->store;
        break;
      }
    sys->lambda2 = lambda2;
    sys->beta = beta;
    if (!sys->store) {
      auto st = std::make_shared<ModalStore>();
      const Mesh& M = ctx->M;
      const Patching* P = nullptr;
      if (direct) P = ctx->patching(field);
      if (method == STX_MIXED && !P)
        throw StxError(STX_EUNSUPPORTED, "mixed precision needs the two-level skeleton solve");
      std::vector<ModeSystem> modes(num_modes);
      std::vector<std::string> errs(num_modes);
      // two-level systems form their patch and interface matrices on the
      // device (token STX_SETUP_HOST = 1: on the host, for comparison)
      const bool l2_device = P && !(ctx->S.tokens.has("STX_SETUP_HOST") && ctx->S.tokens.ivalue("STX_SETUP_HOST"));
      // viscous systems: beta^2 k^2 scaled by the SVV factors of the modes
      // (src/matrix.cpp:78-83)
      const TokenTable& T = ctx->S.tokens;
      const std::vector<double> svz =
          lambda2 > 6.0e-14 ? svv_z(M.nz, num_modes, T.value("SVV_EPSZ"), static_cast<int>(T.value("SVV_MZ")),
                                    T.value("KINVIS"))
                            : std::vector<double>(num_modes, 1.0);
      const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
      unsigned nth = std::max(1u, std::min<unsigned>(hw, num_modes));
      const int inner = static_cast<int>(std::max(1u, hw / nth));  // threads of each mode's dense inverses
      std::vector<std::thread> pool;
      for (unsigned w = 0; w < nth; ++w)
        pool.emplace_back([&, w] {
          for (int m = static_cast<int>(w); m < num_modes; m += nth) {
            try {
              const double bk = beta * (base_mode + m);
              modes[m] = build_mode_system(M, N, P, lambda2, bk * bk * svz[m], method, inner, l2_device);
            } catch (const std::exception& e) {
              errs[m] = e.what();
            }
          }
        });
      for (auto& th : pool) th.join();
      for (auto& e : errs)
        if (!e.empty()) throw StxError(STX_ENUMERIC, e);
      DevModal& d = st->dm;
      d.nmodes = num_modes;
      d.method = method;
      d.nfamily = M.nfamily;
      d.sym_warps = 4;
      d.sym_regcap = 0;
      d.elem_twoblock = ctx->S.tokens.has("STX_ELEM_TWOBLOCK") && ctx->S.tokens.ivalue("STX_ELEM_TWOBLOCK") != 0;
      d.pdl = !ctx->S.tokens.has("STX_PDL") || ctx->S.tokens.ivalue("STX_PDL") != 0;
      // bound of the kernels' bounded waits (token STX_WAIT_NS, default 2 s;
      // 0: one non-blocking probe, which a copy issued just before misses --
      // the error path's tests use it)
      d.wait_ns = kWaitNs;
      if (ctx->S.tokens.has("STX_WAIT_NS")) {
        const double w = ctx->S.tokens.value("STX_WAIT_NS");
        if (!(w >= 0.0)) throw StxError(STX_EINVAL, "STX_WAIT_NS must be at least 0");
        d.wait_ns = static_cast<unsigned long long>(std::min(w, 6.0e10));
      }
      d.nband = N.nband;
      std::vector<double> lam(num_modes), bk2(num_modes);
      std::vector<int> ns(num_modes);
      int nsmax = 0;
      for (int m = 0; m < num_modes; ++m) {
        lam[m] = modes[m].lambda2;
        bk2[m] = modes[m].betak2;
        // skeleton unknowns of the mode (the pinned node excluded)
        ns[m] = P ? (modes[m].singular ? N.nsolve - 1 : N.nsolve) : modes[m].nsolve;
        nsmax = std::max(nsmax, ns[m]);
      }
      st->nsolve = ns;
      d.ns_stride = nsmax;
      d.lambda2 = upload(st->arena, lam);
      d.betak2 = upload(st->arena, bk2);
      d.D = lambda2 > 6.0e-14 && !M.svv_D.empty() ? upload(st->arena, M.svv_D) : ctx->dg.D;
      d.nsolve = upload(st->arena, ns);
      d.l2 = 0;
      d.ew = d.eb = nullptr;
      d.ew_ld = d.eb_ld = 0;
      if (direct) {
        // Element operators for the element kernels, per family and mode
        // (rows zero-padded to element_ld): the recovery operator row i, with
        // columns in the natural node order of the recovery's columns,
        // = (-hbi[b][i] at the element-boundary nodes, hii^-1[i][j] at the
        // interior nodes), so the interior solution is one product with the
        // column (u_b at the boundary nodes, F_i at the interior nodes); the
        // condensation operator row b = hbi[b][.] (interior nodes in
        // boundary-major order, as the condensation's columns).
        const int nx = M.next, ni = M.nint, nn = M.npnp, ldw = element_ld(nn), ldc = element_ld(ni);
        const size_t nf = static_cast<size_t>(num_modes) * M.nfamily;
        std::vector<double> ew(nf * ni * ldw, 0.0), eb(nf * nx * ldc, 0.0);
        for (int m = 0; m < num_modes; ++m)
          for (int f = 0; f < M.nfamily; ++f) {
            const size_t fm = static_cast<size_t>(m) * M.nfamily + f;
            const double* hb = modes[m].hbi.data() + static_cast<size_t>(f) * nx * ni;
            const double* hi = modes[m].hii.data() + static_cast<size_t>(f) * ni * ni;
            double* w = ew.data() + fm * ni * ldw;
            double* c = eb.data() + fm * nx * ldc;
            for (int t = 0; t < nn; ++t) {
              const int p = M.pmap[t];
              for (int i = 0; i < ni; ++i)
                w[static_cast<size_t>(i) * ldw + t] =
                    p < nx ? -hb[static_cast<size_t>(p) * ni + i] : hi[static_cast<size_t>(i) * ni + p - nx];
            }
            for (int b = 0; b < nx; ++b)
              for (int j = 0; j < ni; ++j) c[static_cast<size_t>(b) * ldc + j] = hb[static_cast<size_t>(b) * ni + j];
          }
        d.ew = upload(st->arena, ew.empty() ? std::vector<double>{0.0, 0.0} : ew);
        d.eb = upload(st->arena, eb.empty() ? std::vector<double>{0.0, 0.0} : eb);
        d.ew_ld = ldw;
        d.eb_ld = ldc;
      }
      if (direct && P) {
        // Two-level data: the patch-interior inverses S_II^-1 (one per patch
        // family and mode) and the interface inverse (one per mode), packed
        // symmetric; the element Schur complements (rows padded to
        // element_ld); per element node (chunk order) its skeleton id and
        // class (essential / patch-interior / interface).
        const int nx = M.next;
        std::vector<double> hbi, hii, sc, pack;
        const int ldsc = element_ld(nx);
        std::vector<long long> fam_off(static_cast<size_t>(num_modes) * P->nfamily), if_off(num_modes);
        std::vector<long long> g_off(static_cast<size_t>(num_modes) * P->nfamily);
        const size_t nB_max = std::max(1, P->nB_max);
        std::vector<int> pin(num_modes, -1);
        const size_t nI_max = std::max(1, P->nI_max);
        // packed layout per mode: S_II^-1 of each patch family, G of each
        // patch family, the interface inverse
        long long pack_total = 0;
        for (int m = 0; m < num_modes; ++m) {
          for (int f = 0; f < P->nfamily; ++f) {
            fam_off[static_cast<size_t>(m) * P->nfamily + f] = pack_total;
            pack_total += sym_size(P->nI[P->family_rep[f]]);
          }
          for (int f = 0; f < P->nfamily; ++f) {
            const int rep = P->family_rep[f];
            g_off[static_cast<size_t>(m) * P->nfamily + f] = pack_total;
            pack_total += gen_size(P->nI[rep], P->nB[rep]);
          }
          if_off[m] = pack_total;
          pack_total += sym_size(P->niface);
        }
        std::vector<double> hbb_dev;
        for (int m = 0; m < num_modes; ++m) {
          hbi.insert(hbi.end(), modes[m].hbi.begin(), modes[m].hbi.end());
          hii.insert(hii.end(), modes[m].hii.begin(), modes[m].hii.end());
          for (int f = 0; f < M.nfamily; ++f) {
            const double* h = modes[m].hsc.data() + static_cast<size_t>(f) * nx * nx;
            for (int a = 0; a < nx; ++a)
              for (int b = 0; b < ldsc; ++b) sc.push_back(b < nx ? h[static_cast<size_t>(a) * nx + b] : 0.0);
          }
          pin[m] = modes[m].pin_iid;
          if (l2_device) {
            hbb_dev.insert(hbb_dev.end(), modes[m].hsc.begin(), modes[m].hsc.end());
            modes[m] = ModeSystem();
            continue;
          }
          for (int f = 0; f < P->nfamily; ++f) {
            const int n = P->nI[P->family_rep[f]];
            fam_off[static_cast<size_t>(m) * P->nfamily + f] = static_cast<long long>(pack.size());
            pack.resize(pack.size() + sym_size(n), 0.0);
            sym_pack(n, modes[m].l2_sinv.data() + static_cast<size_t>(f) * nI_max * nI_max, nI_max,
                     pack.data() + fam_off[static_cast<size_t>(m) * P->nfamily + f]);
          }
          for (int f = 0; f < P->nfamily; ++f) {
            const int rep = P->family_rep[f], nI = P->nI[rep], nB = P->nB[rep];
            g_off[static_cast<size_t>(m) * P->nfamily + f] = static_cast<long long>(pack.size());
            pack.resize(pack.size() + gen_size(nI, nB), 0.0);
            gen_pack(nI, nB, modes[m].l2_g.data() + static_cast<size_t>(f) * nI_max * nB_max, nB_max,
                     pack.data() + g_off[static_cast<size_t>(m) * P->nfamily + f]);
          }
          if_off[m] = static_cast<long long>(pack.size());
          pack.resize(pack.size() + sym_size(P->niface), 0.0);
          sym_pack(P->niface, modes[m].l2_ainv.data(), P->niface, pack.data() + if_off[m]);
          pin[m] = modes[m].pin_iid;
          modes[m] = ModeSystem();
        }
        // per node of the elements in chunk order: skeleton id << 2 | class
        std::vector<int> ncode(static_cast<size_t>(M.nel) * nx, 0);
        for (int i = 0; i < M.nel; ++i) {
          const int e = ctx->elem_sorted[i];
          for (int a = 0; a < nx; ++a) {
            const int gi = N.btog[static_cast<size_t>(e) * nx + a];
            const int cls = gi >= N.nsolve ? 0 : (P->iface_of[gi] >= 0 ? 2 : 1);
            ncode[static_cast<size_t>(i) * nx + a] = gi << 2 | cls;
          }
        }
        d.l2 = 1;
        d.npatch = P->npatch;
        d.pfam = P->nfamily;
        d.nI_max = P->nI_max;
        d.nB_max = P->nB_max;
        d.niface = P->niface;
        d.p_family = upload(st->arena, P->family);
        d.p_nI = upload(st->arena, P->nI);
        d.p_nB = upload(st->arena, P->nB);
        d.p_Igid = upload(st->arena, P->I_gid);
        d.p_Biid = upload(st->arena, P->B_iid);
        d.skel_of = upload(st->arena, P->skel_of.empty() ? std::vector<int>{0} : P->skel_of);
        // skeleton ids of each patch's interface nodes (columns of its G)
        std::vector<int> bgid(P->B_iid.size(), 0);
        for (size_t k = 0; k < bgid.size(); ++k) bgid[k] = P->B_iid[k] >= 0 ? P->skel_of[P->B_iid[k]] : 0;
        const int* d_bgid = upload(st->arena, bgid.empty() ? std::vector<int>{0} : bgid);
        d.pin = upload(st->arena, pin);
        d.hbi = upload(st->arena, hbi);
        d.hii = upload(st->arena, hii);
        if (method == STX_MIXED) {
          // FP32 copies of the packed matrices (same entry offsets) and the
          // number of FP64 refinement steps (token STX_REFINE, default 2)
          for (int m = 0; m < num_modes; ++m)
            if (pin[m] >= 0) throw StxError(STX_EUNSUPPORTED, "mixed precision needs a non-singular system");
          if (!N.mixdiag.empty()) throw StxError(STX_EUNSUPPORTED, "mixed precision with mixed (Robin) BCs");
          if (l2_device) {
            DeviceArena t64;
            const size_t np64 = std::max<long long>(pack_total, 32);
            double* d64 = static_cast<double*>(t64.alloc(sizeof(double) * np64));
            cuda_check(cudaMemsetAsync(d64, 0, sizeof(double) * np64, ctx->stream), "pack memset");
            l2_device_setup_guarded(M, N, *P, hbb_dev, num_modes, pin, fam_off, g_off, if_off, d64, ctx->stream);
            float* d32 = static_cast<float*>(st->arena.alloc(sizeof(float) * np64));
            cuda_check(to_float(d64, d32, np64, ctx->stream), "pack to FP32");
            cuda_check(cudaStreamSynchronize(ctx->stream), "pack sync");
            d.l2_pack32 = d32;
          } else {
            std::vector<float> p32(pack.begin(), pack.end());
            if (p32.empty()) p32.assign(32, 0.0f);
            d.l2_pack32 = upload(st->arena, p32);
          }
          d.l2_pack = nullptr;
          d.refine = ctx->S.tokens.has("STX_REFINE") ? ctx->S.tokens.ivalue("STX_REFINE") : 2;
          if (d.refine < 0) throw StxError(STX_EINVAL, "STX_REFINE must be at least 0");
        } else if (l2_device) {
          const size_t np64 = std::max<long long>(pack_total, 32);
          double* d64 = static_cast<double*>(st->arena.alloc(sizeof(double) * np64));
          cuda_check(cudaMemsetAsync(d64, 0, sizeof(double) * np64, ctx->stream), "pack memset");
          l2_device_setup_guarded(M, N, *P, hbb_dev, num_modes, pin, fam_off, g_off, if_off, d64, ctx->stream);
          d.l2_pack = d64;
        } else {
          d.l2_pack = upload(st->arena, pack.empty() ? std::vector<double>(32, 0.0) : pack);
        }
        d.l2_sc = upload(st->arena, sc);
        d.l2_sc_ld = ldsc;
        d.l2_ncode = upload(st->arena, ncode);
        // products: S_II^-1 and -G per (patch, mode), the interface inverse
        // per mode; each streamed by warps in equal runs of tiles
        std::vector<SymProblem> pp, pi, pg;
        for (int m = 0; m < num_modes; ++m)
          for (int p = 0; p < P->npatch; ++p) {
            if (P->nI[p] <= 0) continue;
            const size_t fm = static_cast<size_t>(m) * P->nfamily + P->family[p];
            const int* rows = d.p_Igid + static_cast<size_t>(p) * nI_max;
            pp.push_back(SymProblem{fam_off[fm], P->nI[p], m, -1, rows, 0, nullptr, 1.0});
            if (P->nB[p] > 0)
              pg.push_back(SymProblem{g_off[fm], P->nI[p], m, -1, rows, P->nB[p], d_bgid + static_cast<size_t>(p) * nB_max,
                                      -1.0});
          }
        if (P->niface > 0)
          for (int m = 0; m < num_modes; ++m)
            pi.push_back(SymProblem{if_off[m], P->niface, m, pin[m], d.skel_of, 0, nullptr, 1.0});
        // products' launch shape: warps per block (token STX_SYM_WARPS,
        // default 4) and warps scheduled per full wave (STX_SYM_OCC percent,
        // default 100): autotuner knobs
        const int wpb = ctx->S.tokens.has("STX_SYM_WARPS") ? ctx->S.tokens.ivalue("STX_SYM_WARPS") : 4;
        const int occ = ctx->S.tokens.has("STX_SYM_OCC") ? ctx->S.tokens.ivalue("STX_SYM_OCC") : 100;
        if (wpb < 1 || wpb > 8) throw StxError(STX_EINVAL, "STX_SYM_WARPS must be in 1..8");
        if (occ < 10 || occ > 800) throw StxError(STX_EINVAL, "STX_SYM_OCC must be in 10..800");
        const int rcap = ctx->S.tokens.has("STX_SYM_REGCAP") ? (ctx->S.tokens.ivalue("STX_SYM_REGCAP") != 0) : 0;
        if (wpb > 4 && !rcap) throw StxError(STX_EINVAL, "STX_SYM_WARPS above 4 needs STX_SYM_REGCAP = 1");
        d.sym_warps = wpb;
        d.sym_regcap = rcap;
        const std::vector<SymWarp> wp = sym_schedule(pp, ctx->device, wpb, occ, rcap),
                                   wi = sym_schedule(pi, ctx->device, wpb, occ, rcap),
                                   wg = sym_schedule(pg, ctx->device, wpb, occ, rcap);
        d.prob_gen = pg.empty() ? nullptr : upload(st->arena, pg);
        d.warp_gen = wg.empty() ? nullptr : upload(st->arena, wg);
        d.nwarp_gen = static_cast<int>(wg.size());
        d.prob_patch = pp.empty() ? nullptr : upload(st->arena, pp);
        d.warp_patch = wp.empty() ? nullptr : upload(st->arena, wp);
        d.nwarp_patch = static_cast<int>(wp.size());
        d.prob_iface = pi.empty() ? nullptr : upload(st->arena, pi);
        d.warp_iface = wi.empty() ? nullptr : upload(st->arena, wi);
        d.nwarp_iface = static_cast<int>(wi.size());
        // mode groups (token STX_MODE_GROUPS, default 2): contiguous modes,
        // their own product schedules over their slice of the problems
        const int ng = std::min(num_modes, std::max(1, ctx->S.tokens.has("STX_MODE_GROUPS")
                                                           ? ctx->S.tokens.ivalue("STX_MODE_GROUPS")
                                                           : 2));
        if (ng > 1 && element_plan(ctx->dg, d, N.nglobal > N.nsolve).ok) {
          size_t ppos = 0, ipos = 0, gpos = 0;
          for (int k = 0; k < ng; ++k) {
            const int m0 = num_modes * k / ng, m1 = num_modes * (k + 1) / ng;
            DevModal v = d;
            v.mode0 = m0;
            v.nmodes = m1 - m0;
            std::vector<SymProblem> gp, gi, gg;
            const size_t p0 = ppos, i0 = ipos, q0 = gpos;
            while (ppos < pp.size() && pp[ppos].mode < m1) gp.push_back(pp[ppos++]);
            while (ipos < pi.size() && pi[ipos].mode < m1) gi.push_back(pi[ipos++]);
            while (gpos < pg.size() && pg[gpos].mode < m1) gg.push_back(pg[gpos++]);
            const std::vector<SymWarp> gwp = sym_schedule(gp, ctx->device, wpb, occ, rcap),
                                       gwi = sym_schedule(gi, ctx->device, wpb, occ, rcap),
                                       gwg = sym_schedule(gg, ctx->device, wpb, occ, rcap);
            v.prob_gen = gg.empty() ? nullptr : d.prob_gen + q0;
            v.warp_gen = gwg.empty() ? nullptr : upload(st->arena, gwg);
            v.nwarp_gen = static_cast<int>(gwg.size());
            v.prob_patch = gp.empty() ? nullptr : d.prob_patch + p0;
            v.warp_patch = gwp.empty() ? nullptr : upload(st->arena, gwp);
            v.nwarp_patch = static_cast<int>(gwp.size());
            v.prob_iface = gi.empty() ? nullptr : d.prob_iface + i0;
            v.warp_iface = gwi.empty() ? nullptr : upload(st->arena, gwi);
            v.nwarp_iface = static_cast<int>(gwi.size());
            st->groups.push_back(v);
          }
        }
        d.fwd = d.bwd = d.dinv_fwd = d.dinv_bwd = nullptr;
        d.nbp = 0;
        d.mode_stride = d.dinv_stride = 0;
        d.status = static_cast<int*>(st->arena.alloc(sizeof(int)));
        cuda_check(cudaMemset(d.status, 0, sizeof(int)), "status");
        d.pc = nullptr;
        d.npts = 0;
        for (auto& v : st->groups) {
          v.status = d.status;
          v.pc = nullptr;
          v.npts = 0;
          v.fwd = v.bwd = v.dinv_fwd = v.dinv_bwd = nullptr;
        }
      } else if (direct) {
        // Device band layout: rows padded to an even stride (16-byte rows for
        // bulk copies), modes 256-byte aligned, plus the inverse of every
        // 16x16 diagonal block of each triangular factor.
        const int nb = N.nband, nbp = (nb + 2) / 2 * 2;  // even, >= nb + 1
        const long long mstride = (static_cast<long long>(nsmax) * nbp + 31) / 32 * 32;
        const int nblk = (nsmax + kBandRows - 1) / kBandRows;
        const long long dstride = static_cast<long long>(std::max(1, nblk)) * kBandRows * kBandRows;
        std::vector<double> hbi, hii;
        std::vector<double> fwd(mstride * num_modes, 0.0), bwd(mstride * num_modes, 0.0);
        std::vector<double> dfw(dstride * num_modes, 0.0), dbw(dstride * num_modes, 0.0);
        for (int m = 0; m < num_modes; ++m) {
          hbi.insert(hbi.end(), modes[m].hbi.begin(), modes[m].hbi.end());
          hii.insert(hii.end(), modes[m].hii.begin(), modes[m].hii.end());
          const int n = modes[m].nsolve;
          // skewed rows: column j-kd+t at position t + ((j-kd) & 1)
          for (int j = 0; j < n; ++j) {
            const int off = (j - (nb - 1)) & 1;
            for (int t = 0; t < nb; ++t) {
              fwd[m * mstride + static_cast<long long>(j) * nbp + t + off] = modes[m].fwd[static_cast<size_t>(j) * nb + t];
              bwd[m * mstride + static_cast<long long>(j) * nbp + t + off] = modes[m].bwd[static_cast<size_t>(j) * nb + t];
            }
          }
          band_block_inverses(modes[m].fwd, n, nb, &dfw[m * dstride]);
          band_block_inverses(modes[m].bwd, n, nb, &dbw[m * dstride]);
          modes[m] = ModeSystem();
        }
        d.nbp = nbp;
        d.mode_stride = mstride;
        d.dinv_stride = dstride;
        d.hbi = upload(st->arena, hbi);
        d.hii = upload(st->arena, hii);
        d.fwd = upload(st->arena, fwd);
        d.bwd = upload(st->arena, bwd);
        d.dinv_fwd = upload(st->arena, dfw);
        d.dinv_bwd = upload(st->arena, dbw);
        d.status = static_cast<int*>(st->arena.alloc(sizeof(int)));
        cuda_check(cudaMemset(d.status, 0, sizeof(int)), "status");
        d.pc = nullptr;
        d.npts = 0;
      } else {
        std::vector<double> pc;
        d.npts = N.nglobal + M.nel * M.nint;
        for (int m = 0; m < num_modes; ++m) pc.insert(pc.end(), modes[m].pc.begin(), modes[m].pc.end());
        d.pc = upload(st->arena, pc);
        d.hbi = d.hii = d.fwd = d.bwd = d.dinv_fwd = d.dinv_bwd = nullptr;
        d.status = nullptr;
      }
      sys->store = st;
    }
    ctx->modals.push_back(sys.get());
    *out = sys.release();
  });
}

int stx_modal_destroy(stx_modal* sys) {
  return guarded([&] {
    if (!sys) return;
    auto& v = sys->ctx->modals;
    for (auto it = v.begin(); it != v.end(); ++it)
      if (*it == sys) {
        v.erase(it);
        break;
      }
    cudaSetDevice(sys->ctx->device);
    cudaStreamSynchronize(sys->ctx->stream);
    delete sys;
  });
}

int stx_modal_info(const stx_modal* sys, int mode, int* nsolve, int* nband) {
  return guarded([&] {
    if (!sys || mode < 0 || mode >= sys->store->dm.nmodes) throw StxError(STX_EINVAL, "bad mode");
    if (nsolve) *nsolve = sys->store->nsolve[mode];
    if (nband) *nband = sys->store->dm.nband;
  });
}

namespace {

// A DIRECT (or MIXED) solve of every plane with the BC values `lines` in
// place of the field's own (same [nz][nline] layout).
void direct_solve_lines(stx_modal* sys, const double* d_forcing, double* d_unknown, const double* lines) {
  stx_context* ctx = sys->ctx;
  FieldDev& F = ctx->fields.at(sys->field);
  double* work = ctx->workspace(helmholtz_workspace_doubles(ctx->dg, F.dn, sys->store->dm));
  const auto& groups = sys->store->groups;
  if (groups.size() > 1) {
    // mode groups on parallel streams, forked from and joined back into
    // the context stream
    ctx->ensure_aux(groups.size() - 1);
    cuda_check(cudaEventRecord(ctx->aux_ev[0], ctx->stream), "fork");
    for (size_t k = 1; k < groups.size(); ++k)
      cuda_check(cudaStreamWaitEvent(ctx->aux[k - 1], ctx->aux_ev[0], 0), "fork wait");
    const bool stag = ctx->stagger();
    if (stag) ctx->ensure_stagger(groups.size());
    for (size_t k = 0; k < groups.size(); ++k) {
      cudaStream_t sk = k ? ctx->aux[k - 1] : ctx->stream;
      if (stag && k) cuda_check(cudaStreamWaitEvent(sk, ctx->stagger_ev[k - 1], 0), "stagger wait");
      cuda_check(helmholtz_direct_solve(ctx->dg, F.dn, groups[k], d_forcing, d_unknown, lines, F.nline, work, sk,
                                        nullptr, stag ? ctx->stagger_ev[k] : nullptr),
                 "direct solve");
    }
    for (size_t k = 1; k < groups.size(); ++k) {
      cuda_check(cudaEventRecord(ctx->aux_ev[k], ctx->aux[k - 1]), "join");
      cuda_check(cudaStreamWaitEvent(ctx->stream, ctx->aux_ev[k], 0), "join wait");
    }
  } else {
    cuda_check(helmholtz_direct_solve(ctx->dg, F.dn, sys->store->dm, d_forcing, d_unknown, lines, F.nline, work,
                                      ctx->stream),
               "direct solve");
  }
}

}  // namespace

}  // extern "C"

namespace stx {

int field_solve_with_lines(stx_modal* sys, const double* d_forcing, double* d_unknown, const double* d_lines) {
  return guarded([&] {
    if (!sys || !d_forcing || !d_unknown || !d_lines) throw StxError(STX_EINVAL, "null argument");
    if (sys->method == STX_JACPCG) throw StxError(STX_EINVAL, "solve with given BC values: DIRECT systems only");
    cudaSetDevice(sys->ctx->device);
    direct_solve_lines(sys, d_forcing, d_unknown, d_lines);
  });
}

}  // namespace stx

extern "C" {

int stx_field_solve(stx_modal* sys, const double* d_forcing, double* d_unknown, double tol_rel,
                    int step_max, int* iterations) {
  return guarded([&] {
    if (!sys || !d_forcing || !d_unknown) throw StxError(STX_EINVAL, "null argument");
    stx_context* ctx = sys->ctx;
    FieldDev& F = ctx->fields.at(sys->field);
    cudaSetDevice(ctx->device);
    if (sys->method != STX_JACPCG) {
      direct_solve_lines(sys, d_forcing, d_unknown, F.d_lines);
    } else {
      double* work = ctx->workspace(jacpcg_workspace_doubles(ctx->dg, F.dn));
      std::vector<int> it(ctx->M.nz, -1);
      cudaError_t e = helmholtz_jacpcg_solve(ctx->dg, F.dn, sys->store->dm, d_forcing, d_unknown,
                                             F.d_lines, F.nline, tol_rel, step_max, work,
                                             it.data(), ctx->stream);
      if (iterations) std::memcpy(iterations, it.data(), sizeof(int) * it.size());
      if (e == cudaErrorNotReady) throw StxError(STX_ENOCONV, "Field::solve: step limit exceeded");
      cuda_check(e, "jacpcg solve");
    }
  });
}

int stx_field_solve_multi(stx_modal* const* systems, int n, const double* const* d_forcing,
                          double* const* d_unknown) {
  return guarded([&] {
    if (!systems || !d_forcing || !d_unknown || n < 1) throw StxError(STX_EINVAL, "bad argument");
    for (int f = 0; f < n; ++f)
      if (!systems[f] || !d_forcing[f] || !d_unknown[f]) throw StxError(STX_EINVAL, "null system or buffer");
    stx_context* ctx = systems[0]->ctx;
    bool shared = n <= 3;
    for (int f = 0; f < n; ++f) {
      if (systems[f]->ctx != ctx) throw StxError(STX_EINVAL, "systems of different contexts");
      if (systems[f]->method == STX_JACPCG) throw StxError(STX_EINVAL, "multi-field solves are DIRECT");
      shared = shared && systems[f]->store == systems[0]->store;
    }
    cudaSetDevice(ctx->device);
    std::vector<const DevNumbering*> N(n);
    std::vector<const double*> lines(n);
    std::vector<int> nline(n);
    for (int f = 0; f < n; ++f) {
      const FieldDev& F = ctx->fields.at(systems[f]->field);
      N[f] = &F.dn;
      lines[f] = F.d_lines;
      nline[f] = F.nline;
    }
    const ModalStore& st = *systems[0]->store;
    if (n == 1 || !shared || !helmholtz_fields_supported(ctx->dg, *N[0], st.dm)) {
      for (int f = 0; f < n; ++f) {
        const int rc = stx_field_solve(systems[f], d_forcing[f], d_unknown[f], 0.0, 0, nullptr);
        if (rc != STX_OK) throw StxError(rc, stx_last_error());
      }
      return;
    }
    double* work = ctx->workspace(helmholtz_fields_workspace_doubles(ctx->dg, *N[0], n));
    const auto& groups = st.groups;
    if (groups.size() > 1) {
      ctx->ensure_aux(groups.size() - 1);
      cuda_check(cudaEventRecord(ctx->aux_ev[0], ctx->stream), "fork");
      for (size_t k = 1; k < groups.size(); ++k)
        cuda_check(cudaStreamWaitEvent(ctx->aux[k - 1], ctx->aux_ev[0], 0), "fork wait");
      const bool stag = ctx->stagger();
      if (stag) ctx->ensure_stagger(groups.size());
      for (size_t k = 0; k < groups.size(); ++k) {
        cudaStream_t sk = k ? ctx->aux[k - 1] : ctx->stream;
        if (stag && k) cuda_check(cudaStreamWaitEvent(sk, ctx->stagger_ev[k - 1], 0), "stagger wait");
        cuda_check(helmholtz_direct_solve_fields(ctx->dg, N.data(), groups[k], d_forcing, d_unknown, lines.data(),
                                                 nline.data(), n, work, sk, stag ? ctx->stagger_ev[k] : nullptr),
                   "multi-field solve");
      }
      for (size_t k = 1; k < groups.size(); ++k) {
        cuda_check(cudaEventRecord(ctx->aux_ev[k], ctx->aux[k - 1]), "join");
        cuda_check(cudaStreamWaitEvent(ctx->stream, ctx->aux_ev[k], 0), "join wait");
      }
    } else {
      cuda_check(helmholtz_direct_solve_fields(ctx->dg, N.data(), st.dm, d_forcing, d_unknown, lines.data(),
                                               nline.data(), n, work, ctx->stream),
                 "multi-field solve");
    }
  });
}

int stx_field_solve_profiled(stx_modal* sys, const double* d_forcing, double* d_unknown,
                             float* phase_ms, int* launches) {
  return guarded([&] {
    if (!sys || !d_forcing || !d_unknown || !phase_ms) throw StxError(STX_EINVAL, "null argument");
    if (sys->method == STX_JACPCG) throw StxError(STX_EINVAL, "profiled solve is for DIRECT systems");
    stx_context* ctx = sys->ctx;
    FieldDev& F = ctx->fields.at(sys->field);
    cudaSetDevice(ctx->device);
    cudaEvent_t ev[5];
    for (auto& e : ev) cuda_check(cudaEventCreate(&e), "event");
    double* work = ctx->workspace(helmholtz_workspace_doubles(ctx->dg, F.dn, sys->store->dm));
    cudaError_t err = helmholtz_direct_solve(ctx->dg, F.dn, sys->store->dm, d_forcing, d_unknown,
                                             F.d_lines, F.nline, work, ctx->stream, ev);
    if (err == cudaSuccess) err = cudaEventSynchronize(ev[4]);
    for (int i = 0; i < 4 && err == cudaSuccess; ++i) err = cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    cuda_check(err, "profiled solve");
    check_sweep_status(sys);
    if (launches) *launches = helmholtz_direct_launches(F.dn, sys->store->dm, ctx->M.np);
  });
}

int stx_modal_status(stx_modal* sys, int* status) {
  return guarded([&] {
    if (!sys || !status) throw StxError(STX_EINVAL, "null argument");
    cudaSetDevice(sys->ctx->device);
    cuda_check(cudaStreamSynchronize(sys->ctx->stream), "sync");
    *status = status_word(sys);
    if (*status == 0 && fft_timeout_flag() > 0) *status = 5;
  });
}

int stx_modal_launches(const stx_modal* sys, int* launches) {
  return guarded([&] {
    if (!sys || !launches) throw StxError(STX_EINVAL, "null argument");
    if (sys->method == STX_JACPCG) throw StxError(STX_EINVAL, "launch count is for DIRECT systems");
    const stx_context* ctx = sys->ctx;
    const auto& groups = sys->store->groups;
    const int per = helmholtz_direct_launches(ctx->fields.at(sys->field).dn, sys->store->dm, ctx->M.np);
    *launches = per * std::max<int>(1, static_cast<int>(groups.size()));
  });
}

int stx_modal_bytes(const stx_modal* sys, double* bytes) {
  return guarded([&] {
    if (!sys || !bytes) throw StxError(STX_EINVAL, "null argument");
    const stx_context* ctx = sys->ctx;
    const Mesh& M = ctx->M;
    const DevModal& d = sys->store->dm;
    const double w = 8.0;
    const int nz = M.nz, nm = d.nmodes;
    const int solved = nz > 1 ? nz - 1 : 1;
    const double field = w * static_cast<double>(M.nplane) * solved;
    const double rhs = w * ctx->fields.at(sys->field).N.nglobal * solved;
    const double fam = w * d.nfamily * nm;
    // element condensation: forcing in, condensation matrix per family and
    // mode, skeleton RHS out; recovery: forcing and skeleton values in,
    // solution out, both condensation matrices
    bytes[0] = field + fam * M.next * M.nint + rhs;
    bytes[3] = 2 * field + fam * (M.next * M.nint + static_cast<double>(M.nint) * M.nint) + rhs;
    if (d.l2) {
      // first half: S_II^-1 products (packed, once per patch family and
      // mode), element Schur complements, interface products (packed);
      // second half: the G = S_II^-1 S_IB products (tiles, once per patch
      // family and mode)
      const Patching* P = ctx->fields.at(sys->field).P.get();
      double pm = 0;
      for (int f = 0; f < P->nfamily; ++f) pm += static_cast<double>(sym_size(P->nI[P->family_rep[f]]));
      const double sc = static_cast<double>(M.nfamily) * M.next * M.next;
      double gm = 0;
      for (int f = 0; f < P->nfamily; ++f) {
        const int rep = P->family_rep[f];
        gm += static_cast<double>(gen_size(P->nI[rep], P->nB[rep]));
      }
      bytes[1] = w * nm * (pm + sc + static_cast<double>(sym_size(d.niface))) + 4 * rhs;
      bytes[2] = w * nm * gm + 2 * rhs;
    } else {
      double band = 0;
      for (int m = 0; m < nm; ++m) band += w * static_cast<double>(sys->store->nsolve[m]) * d.nband;
      bytes[1] = band + rhs;
      bytes[2] = band + rhs;
    }
  });
}

int stx_transform(stx_context* ctx, double* d_data, int sign) {
  return guarded([&] {
    if (!ctx || !d_data) throw StxError(STX_EINVAL, "null argument");
    if (sign != STX_FORWARD && sign != STX_INVERSE) throw StxError(STX_EINVAL, "bad sign");
    cudaSetDevice(ctx->device);
    cuda_check(z_transform(d_data, ctx->M.nz, ctx->M.plane_size, sign, ctx->d_twiddle, nullptr,
                           ctx->stream),
               "transform");
  });
}

int stx_elliptic_solve_host(stx_modal* sys, const double* h_forcing, double* h_solution) {
  return guarded([&] {
    if (!sys || !h_forcing || !h_solution) throw StxError(STX_EINVAL, "null argument");
    stx_context* ctx = sys->ctx;
    const Mesh& M = ctx->M;
    cudaSetDevice(ctx->device);
    const size_t nplane = M.nplane, ps = M.plane_size, nz = M.nz;
    if (!ctx->d_io) {
      ctx->d_io = static_cast<double*>(ctx->arena.alloc(sizeof(double) * 2 * ps * nz));
      cuda_check(cudaMemset(ctx->d_io, 0, sizeof(double) * 2 * ps * nz), "memset io");
    }
    double* dF = ctx->d_io;
    double* dU = ctx->d_io + ps * nz;
    // one copy per direction: host planes are nplane doubles apart, device
    // planes plane_size
    cuda_check(copy_planes(dF, sizeof(double) * ps, h_forcing, sizeof(double) * nplane, sizeof(double) * nplane,
                           nz, cudaMemcpyHostToDevice, ctx->stream),
               "forcing h2d");
    cuda_check(z_transform(dF, M.nz, M.plane_size, STX_FORWARD, ctx->d_twiddle, nullptr, ctx->stream),
               "forward transform");
    if (nz > 1) cuda_check(cudaMemsetAsync(dF + ps, 0, sizeof(double) * ps, ctx->stream), "nyquist");
    // the solve writes every plane but the Nyquist one
    if (nz > 1) cuda_check(cudaMemsetAsync(dU + ps, 0, sizeof(double) * ps, ctx->stream), "zero nyquist");
    const double tol = ctx->S.tokens.value("TOL_REL");
    const int smax = ctx->S.tokens.ivalue("STEP_MAX");
    int rc = stx_field_solve(sys, dF, dU, tol, smax, nullptr);
    if (rc != STX_OK) throw StxError(rc, g_last_error);
    cuda_check(z_transform(dU, M.nz, M.plane_size, STX_INVERSE, ctx->d_twiddle, nullptr, ctx->stream),
               "inverse transform");
    cuda_check(copy_planes(h_solution, sizeof(double) * nplane, dU, sizeof(double) * ps, sizeof(double) * nplane,
                           nz, cudaMemcpyDeviceToHost, ctx->stream),
               "solution d2h");
    // the status words travel with the solution (no extra synchronisation)
    int* fl = ctx->flags();
    fl[0] = fl[1] = 0;
    if (sys->store->dm.status)
      cuda_check(cudaMemcpyAsync(&fl[0], sys->store->dm.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                 "status d2h");
    if (const int* ft = fft_timeout_address())
      cuda_check(cudaMemcpyAsync(&fl[1], ft, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status d2h");
    cuda_check(cudaStreamSynchronize(ctx->stream), "sync");
    if (fl[0]) {
      const char* where = fl[0] == 1 ? "banded sweep" : fl[0] == 3 ? "element kernel" : "packed skeleton product";
      throw StxError(STX_ECUDA, std::string(where) + ": a bounded wait for a bulk copy expired");
    }
    if (fl[1]) throw StxError(STX_ECUDA, "z-FFT: a bounded wait for a bulk copy expired");
  });
}

int stx_elliptic_solve_host_batch(stx_modal* sys, int n, const double* const* h_forcing,
                                  double* const* h_solution) {
  return guarded([&] {
    if (!sys || n < 0 || (n && (!h_forcing || !h_solution))) throw StxError(STX_EINVAL, "bad argument");
    for (int i = 0; i < n; ++i)
      if (!h_forcing[i] || !h_solution[i]) throw StxError(STX_EINVAL, "null host buffer");
    if (n == 0) return;
    stx_context* ctx = sys->ctx;
    const Mesh& M = ctx->M;
    cudaSetDevice(ctx->device);
    const size_t nplane = M.nplane, ps = M.plane_size, nz = M.nz;
    const size_t set = 2 * ps * nz;  // forcing and solution planes of one set
    ctx->ensure_pipeline(set);
    const double tol = ctx->S.tokens.value("TOL_REL");
    const int smax = ctx->S.tokens.ivalue("STEP_MAX");
    for (int i = 0; i < n; ++i) {
      const int b = i % stx_context::kIoSets;
      double* dF = ctx->d_io2 + set * b;
      double* dU = dF + ps * nz;
      // in: set b's forcing is free once solve i - kIoSets has run
      cuda_check(cudaStreamWaitEvent(ctx->s_h2d, ctx->ev_comp[b], 0), "wait");
      cuda_check(copy_planes(dF, sizeof(double) * ps, h_forcing[i], sizeof(double) * nplane,
                             sizeof(double) * nplane, nz, cudaMemcpyHostToDevice, ctx->s_h2d),
                 "forcing h2d");
      cuda_check(cudaEventRecord(ctx->ev_in[b], ctx->s_h2d), "record");
      // solve: after the forcing landed and set b's solution was read out
      cuda_check(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[b], 0), "wait");
      cuda_check(cudaStreamWaitEvent(ctx->stream, ctx->ev_out[b], 0), "wait");
      cuda_check(z_transform(dF, M.nz, M.plane_size, STX_FORWARD, ctx->d_twiddle, nullptr, ctx->stream),
                 "forward transform");
      if (nz > 1) {
        cuda_check(cudaMemsetAsync(dF + ps, 0, sizeof(double) * ps, ctx->stream), "nyquist");
        cuda_check(cudaMemsetAsync(dU + ps, 0, sizeof(double) * ps, ctx->stream), "zero nyquist");
      }
      const int rc = stx_field_solve(sys, dF, dU, tol, smax, nullptr);
      if (rc != STX_OK) throw StxError(rc, g_last_error);
      cuda_check(z_transform(dU, M.nz, M.plane_size, STX_INVERSE, ctx->d_twiddle, nullptr, ctx->stream),
                 "inverse transform");
      cuda_check(cudaEventRecord(ctx->ev_comp[b], ctx->stream), "record");
      // out
      cuda_check(cudaStreamWaitEvent(ctx->s_d2h, ctx->ev_comp[b], 0), "wait");
      cuda_check(copy_planes(h_solution[i], sizeof(double) * nplane, dU, sizeof(double) * ps,
                             sizeof(double) * nplane, nz, cudaMemcpyDeviceToHost, ctx->s_d2h),
                 "solution d2h");
      cuda_check(cudaEventRecord(ctx->ev_out[b], ctx->s_d2h), "record");
    }
    int* fl = ctx->flags();
    fl[0] = fl[1] = 0;
    if (sys->store->dm.status)
      cuda_check(cudaMemcpyAsync(&fl[0], sys->store->dm.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                 "status d2h");
    if (const int* ft = fft_timeout_address())
      cuda_check(cudaMemcpyAsync(&fl[1], ft, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status d2h");
    cuda_check(cudaStreamSynchronize(ctx->stream), "sync");
    cuda_check(cudaStreamSynchronize(ctx->s_d2h), "sync");
    if (fl[0]) {
      const char* where = fl[0] == 1 ? "banded sweep" : fl[0] == 3 ? "element kernel" : "packed skeleton product";
      throw StxError(STX_ECUDA, std::string(where) + ": a bounded wait for a bulk copy expired");
    }
    if (fl[1]) throw StxError(STX_ECUDA, "z-FFT: a bounded wait for a bulk copy expired");
  });
}

int stx_context_stream(const stx_context* ctx, void** stream) {
  return guarded([&] {
    if (!ctx || !stream) throw StxError(STX_EINVAL, "null argument");
    *stream = static_cast<void*>(ctx->stream);
  });
}

int stx_sync(stx_context* ctx) {
  return guarded([&] {
    if (!ctx) throw StxError(STX_EINVAL, "null context");
    cuda_check(cudaStreamSynchronize(ctx->stream), "sync");
  });
}

int stx_context_scratch(stx_context* ctx, unsigned long long bytes, void** d_ptr) {
  return guarded([&] {
    if (!ctx || !d_ptr) throw StxError(STX_EINVAL, "null argument");
    *d_ptr = ctx->scratch(bytes);
  });
}

}  // extern "C"
