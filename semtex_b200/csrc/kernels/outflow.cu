// Computed outflow BCs on the device (see outflow.cuh).  One block per
// (outflow edge, plane); a thread per edge node.
#include "outflow.cuh"

#include "elemderiv.cuh"

namespace stx {

namespace {

struct Levels {
  const double* p[3];
  double ex[3];
  int n;
};

__global__ void k_outflow_gather(DevGeom g, OutflowEdges E, const double* U, const double* V, const double* W,
                                 double* lv) {
  const int eo = blockIdx.x, k = blockIdx.y, np = g.np;
  const int c = threadIdx.x / np, r = threadIdx.x - c * np;
  if (c >= 3) return;
  const double* src = c == 0 ? U : (c == 1 ? V : W);
  const int e = E.elmt[eo];
  const size_t x = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp + side_node(E.side[eo], r, np);
  lv[(static_cast<size_t>(c) * g.nz + k) * E.ostride + static_cast<size_t>(eo) * np + r] = src ? src[x] : 0.0;
}

__global__ void k_outflow_fourier(DevGeom g, OutflowEdges E, const double* U, const double* V, const double* W,
                                  double nu, double beta, double* divu, double* gradu) {
  extern __shared__ double sm[];
  const int eo = blockIdx.x, k = blockIdx.y, np = g.np, nn = g.npnp, nz = g.nz;
  const size_t out = static_cast<size_t>(k) * E.ostride + static_cast<size_t>(eo) * np;
  if (nz > 1 && k == 1) {  // the Nyquist plane carries no terms
    for (int r = threadIdx.x; r < np; r += blockDim.x) divu[out + r] = gradu[out + r] = 0.0;
    return;
  }
  double* sD = sm;
  double* su = sm + np * np;
  double* sv = su + nn;
  const int e = E.elmt[eo];
  // du/dx, du/dy of the imaginary planes of the higher modes from the
  // highest mode's imaginary plane (src/bcmgr.cpp:1231-1238, as computed)
  const int kx = (k > 1 && (k & 1)) ? nz - 1 : k;
  const size_t bu = static_cast<size_t>(kx) * g.plane_size + static_cast<size_t>(e) * nn;
  const size_t bv = static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * nn;
  for (int q = threadIdx.x; q < np * np; q += blockDim.x) sD[q] = g.D[q];
  for (int q = threadIdx.x; q < nn; q += blockDim.x) {
    su[q] = U[bu + q];
    sv[q] = V[bv + q];
  }
  __syncthreads();
  for (int r = threadIdx.x; r < np; r += blockDim.x) {
    const int t = side_node(E.side[eo], r, np);
    const double nxv = E.nx[eo * np + r], nyv = E.ny[eo * np + r];
    const double ux = elem_deriv(g, su, sD, e, t, 0), uy = elem_deriv(g, su, sD, e, t, 1);
    const double vx = elem_deriv(g, sv, sD, e, t, 0), vy = elem_deriv(g, sv, sD, e, t, 1);
    double dv = ux;
    double gr = (ux * nxv + uy * nyv) * nxv;
    dv += vy;
    gr += (vx * nxv + vy * nyv) * nyv;
    if (W && k >= 2) {  // Fourier z-derivative of w: -beta m w_Im (real plane), +beta m w_Re
      const double bk = (k >> 1) * beta;
      const int kz = (k & 1) ? k - 1 : k + 1;
      const double wz = W[static_cast<size_t>(kz) * g.plane_size + static_cast<size_t>(e) * nn + t];
      dv += ((k & 1) ? bk : -bk) * wz;
    }
    divu[out + r] = nu * dv;
    gradu[out + r] = nu * gr;
  }
}

__global__ void k_outflow_energy(DevGeom g, OutflowEdges E, Levels L, double iuzd, double* fb) {
  const int eo = blockIdx.x, k = blockIdx.y, np = g.np, nz = g.nz;
  const int r = threadIdx.x;
  if (r >= np) return;
  const size_t o = static_cast<size_t>(eo) * np + r;
  double u = 0.0, v = 0.0, w = 0.0;
  for (int q = 0; q < L.n; ++q) {
    u += L.ex[q] * L.p[q][(0 * static_cast<size_t>(nz) + k) * E.ostride + o];
    v += L.ex[q] * L.p[q][(1 * static_cast<size_t>(nz) + k) * E.ostride + o];
    w += L.ex[q] * L.p[q][(2 * static_cast<size_t>(nz) + k) * E.ostride + o];
  }
  const double unp = E.nx[o] * u + E.ny[o] * v;
  const double ke = 0.5 * (w * w + (v * v + u * u));
  const double s0 = 0.5 * (1.0 - tanh(unp * iuzd));
  fb[static_cast<size_t>(k) * E.ostride + o] = ke * s0;
}

__global__ void k_outflow_plines(DevGeom g, OutflowEdges E, Levels L, const double* fb, double* lines, int nline) {
  const int eo = blockIdx.x, k = blockIdx.y, np = g.np;
  const int r = threadIdx.x;
  if (r >= np) return;
  const size_t o = static_cast<size_t>(k) * E.ostride + static_cast<size_t>(eo) * np + r;
  double v = 0.0;
  if (!(g.nz > 1 && k == 1)) {
    double s = 0.0;
    for (int q = 0; q < L.n; ++q) s += L.ex[q] * L.p[q][o];
    v = s - fb[o];
  }
  lines[static_cast<size_t>(k) * nline + static_cast<size_t>(E.line[eo]) * np + r] = v;
}

__global__ void k_outflow_ulines(DevGeom g, OutflowEdges E, Levels L, const double* fb, const double* p, double nu,
                                 int dir, double* lines, int nline) {
  const int eo = blockIdx.x, k = blockIdx.y, np = g.np;
  const int r = threadIdx.x;
  if (r >= np) return;
  const size_t o = static_cast<size_t>(k) * E.ostride + static_cast<size_t>(eo) * np + r;
  double v = 0.0;
  if (!(g.nz > 1 && k == 1)) {
    const int e = E.elmt[eo];
    const double pe =
        p[static_cast<size_t>(k) * g.plane_size + static_cast<size_t>(e) * g.npnp + side_node(E.side[eo], r, np)];
    double work = 0.0;
    for (int q = 0; q < L.n; ++q) work += L.ex[q] * L.p[q][o];
    const double nrm = dir ? E.ny[eo * np + r] : E.nx[eo * np + r];
    v = ((1.0 / nu) * fb[o] + (pe - work)) * nrm;
  }
  lines[static_cast<size_t>(k) * nline + static_cast<size_t>(E.line[eo]) * np + r] = v;
}

Levels levels(const double* const* p, const double* ex, int n) {
  Levels L{};
  L.n = n;
  for (int q = 0; q < n && q < 3; ++q) {
    L.p[q] = p[q];
    L.ex[q] = ex[q];
  }
  return L;
}

}  // namespace

cudaError_t outflow_gather(const DevGeom& g, const OutflowEdges& E, const double* U, const double* V,
                           const double* W, double* lv, cudaStream_t st) {
  if (E.no <= 0) return cudaSuccess;
  k_outflow_gather<<<dim3(E.no, g.nz), 3 * g.np, 0, st>>>(g, E, U, V, W, lv);
  return cudaGetLastError();
}

cudaError_t outflow_fourier(const DevGeom& g, const OutflowEdges& E, const double* U, const double* V,
                            const double* W, double nu, double beta, double* divu, double* gradu, cudaStream_t st) {
  if (E.no <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * (static_cast<size_t>(g.np) * g.np + 2 * static_cast<size_t>(g.npnp));
  k_outflow_fourier<<<dim3(E.no, g.nz), 64, smem, st>>>(g, E, U, V, W, nu, beta, divu, gradu);
  return cudaGetLastError();
}

cudaError_t outflow_energy(const DevGeom& g, const OutflowEdges& E, const double* const* lv, const double* ex,
                           int Jx, double iuzd, double* fb, cudaStream_t st) {
  if (E.no <= 0) return cudaSuccess;
  k_outflow_energy<<<dim3(E.no, g.nz), 32 * ((g.np + 31) / 32), 0, st>>>(g, E, levels(lv, ex, Jx), iuzd, fb);
  return cudaGetLastError();
}

cudaError_t outflow_plines(const DevGeom& g, const OutflowEdges& E, const double* const* gradu, const double* ex,
                           int Jx, const double* fb, double* lines, int nline, cudaStream_t st) {
  if (E.no <= 0) return cudaSuccess;
  k_outflow_plines<<<dim3(E.no, g.nz), 32 * ((g.np + 31) / 32), 0, st>>>(g, E, levels(gradu, ex, Jx), fb, lines,
                                                                         nline);
  return cudaGetLastError();
}

cudaError_t outflow_ulines(const DevGeom& g, const OutflowEdges& E, const double* const* divu, const double* ex,
                           int Jx, const double* fb, const double* p, double nu, int dir, double* lines, int nline,
                           cudaStream_t st) {
  if (E.no <= 0) return cudaSuccess;
  k_outflow_ulines<<<dim3(E.no, g.nz), 32 * ((g.np + 31) / 32), 0, st>>>(g, E, levels(divu, ex, Jx), fb, p, nu,
                                                                         dir, lines, nline);
  return cudaGetLastError();
}

}  // namespace stx
