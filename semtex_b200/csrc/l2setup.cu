// Two-level system setup on the device (FP64): the patch and interface
// matrices of every Fourier mode, the part of MatrixSys
// (src/matrix.cpp:132-267) whose cost is cubic.  The host forms only the
// element-level condensation per geometry family (Element::HelmholtzSC,
// src/element.cpp:131-214: matrices of order 4(N_P - 1)); from those, per
// chunk of modes:
//   1. each patch family's matrix is assembled from its elements' Schur
//      complements (patch_assemble) and swept over its interior nodes:
//      -S_II^-1, G = S_II^-1 S_IB and the patch Schur complement T at once;
//   2. S_II^-1 and G are packed into the product kernels' tile layout;
//   3. every patch's T is scattered into its mode's interface matrix, the
//      mixed-BC diagonal and the pin of a singular mode are applied, and the
//      interface matrix is swept whole (minus its inverse), then packed.
// A non-positive pivot anywhere (a system that is not positive definite)
// fails the call as the reference's dpbtrf check does (src/matrix.cpp:254).
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels/sweep.cuh"
#include "kernels/symtile.hpp"
#include "l2setup.hpp"
#include "stx_internal.hpp"

namespace stx {

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("device setup: ") + what + ": " + cudaGetErrorString(e));
}

template <class T>
T* up(DeviceArena& A, const std::vector<T>& v) {
  T* p = static_cast<T*>(A.alloc(sizeof(T) * std::max<size_t>(1, v.size())));
  if (!v.empty()) ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "upload");
  return p;
}

}  // namespace

namespace {

void l2_device_setup(const Mesh& M, const Numbering& N, const Patching& P, const std::vector<double>& hbb,
                     int nmodes, const std::vector<int>& pin, const std::vector<long long>& fam_off,
                     const std::vector<long long>& g_off, const std::vector<long long>& if_off, double* d_pack,
                     cudaStream_t st, size_t budget_bytes) {
  DeviceArena tmp;
  // destroyed before tmp: on any exit no kernel still reads the temporaries
  struct SyncGuard {
    cudaStream_t s;
    ~SyncGuard() { cudaStreamSynchronize(s); }
  } guard{st};
  const int nx = M.next, nf = P.nfamily;
  const size_t hbb_mode = static_cast<size_t>(M.nfamily) * nx * nx;
  if (hbb.size() != hbb_mode * nmodes) throw std::runtime_error("device setup: element matrices of wrong size");
  const double* d_hbb = up(tmp, hbb);
  int* d_status = static_cast<int*>(tmp.alloc(sizeof(int)));
  ck(cudaMemsetAsync(d_status, 0, sizeof(int), st), "status");
  // per patch family: the representative patch's element families, local
  // maps, interior mixed-BC diagonal; sizes
  struct Fam {
    int nI, nB, pI, ld, nelem;
    const int* efam;
    const int* local;
    const double* mixI;
    const long long* off_s;  // [nmodes] offsets of S_II^-1
    const long long* off_g;  // [nmodes] offsets of G
  };
  std::vector<Fam> fam(nf);
  for (int f = 0; f < nf; ++f) {
    const int rep = P.family_rep[f];
    Fam& F = fam[f];
    F.nI = P.nI[rep];
    F.nB = P.nB[rep];
    F.pI = sweep_pad(F.nI);
    F.ld = F.pI + sweep_pad(F.nB);
    F.nelem = static_cast<int>(P.elems[rep].size());
    std::vector<int> ef(F.nelem);
    for (int k = 0; k < F.nelem; ++k) ef[k] = M.family[P.elems[rep][k]];
    F.efam = up(tmp, ef);
    F.local = up(tmp, P.local[rep]);
    F.mixI = nullptr;
    if (!N.mixdiag.empty() && F.nI > 0) {
      std::vector<double> mi(F.nI);
      for (int a = 0; a < F.nI; ++a) mi[a] = N.mixdiag[P.I_gid[static_cast<size_t>(rep) * P.nI_max + a]];
      F.mixI = up(tmp, mi);
    }
    std::vector<long long> os(nmodes), og(nmodes);
    for (int m = 0; m < nmodes; ++m) {
      os[m] = fam_off[static_cast<size_t>(m) * nf + f];
      og[m] = g_off[static_cast<size_t>(m) * nf + f];
    }
    F.off_s = up(tmp, os);
    F.off_g = up(tmp, og);
  }
  const int ni = P.niface, nip = sweep_pad(std::max(ni, 1));
  const double* d_idiag = nullptr;
  if (!N.mixdiag.empty() && ni > 0) {
    std::vector<double> dg(ni);
    for (int q = 0; q < ni; ++q) dg[q] = N.mixdiag[P.skel_of[q]];
    d_idiag = up(tmp, dg);
  }
  const int* d_biid = up(tmp, P.B_iid);
  const int* d_pin = up(tmp, pin);
  const long long* d_ifoff = up(tmp, if_off);
  // modes per chunk within the memory budget
  size_t per_mode = static_cast<size_t>(nip) * nip;
  size_t scratch_mode = sweep_scratch_doubles(nip, 1);
  for (const Fam& F : fam) {
    per_mode += static_cast<size_t>(F.ld) * F.ld;
    scratch_mode = std::max(scratch_mode, sweep_scratch_doubles(F.ld, 1));
  }
  per_mode = (per_mode + scratch_mode) * sizeof(double);
  const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(nmodes, budget_bytes / per_mode)));
  std::vector<double*> buf(nf);
  for (int f = 0; f < nf; ++f)
    buf[f] = static_cast<double*>(tmp.alloc(sizeof(double) * static_cast<size_t>(chunk) * fam[f].ld * fam[f].ld));
  double* AI = static_cast<double*>(tmp.alloc(sizeof(double) * static_cast<size_t>(chunk) * nip * nip));
  double* scratch = static_cast<double*>(tmp.alloc(sizeof(double) * scratch_mode * chunk));
  for (int m0 = 0; m0 < nmodes; m0 += chunk) {
    const int nm = std::min(chunk, nmodes - m0);
    for (int f = 0; f < nf; ++f) {
      const Fam& F = fam[f];
      const long long ls = static_cast<long long>(F.ld) * F.ld;
      ck(cudaMemsetAsync(buf[f], 0, sizeof(double) * ls * nm, st), "memset");
      PatchAssembly pa{d_hbb + hbb_mode * m0, M.nfamily, nx, F.efam, F.local, F.nelem, F.nI, F.nB, F.pI, F.ld,
                       F.mixI};
      ck(patch_assemble(pa, buf[f], ls, nm, st), "patch assembly");
      if (F.nI > 0) {
        ck(sym_sweep(buf[f], F.ld, ls, nm, F.pI, scratch, d_status, st), "patch sweep");
        ck(pack_sym(buf[f], ls, F.ld, F.nI, -1.0, d_pack, F.off_s + m0, nm, st), "pack S_II^-1");
        if (F.nB > 0) ck(pack_gen_t(buf[f], ls, F.ld, F.pI, F.nI, F.nB, d_pack, F.off_g + m0, nm, st), "pack G");
      }
    }
    if (ni > 0) {
      const long long is = static_cast<long long>(nip) * nip;
      ck(cudaMemsetAsync(AI, 0, sizeof(double) * is * nm, st), "memset");
      for (int p = 0; p < P.npatch; ++p) {
        const Fam& F = fam[P.family[p]];
        ck(interface_scatter(buf[P.family[p]], static_cast<long long>(F.ld) * F.ld, F.ld, F.pI, P.nB[p],
                             d_biid + static_cast<size_t>(p) * P.nB_max, AI, is, nip, nm, st),
           "interface scatter");
      }
      ck(interface_finish(AI, is, nip, ni, d_idiag, d_pin + m0, nm, st), "interface finish");
      ck(sym_sweep(AI, nip, is, nm, nip, scratch, d_status, st), "interface sweep");
      ck(pack_sym(AI, is, nip, ni, -1.0, d_pack, d_ifoff + m0, nm, st), "pack interface");
    }
  }
  int status = 0;
  ck(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
  ck(cudaStreamSynchronize(st), "sync");
  if (status) throw std::runtime_error("failed to factor Helmholtz matrix (not positive definite)");
}

}  // namespace

void l2_device_setup_guarded(const Mesh& M, const Numbering& N, const Patching& P, const std::vector<double>& hbb,
                             int nmodes, const std::vector<int>& pin, const std::vector<long long>& fam_off,
                             const std::vector<long long>& g_off, const std::vector<long long>& if_off,
                             double* d_pack, cudaStream_t st, size_t budget_bytes) {
  l2_device_setup(M, N, P, hbb, nmodes, pin, fam_off, g_off, if_off, d_pack, st, budget_bytes);
}

}  // namespace stx
