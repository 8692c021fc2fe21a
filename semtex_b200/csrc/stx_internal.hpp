// Internal definitions of the opaque C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host/mesh.hpp"
#include "host/patch.hpp"
#include "host/session.hpp"
#include "kernels/device.hpp"
#include "kernels/symtile.hpp"

namespace stx {

// Device allocations freed together.
struct DeviceArena {
  std::vector<void*> ptrs;
  void* alloc(size_t bytes);
  DeviceArena() = default;
  DeviceArena(const DeviceArena&) = delete;
  DeviceArena& operator=(const DeviceArena&) = delete;
  ~DeviceArena();
};

struct FieldDev {
  Numbering N;
  std::unique_ptr<Patching> P;  // two-level condensation, built on first DIRECT system
  bool patch_done = false;
  DevNumbering dn{};
  double* d_lines = nullptr;  // [nz][nline] Fourier-space BC values
  int nline = 0;
};

struct ModalStore {
  DeviceArena arena;
  DevModal dm{};
  std::vector<int> nsolve;
  // Two-level DIRECT systems: views of dm over contiguous mode groups, each
  // with its own product schedules.  The groups of a solve run on parallel
  // streams (the modes are independent), so the phases of one group overlap
  // those of another.
  std::vector<DevModal> groups;
};

void host_dft_forward(std::vector<double>& a, int nz, int n);

// Message returned by stx_last_error() on this thread.
void set_last_error(const std::string& msg);

}  // namespace stx

struct stx_modal;

struct stx_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  stx::Session S;
  stx::Mesh M;
  std::map<char, stx::FieldDev> fields;
  stx::DeviceArena arena;
  stx::DevGeom dg{};
  std::vector<int> elem_sorted;  // host copy of dg.elem_sorted
  double* d_twiddle = nullptr;
  double* d_io = nullptr;
  std::vector<stx_modal*> modals;

  // Patching of a field's numbering for the two-level direct solve, or null
  // when the single banded factor is used (token STX_TWOLEVEL = 0, element
  // boundaries of more than 64 nodes, or an interface too large for a dense
  // inverse).  The patch size is the one of {8, 16, 36, 64} elements that
  // minimises the matrix bytes read per mode (the interface inverse and,
  // per patch family, S_II^-1 and G = S_II^-1 S_IB once each).
  const stx::Patching* patching(char field) {
    stx::FieldDev& F = fields.at(field);
    if (!F.patch_done) {
      F.patch_done = true;
      const bool want = (!S.tokens.has("STX_TWOLEVEL") || S.tokens.ivalue("STX_TWOLEVEL") != 0) && M.next <= 64;
      // token STX_PATCH_CAP (8, 16, 36 or 64) fixes the patch size (the
      // autotuner's choice) instead of the byte model
      const int fixed = S.tokens.has("STX_PATCH_CAP") ? S.tokens.ivalue("STX_PATCH_CAP") : 0;
      if (fixed && fixed != 8 && fixed != 16 && fixed != 36 && fixed != 64)
        throw std::runtime_error("STX_PATCH_CAP must be 8, 16, 36 or 64");
      if (want) {
        double best = 0;
        for (int cap : {8, 16, 36, 64}) {
          if (fixed && cap != fixed) continue;
          auto P = std::make_unique<stx::Patching>(stx::build_patching(M, F.N, cap));
          if (P->niface > 6000) continue;
          double bytes = static_cast<double>(stx::sym_size(P->niface));
          for (int f = 0; f < P->nfamily; ++f) {
            const int rep = P->family_rep[f];
            bytes += static_cast<double>(stx::sym_size(P->nI[rep]) + stx::gen_size(P->nI[rep], P->nB[rep]));
          }
          if (!F.P || bytes < best) {
            best = bytes;
            F.P = std::move(P);
          }
        }
      }
    }
    return F.P.get();
  }

  // Solver workspace, grown on demand (synchronises before regrowing).
  double* d_work = nullptr;
  size_t work_doubles = 0;
  double* workspace(size_t n) {
    if (n > work_doubles) {
      cudaStreamSynchronize(stream);
      if (d_work) cudaFree(d_work);
      d_work = nullptr;
      if (cudaMalloc(&d_work, sizeof(double) * n) != cudaSuccess)
        throw std::runtime_error("cudaMalloc of solver workspace failed");
      work_doubles = n;
    }
    return d_work;
  }
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  void* scratch(size_t n) {
    if (n > scratch_bytes) {
      cudaStreamSynchronize(stream);
      if (d_scratch) cudaFree(d_scratch);
      d_scratch = nullptr;
      if (cudaMalloc(&d_scratch, n) != cudaSuccess)
        throw std::runtime_error("cudaMalloc of scratch failed");
      scratch_bytes = n;
    }
    return d_scratch;
  }
  // Streams of mode groups 1.. (group 0 runs on `stream`) and the events
  // that fork them from `stream` and join them back.
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> aux_ev;  // [0] fork, [i] join of aux[i - 1]
  // [k]: mode group k has finished its element condensation; with token
  // STX_STAGGER = 1 group k + 1 starts after it, so that one group's element
  // phase meets the other's skeleton products (a tuning knob: on c2 the
  // groups started together measured faster, 0.175 against 0.196 ms)
  std::vector<cudaEvent_t> stagger_ev;
  bool stagger() const { return S.tokens.has("STX_STAGGER") && S.tokens.ivalue("STX_STAGGER") != 0; }
  void ensure_stagger(size_t n) {
    while (stagger_ev.size() < n) {
      cudaEvent_t e;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        throw std::runtime_error("event creation failed");
      stagger_ev.push_back(e);
    }
  }
  void ensure_aux(size_t n) {
    if (aux_ev.empty()) {
      aux_ev.resize(1);
      if (cudaEventCreateWithFlags(&aux_ev[0], cudaEventDisableTiming) != cudaSuccess)
        throw std::runtime_error("event creation failed");
    }
    while (aux.size() < n) {
      cudaStream_t s;
      cudaEvent_t e;
      if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        throw std::runtime_error("stream creation failed");
      aux.push_back(s);
      aux_ev.push_back(e);
    }
  }
  // Pipelined host-buffer solves: kIoSets sets of device forcing / solution
  // planes (a third set, so that the copy in of solve i + 1, solve i and the
  // copy out of solve i - 1 never share one, measured no faster: the two
  // PCIe directions bound the pipeline), the copy streams (host -> device,
  // device -> host) and the events that hand a set from stage to stage.
  static constexpr int kIoSets = 2;
  double* d_io2 = nullptr;  // [kIoSets][2][nz][plane_size]
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t ev_in[kIoSets] = {}, ev_comp[kIoSets] = {}, ev_out[kIoSets] = {};
  void ensure_pipeline(size_t doubles_per_set) {
    if (!d_io2) {
      d_io2 = static_cast<double*>(arena.alloc(sizeof(double) * kIoSets * doubles_per_set));
      if (cudaMemset(d_io2, 0, sizeof(double) * kIoSets * doubles_per_set) != cudaSuccess)
        throw std::runtime_error("memset of the pipeline buffers failed");
    }
    if (!s_h2d) {
      if (cudaStreamCreateWithFlags(&s_h2d, cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&s_d2h, cudaStreamNonBlocking) != cudaSuccess)
        throw std::runtime_error("stream creation failed");
      for (int b = 0; b < kIoSets; ++b)
        if (cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_comp[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming) != cudaSuccess)
          throw std::runtime_error("event creation failed");
    }
  }
  // Pinned host words the status flags of a synchronising call are copied
  // into on the stream (no extra synchronisation): [0] system, [1] z-FFT.
  int* h_flags = nullptr;
  int* flags() {
    if (!h_flags && cudaMallocHost(&h_flags, 2 * sizeof(int)) != cudaSuccess)
      throw std::runtime_error("cudaMallocHost of the status words failed");
    return h_flags;
  }
  ~stx_context() {
    for (auto s : aux) cudaStreamDestroy(s);
    for (auto e : aux_ev) cudaEventDestroy(e);
    for (auto e : stagger_ev) cudaEventDestroy(e);
    if (s_h2d) cudaStreamDestroy(s_h2d);
    if (s_d2h) cudaStreamDestroy(s_d2h);
    for (int b = 0; b < kIoSets; ++b)
      for (cudaEvent_t e : {ev_in[b], ev_comp[b], ev_out[b]})
        if (e) cudaEventDestroy(e);
    if (d_work) cudaFree(d_work);
    if (d_scratch) cudaFree(d_scratch);
    if (h_flags) cudaFreeHost(h_flags);
  }
};

struct stx_modal {
  stx_context* ctx = nullptr;
  char field = 0;
  int method = 0;
  double lambda2 = 0, beta = 0;
  std::shared_ptr<stx::ModalStore> store;
};

namespace stx {

// Field::solve DIRECT (or MIXED) over every plane, with the Fourier BC
// values `d_lines` ([nz][nline] of the field) in place of the field's own;
// asynchronous on the context stream.  Returns an STX_* status.
int field_solve_with_lines(stx_modal* sys, const double* d_forcing, double* d_unknown, const double* d_lines);

}  // namespace stx
