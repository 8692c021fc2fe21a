// Direct Helmholtz solve that allocates no device memory.
//
// stx_field_solve needs scratch for the boundary right-hand sides and the
// essential values of every plane and grows it with cudaMalloc on first use.
// Some callers cannot allow that: a host that has handed all device memory to
// its own allocator and forbids libraries from allocating after start-up, or
// a time-stepping loop that cannot afford the device-wide synchronisation
// cudaMalloc/cudaFree may imply.  For them this file provides
// stx_field_solve_noalloc, which runs the same kernels with the scratch placed
// in a fixed file-scope device array instead.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/semtex_b200.h"
#include "kernels/helmholtz.cuh"
#include "stx_internal.hpp"

namespace {

// Upper bound of the scratch a call may use: 2^20 doubles (8 MiB).  CUDA loads
// this file's device code lazily, so a GPU maps the array at the first call
// made on it (which may allocate and synchronise like any module load: make
// it at start-up) and holds it until the process exits.
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 20;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch per device.  In host code the array's
// name is only a host-side stand-in, so the address must come from
// cudaGetSymbolAddress, called with the device current.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
  stx::set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int stx_field_solve_noalloc(stx_modal* sys, const double* d_forcing, double* d_unknown) {
  if (!sys || !d_forcing || !d_unknown) return fail(STX_EINVAL, "null argument");
  if (sys->method != STX_DIRECT) return fail(STX_EINVAL, "stx_field_solve_noalloc needs a DIRECT system");
  stx_context* ctx = sys->ctx;
  const auto it = ctx->fields.find(sys->field);
  if (it == ctx->fields.end()) return fail(STX_EINVAL, "field not in context");
  const stx::FieldDev& F = it->second;
  const size_t need = stx::helmholtz_workspace_doubles(ctx->dg, F.dn, sys->store->dm);
  if (need > kNoAllocScratchDoubles) {
    return fail(STX_EINVAL, "stx_field_solve_noalloc: this problem needs " + std::to_string(need) +
                                " doubles of scratch, more than the static maximum of " +
                                std::to_string(kNoAllocScratchDoubles));
  }
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(STX_EINVAL, "device index out of range");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return fail(STX_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[ctx->device]) {
      // One-time set-up on this device, with the device current.
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(STX_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[ctx->device] = static_cast<double*>(p);
    }
    scratch = g_addr[ctx->device];
  }
  // helmholtz_direct_solve zeroes the part of the scratch it accumulates into
  // (cudaMemsetAsync on the context stream) before its first kernel.
  e = stx::helmholtz_direct_solve(ctx->dg, F.dn, sys->store->dm, d_forcing, d_unknown, F.d_lines, F.nline,
                                  scratch, ctx->stream);
  if (e != cudaSuccess) return fail(STX_ECUDA, std::string("direct solve: ") + cudaGetErrorString(e));
  stx::set_last_error("");
  return STX_OK;
}
