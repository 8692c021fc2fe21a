// Host-side launch helpers shared by the kernel sources.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <mutex>
#include <utility>

namespace stx {

// Raise `kernel`'s dynamic shared-memory limit to at least `bytes` on the
// current device.  The attribute is per device, so it is recorded per
// (kernel, device); thread-safe, and a no-op once the limit is high enough
// (so nothing is set while a stream is being captured after warm-up).
inline void raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[{kernel, dev}];
  if (bytes > have) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    have = bytes;
  }
}

// Launch `kernel` on `st`, with the programmatic stream serialisation
// attribute when `pdl` is set: its blocks may start as soon as every block of
// the previous kernel in the stream has called pdl_trigger (ptx.cuh), and
// everything it reads that earlier work wrote must come after its pdl_wait.
template <class... KArgs, class... Args>
cudaError_t launch_ex(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                      Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace stx
