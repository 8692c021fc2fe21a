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

}  // namespace stx
