// Inline-PTX helpers shared by the kernels: shared-memory addresses,
// mbarriers with bounded waits, bulk (TMA) and 8-byte asynchronous copies
// global -> shared, and the FP64 tensor-core product m8n8k4.
#pragma once

#include <cstdint>

namespace stx {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned),
// completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Programmatic dependent launch (a kernel launched with the programmatic
// stream serialisation attribute may start while the previous kernel of its
// stream finishes): pdl_wait blocks until that kernel has completed and its
// writes are visible (a no-op for a kernel launched without the attribute);
// pdl_trigger lets the next such kernel start launching its blocks.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Default bound of an mbarrier wait, and of every wait that drains copies
// still in flight after an expired one: 2 s of wall time.
constexpr unsigned long long kWaitNs = 2000000000ull;
// Longest sleep of one try_wait (the bound above is checked between them).
constexpr unsigned kWaitHintNs = 100000u;

// Bounded wait (`limit_ns` of wall time) for phase `parity` of an mbarrier;
// false if the bound expired.  limit_ns = 0 probes once without blocking
// (the error path's tests use it: a copy issued just before has not landed).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long limit_ns = kWaitNs) {
  const uint32_t a = smem_u32(bar);
  if (limit_ns == 0) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
  }
  const unsigned long long t0 = global_ns();
  for (;;) {
    // the thread may sleep in try_wait until the phase completes, for at
    // most the hint (ns): waiting warps then take no issue slots and no
    // shared-memory cycles from the warps that compute
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity), "r"(kWaitHintNs)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// 8-byte asynchronous copy global -> shared (both 8-byte aligned); completed
// by cp_async_wait_all().
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Close the group of this thread's cp.async copies issued so far; wait until
// at most one group (the newest) is still in flight.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_group1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Arrive on `bar` once all of this thread's earlier cp.async copies have
// landed (the arrival is not added to the expected count: the barrier's
// initial count must include it).
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// D(8x8) += A(8x4) B(4x8) in FP64.  Lane l = 4 g + t holds A[g][t], B[t][g]
// and D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

}  // namespace stx
