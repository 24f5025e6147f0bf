// Shared-memory barriers (mbarrier) for sm_100a, as inline PTX.  Every wait
// is bounded: it gives up after a limit of wall time (globaltimer), so that a
// copy that never lands ends in an error status, not a hung kernel.
#pragma once
#include <stdint.h>

namespace devsync {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
// Arrive once and expect `bytes` of copies to complete on the barrier.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// The same test, letting the hardware suspend the thread until the phase
// completes or about `hint_ns` have passed, so that a waiting warp does not
// take issue slots from the warps it shares a scheduler with.
__device__ __forceinline__ bool mbar_try_suspend(uint64_t* b, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity; false after `limit_ns` of wall
// time without completion (checked every 16 suspended tests of at most 10 us).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(b, parity)) return true;
  const uint64_t t0 = gtimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_suspend(b, parity, 10000u)) return true;
    if ((i & 15u) == 0 && gtimer() - t0 > limit_ns) return false;
  }
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
}  // namespace devsync
