// One-dimensional bulk copies from global to shared memory (the TMA's untiled
// form, cp.async.bulk), completed through an mbarrier in shared memory. One
// thread issues the copies; every thread of the block waits on the barrier.
// Never with .multicast::cluster: each block copies only into its own shared
// memory. Both addresses must be 16-byte aligned and the size a multiple of 16.
#pragma once

#include <cstdint>

namespace sb {

__device__ __forceinline__ uint32_t smem_address(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialises a barrier that completes when `arrivals` threads have arrived
// and the expected bytes have landed; makes it visible to the copy engine.
__device__ __forceinline__ void bulk_barrier_init(uint64_t *bar, uint32_t arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_address(bar)), "r"(arrivals) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives on the barrier and adds `bytes` to the bytes the phase waits for.
__device__ __forceinline__ void bulk_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_address(bar)), "r"(bytes) : "memory");
}

// Copies `bytes` from global `src` into this block's shared `dst`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_address(dst)),
               "l"(src), "r"(bytes), "r"(smem_address(bar))
               : "memory");
}

__device__ __forceinline__ bool bulk_try_wait(uint64_t *bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_address(bar)), "r"(phase)
      : "memory");
  return done != 0u;
}

// Waits for phase `phase` of the barrier, at most `limit` polls (each poll
// may suspend the thread for a while). Returns false if it gave up.
__device__ __forceinline__ bool bulk_wait(uint64_t *bar, uint32_t phase, int limit) {
  for (int i = 0; i < limit; ++i)
    if (bulk_try_wait(bar, phase)) return true;
  return false;
}

} // namespace sb
