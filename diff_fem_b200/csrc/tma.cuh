// tma.cuh — bulk asynchronous global -> shared copies (the TMA unit's 1-D
// bulk path, cp.async.bulk) completed on a shared-memory mbarrier.
//
// One elected thread posts the expected byte count and issues the copies;
// every thread then waits on the barrier.  The wait is bounded: after
// kMbarTries polls it gives up and reports failure (the caller records an
// error status and leaves), so a lost completion can never hang the GPU.
// Source and destination must be 16-byte aligned and sizes multiples of 16.
#pragma once
#include <cstdint>

namespace dfem {

constexpr int kMbarTries = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's (and, after a CTA barrier, the CTA's) earlier generic
// accesses to shared memory before later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `phase` of the barrier; false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase) {
  for (int i = 0; i < kMbarTries; ++i)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

}  // namespace dfem
