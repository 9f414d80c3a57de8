// pipeline.cuh -- mbarrier and bulk-copy (TMA) primitives for the streamed
// fused kernel, as inline PTX for sm_100a.  Every wait is bounded: it gives up
// after `kSpinLimit` polls and reports failure instead of hanging the GPU.
#pragma once

#include <cstdint>

namespace micmb
{
  constexpr uint32_t kSpinLimit = 1u << 22;  // polls (~100 ns apart once backing off) before a timeout

  __device__ __forceinline__ uint32_t smem_addr(const void* p)
  {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
  }

  __device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  }

  // make barrier initialisation visible to the async (bulk-copy) proxy
  __device__ __forceinline__ void fence_barrier_init()
  {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }

  __device__ __forceinline__ void mbar_arrive(uint64_t* bar)
  {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
  }

  __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
  {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
  }

  // non-blocking poll: has the phase with this parity completed?
  __device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity)
  {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
  }

  // bounded wait for the phase with the given parity (well under a second);
  // false on timeout
  __device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
  {
    for (uint32_t i = 0; i < kSpinLimit; ++i)
    {
      if (mbar_test_wait(bar, parity))
        return true;
      if (i > 64)
        __nanosleep(64);
    }
    return false;
  }

  // global -> shared bulk copy completing `bytes` on `bar`; 16-byte aligned, size % 16 == 0
  __device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
  {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
  }

  // named barrier over `threads` threads (multiple of 32)
  __device__ __forceinline__ void named_barrier(uint32_t id, uint32_t threads)
  {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
  }
}  // namespace micmb
