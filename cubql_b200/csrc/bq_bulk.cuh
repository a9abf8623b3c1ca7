// bq_bulk.cuh -- 1D bulk asynchronous copies from global to this CTA's own
// shared memory (cp.async.bulk, completion counted on an mbarrier), for
// kernels that stream a contiguous array tile by tile.  No multicast: each
// CTA copies only into its own shared memory, from this GPU's memory.
//
// Rules the callers keep: source and destination 16-byte aligned, size a
// multiple of 16 bytes; one thread initialises the barriers and issues the
// copies; every wait is bounded (bulk_wait returns false after `limit`
// polls, and the caller then records an error, waits again -- bounded -- for
// the copies it issued, and returns).
#pragma once

#include <stdint.h>

namespace bq {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// one arrival expected per phase (the issuing thread's expect_tx)
__device__ __forceinline__ void bulk_bar_init(uint64_t *bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// makes the barrier initialisation visible to the asynchronous copies
__device__ __forceinline__ void bulk_bar_init_fence()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders this thread's earlier shared-memory accesses (after a barrier with
// the other threads, theirs too) before later asynchronous copies into it
__device__ __forceinline__ void bulk_proxy_fence()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// copies `bytes` from global `src` into shared `dst`; completion is counted on
// `bar`, whose current phase then completes
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool bulk_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// waits for the phase with this parity to complete; false after `limit` polls
__device__ __forceinline__ bool bulk_wait(uint64_t *bar, uint32_t parity, uint32_t limit)
{
  for (uint32_t i = 0; i < limit; i++)
    if (bulk_try_wait(bar, parity)) return true;
  return false;
}

} // namespace bq
