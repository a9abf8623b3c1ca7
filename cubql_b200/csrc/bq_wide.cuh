// bq_wide.cuh -- slot layout of WideBVH<float,3,W> (cuBQL/bvh.h:113-141).
//
// A wide node is W consecutive 32-byte slots.  A slot is laid out like a
// binary Node (box in the first 24 bytes), its 64-bit word being the
// reference's Child bit field: bit 0 valid, bits 1..45 offset, bits
// 46..61 count.  So one slot is one ldg_node() (two 16-byte loads).
#pragma once

#include "bq_internal.cuh"

namespace bq {

constexpr uint64_t WSLOT_OFFSET_MASK = (1ull << 45) - 1;

__host__ __device__ __forceinline__ uint64_t make_wslot(uint64_t offset, uint32_t count)
{
  return 1ull | ((offset & WSLOT_OFFSET_MASK) << 1) | ((uint64_t)(count & 0xFFFFu) << 46);
}
// unused slot as the reference writes it (wide_gpu_builder.h:150-160):
// valid 0, offset (uint32_t)-1, count (uint32_t)-1 truncated to 16 bits
constexpr uint64_t WSLOT_UNUSED = (0xFFFFFFFFull << 1) | (0xFFFFull << 46);

__device__ __forceinline__ bool wslot_valid(uint64_t w) { return (w & 1ull) != 0; }
__device__ __forceinline__ uint64_t wslot_offset(uint64_t w) { return (w >> 1) & WSLOT_OFFSET_MASK; }
__device__ __forceinline__ uint32_t wslot_count(uint64_t w) { return (uint32_t)(w >> 46) & 0xFFFFu; }

template <int W>
struct WideLog;
template <>
struct WideLog<2> { enum { value = 1 }; };
template <>
struct WideLog<4> { enum { value = 2 }; };
template <>
struct WideLog<8> { enum { value = 3 }; };

} // namespace bq
