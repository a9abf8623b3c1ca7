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

// union of the root's valid slots -> 6 floats (lower xyz, upper xyz)
template <int W>
__global__ void k_wide_root_box(const Node *__restrict__ slots, float *__restrict__ box)
{
  griddep_wait();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int c = 0; c < W; c++) {
    const Node sl = ldg_node(slots + c);
    if (!wslot_valid(node_admin(sl))) continue;
    lo[0] = fminf(lo[0], sl.a.x); lo[1] = fminf(lo[1], sl.a.y); lo[2] = fminf(lo[2], sl.a.z);
    hi[0] = fmaxf(hi[0], sl.a.w); hi[1] = fmaxf(hi[1], sl.b.x); hi[2] = fmaxf(hi[2], sl.b.y);
  }
  for (int d = 0; d < 3; d++) {
    box[d] = lo[d];
    box[3 + d] = hi[d];
  }
}

} // namespace bq
