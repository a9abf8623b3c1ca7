// bq_agglom.cuh -- bottom-up construction of a radix tree and its boxes.
//
// Input: sorted prims (ids), and for every adjacent pair (i, i+1) a split
// level delta[i] (bq_morton.cu explains why the tree built from these
// levels is the reference radixBuilder's tree).  A node covering sorted
// positions [l, r] is the child of the split at whichever of its two
// boundaries carries the lower level; its box is the union of its
// children's.  Children of split s are stored at nodes[2s], nodes[2s+1]
// (relative to the node block of the prim range), the root at the block's
// first node, the block's second node unused.
//
// Two kernels:
//   k_agg_local   one CTA per chunk of AGG_CHUNK (128) sorted prims, whose
//                 split levels are staged in shared memory.  Threads
//                 start at their leaf and climb; the first child to reach
//                 a split parks its range end and box in shared memory and
//                 stops, the second merges and climbs on.  Everything
//                 below the chunk's boundaries is finished here with
//                 block-scope synchronisation only.  A node whose parent
//                 split lies on a chunk boundary is handed to the global
//                 phase (at most two per chunk); children parked at a split
//                 whose sibling reaches outside the chunk are published to
//                 the global slot array.
//   k_agg_global  one thread per handed-over node continues the climb with
//                 device-scope acquire/release exchanges on global slots.
// With SEG, the prims form independent ranges (clouds) [b0, e0); each
// climb ends at its range's root and never crosses into a neighbour.
#pragma once

#include <cuda/atomic>

#include "bq_internal.cuh"

namespace bq {

// first index of the run of key a ending at or after position i (keys[i] == a),
// not before lo: galloping search (runs are short), then binary search
__device__ __forceinline__ uint32_t run_begin(const uint64_t *__restrict__ keys, uint32_t lo, uint32_t i, uint64_t a)
{
  uint32_t step = 1, hi = i;  // keys[hi] == a
  while (hi > lo) {
    const uint32_t probe = hi - min(step, hi - lo);
    if (keys[probe] != a) { lo = probe + 1; break; }
    hi = probe;
    step <<= 1;
  }
  while (lo < hi) {  // first index in [lo, hi] with key == a
    const uint32_t m = lo + ((hi - lo) >> 1);
    if (keys[m] < a) lo = m + 1; else hi = m;
  }
  return lo;
}

// one past the last index of the run of key a (keys[i] == a), at most hi
__device__ __forceinline__ uint32_t run_end(const uint64_t *__restrict__ keys, uint32_t i, uint32_t hi, uint64_t a)
{
  uint32_t step = 1, lo = i + 1;  // keys[lo-1] == a
  while (lo < hi) {
    const uint32_t probe = lo - 1 + min(step, hi - lo + 1);
    if (probe >= hi || keys[probe] != a) { hi = min(probe, hi); break; }
    lo = probe + 1;
    step <<= 1;
  }
  while (lo < hi) {  // first index in [lo, hi) with key > a
    const uint32_t m = lo + ((hi - lo) >> 1);
    if (keys[m] <= a) lo = m + 1; else hi = m;
  }
  return lo;
}

constexpr int AGG_CHUNK = 128;  // prims per CTA of the local phase
constexpr uint32_t AGG_EMPTY = 0xffffffffu;

// prim range of position i: [0, nv) or the cloud containing i
template <bool SEG>
__device__ __forceinline__ void agg_range(uint32_t i, uint32_t nv, const uint32_t *__restrict__ off, uint32_t numSegs,
                                          uint32_t &b0, uint32_t &e0)
{
  if (!SEG) {
    b0 = 0;
    e0 = nv;
    return;
  }
  uint32_t lo = 0, hi = numSegs;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (__ldg(off + m) <= i) lo = m; else hi = m;
  }
  b0 = __ldg(off + lo);
  e0 = __ldg(off + lo + 1);
}

struct AggBox {
  float lx, ly, lz, hx, hy, hz;
};

__device__ __forceinline__ AggBox agg_union(const AggBox &left, const AggBox &right)
{
  // min(l,r) / max(l,r) in the reference's operand order (sm_builder.h:669-670)
  return AggBox{fminf(left.lx, right.lx), fminf(left.ly, right.ly), fminf(left.lz, right.lz),
                fmaxf(left.hx, right.hx), fmaxf(left.hy, right.hy), fmaxf(left.hz, right.hz)};
}

template <typename LevT>
struct AggArgsT {
  const LevT *delta;      // split level of pair (i, i+1)
  uint32_t *slot;         // global slots (one per split position), set by the local phase
  const uint32_t *ids;    // sorted prim ids (global indices)
  const bq_box3f *boxes;
  Node *nodes;            // output (full tree layout)
  uint32_t *primIDsOut;   // SEG: cloud-local prim ids are written here
  const uint32_t *nvPtr;  // number of sorted prims
  uint2 *ranges;          // optional: [l, r] of every split's node
  uint2 *pending;         // 2 per chunk: nodes handed to the global phase
  const uint32_t *off;    // SEG: cloud offsets
  uint32_t numSegs;
};
using AggArgs = AggArgsT<uint8_t>;

template <bool SEG, typename LevT>
__global__ void __launch_bounds__(AGG_CHUNK) k_agg_local(AggArgsT<LevT> a)
{
  griddep_wait();
  __shared__ uint32_t sSlot[AGG_CHUNK + 1];
  __shared__ float4 sBox[AGG_CHUNK + 1][2][2];  // a box as two 16-byte words: lx ly lz hx | hy hz - -
  __shared__ LevT sLev[AGG_CHUNK + 2];  // delta[c0 - 1 .. c0 + AGG_CHUNK]
  const uint32_t nv = *a.nvPtr;
  const uint32_t c0 = blockIdx.x * AGG_CHUNK;
  if (c0 >= nv) return;  // whole CTA: no barrier below is skipped by part of it
  const uint32_t cEnd = c0 + AGG_CHUNK;  // first split position outside the chunk
  // this thread's prim id and its box (a random gather) first, so that their
  // latency overlaps the staging of the chunk's levels below
  const uint32_t i = c0 + threadIdx.x;
  uint32_t id = 0;
  float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0;
  // the ids are read once and the nodes written once: evict_first in L2, so
  // that the boxes (gathered at random, 2-3 to a 64-byte line) stay longer
  const uint64_t once = l2_policy_evict_first();
  if (i < nv) {
    id = ldg_u32_policy(a.ids + i, once);
    const float2 *bp = reinterpret_cast<const float2 *>(a.boxes + id);
    p0 = __ldg(bp);
    p1 = __ldg(bp + 1);
    p2 = __ldg(bp + 2);
  }
  for (int j = threadIdx.x; j <= AGG_CHUNK; j += blockDim.x) sSlot[j] = AGG_EMPTY;
  for (int j = threadIdx.x; j < AGG_CHUNK + 2; j += blockDim.x) {
    const int64_t g = (int64_t)c0 - 1 + j;  // pairs (g, g+1) exist for 0 <= g < nv - 1
    sLev[j] = (g >= 0 && g + 1 < (int64_t)nv) ? __ldg(a.delta + g) : (LevT)0;
  }
  if (threadIdx.x < 2) a.pending[2 * blockIdx.x + threadIdx.x] = make_uint2(AGG_EMPTY, AGG_EMPTY);
  __syncthreads();
  if (i < nv) {
    uint32_t b0, e0;
    agg_range<SEG>(i, nv, a.off, a.numSegs, b0, e0);
    const uint64_t nodeBase = SEG ? 2ull * b0 : 0ull;
    if (SEG) a.primIDsOut[i] = id - b0;
    if (i == b0) a.nodes[nodeBase + 1] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0);
    AggBox box{p0.x, p0.y, p1.x, p1.y, p2.x, p2.y};
    uint32_t l = i, r = i;
    uint64_t admin = make_admin(i - b0, 1);
    while (true) {
      if (l == b0 && r == e0 - 1) {  // root of the whole range
        st_node_policy(a.nodes + nodeBase, make_node(box.lx, box.ly, box.lz, box.hx, box.hy, box.hz, admin), once);
        break;
      }
      // c0 <= l <= r < cEnd here: delta[l - 1] and delta[r] are in sLev
      const bool leftChild = (l == b0) ? true : (r == e0 - 1) ? false : (sLev[l - c0] > sLev[r - c0 + 1]);
      const uint32_t s = leftChild ? r + 1 : l;
      const uint32_t side = leftChild ? 0 : 1;
      if (s <= c0 || s >= cEnd) {  // sibling outside the chunk: global phase
        st_node_policy(a.nodes + 2ull * s + side, make_node(box.lx, box.ly, box.lz, box.hx, box.hy, box.hz, admin),
                       once);
        a.pending[2 * blockIdx.x + (s <= c0 ? 0 : 1)] = make_uint2(l, r);
        break;
      }
      const uint32_t js = s - c0;
      sBox[js][side][0] = make_float4(box.lx, box.ly, box.lz, box.hx);
      sBox[js][side][1] = make_float4(box.hy, box.hz, 0.f, 0.f);
      // block-scope release/acquire: the box is visible to the sibling that
      // sees this exchange, and this thread sees the sibling's box
      cuda::atomic_ref<uint32_t, cuda::thread_scope_block> slotRef(sSlot[js]);
      const uint32_t other = slotRef.exchange(leftChild ? l : r, cuda::memory_order_acq_rel);
      // the node itself is read only by the global phase (a later launch)
      st_node_policy(a.nodes + 2ull * s + side, make_node(box.lx, box.ly, box.lz, box.hx, box.hy, box.hz, admin),
                     once);
      if (other == AGG_EMPTY) break;  // parked; the sibling (here or in the global phase) carries on
      const float4 s0 = sBox[js][side ^ 1][0], s1 = sBox[js][side ^ 1][1];
      const AggBox sib{s0.x, s0.y, s0.z, s0.w, s1.x, s1.y};
      box = leftChild ? agg_union(box, sib) : agg_union(sib, box);
      if (leftChild) r = other; else l = other;
      if (a.ranges) a.ranges[s] = make_uint2(l, r);
      admin = make_admin(2ull * s - nodeBase, 0);
    }
  }
  __syncthreads();
  // The global slots of this chunk's splits, for the global phase (a later
  // launch): a child parked at a split whose sibling never came publishes
  // its range end there; every other slot, the chunk's first split (on its
  // boundary) included, starts empty.  (A slot whose two children met here
  // keeps the second one's end: no global climb ever reaches that split.)
  for (int j = threadIdx.x; j < AGG_CHUNK; j += blockDim.x)
    if (c0 + j < nv) a.slot[c0 + j] = j == 0 ? AGG_EMPTY : sSlot[j];
}

template <bool SEG, typename LevT>
__global__ void k_agg_global(AggArgsT<LevT> a, uint32_t numPending)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numPending) return;
  const uint32_t nv = *a.nvPtr;
  if ((uint64_t)(t / 2) * AGG_CHUNK >= nv) return;  // chunk had no prims: entry never written
  const uint2 pr = a.pending[t];
  if (pr.x == AGG_EMPTY) return;
  uint32_t l = pr.x, r = pr.y;
  uint32_t b0, e0;
  agg_range<SEG>(l, nv, a.off, a.numSegs, b0, e0);
  const uint64_t nodeBase = SEG ? 2ull * b0 : 0ull;
  // the split levels at the range's two boundaries, kept across steps: a
  // step changes one boundary, so it loads one level, together with the
  // sibling's box (one round trip to L2 per step besides the exchange)
  LevT dl = l > b0 ? __ldg(a.delta + l - 1) : (LevT)0;
  LevT dr = r < e0 - 1 ? __ldg(a.delta + r) : (LevT)0;
  // the node was written by the local phase: recover its box and admin
  bool leftChild = (l == b0) ? true : (r == e0 - 1) ? false : (dl > dr);
  uint32_t s = leftChild ? r + 1 : l;
  const Node me = ldcg_node(a.nodes + 2ull * s + (leftChild ? 0 : 1));
  AggBox box{me.a.x, me.a.y, me.a.z, me.a.w, me.b.x, me.b.y};
  uint64_t admin = node_admin(me);
  while (true) {
    if (l == b0 && r == e0 - 1) {
      a.nodes[nodeBase] = make_node(box.lx, box.ly, box.lz, box.hx, box.hy, box.hz, admin);
      return;
    }
    leftChild = (l == b0) ? true : (r == e0 - 1) ? false : (dl > dr);
    s = leftChild ? r + 1 : l;
    const uint64_t myPos = 2ull * s + (leftChild ? 0 : 1);
    a.nodes[myPos] = make_node(box.lx, box.ly, box.lz, box.hx, box.hy, box.hz, admin);
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> slotRef(a.slot[s]);
    const uint32_t other = slotRef.exchange(leftChild ? l : r, cuda::memory_order_acq_rel);
    if (other == AGG_EMPTY) return;
    if (leftChild) r = other; else l = other;
    // independent loads: the sibling's box and the new boundary's level
    const Node sn = ldcg_node(a.nodes + (myPos ^ 1));
    if (leftChild) dr = r < e0 - 1 ? __ldg(a.delta + r) : (LevT)0;
    else dl = l > b0 ? __ldg(a.delta + l - 1) : (LevT)0;
    const AggBox sib{sn.a.x, sn.a.y, sn.a.z, sn.a.w, sn.b.x, sn.b.y};
    box = leftChild ? agg_union(box, sib) : agg_union(sib, box);
    if (a.ranges) a.ranges[s] = make_uint2(l, r);
    admin = make_admin(2ull * s - nodeBase, 0);
  }
}

// launches both phases for nvMax (upper bound of *nvPtr) prims, each under
// its own profiler scope; split
// levels are 8-bit (Morton-63 builders) or 16-bit (rebin builder)
template <bool SEG, typename LevT>
inline int agglomerate(AggArgsT<LevT> a, uint32_t nvMax, cudaStream_t s, const char *profLocal = nullptr,
                       const char *profGlobal = nullptr)
{
  const int chunks = div_up(nvMax, AGG_CHUNK);
  {
    ProfScope ps(profLocal ? profLocal : "agg.local", s);
    BQ_CUDA(launch_pdl(k_agg_local<SEG, LevT>, dim3(chunks), dim3(AGG_CHUNK), 0, s, a));
  }
  {
    ProfScope ps(profGlobal ? profGlobal : "agg.global", s);
    BQ_CUDA(launch_pdl(k_agg_global<SEG, LevT>, dim3(div_up(2 * chunks, 128)), dim3(128), 0, s, a, 2u * chunks));
  }
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

} // namespace bq
