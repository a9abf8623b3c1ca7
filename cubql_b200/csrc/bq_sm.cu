// bq_sm.cu -- spatial-median BVH builder (the cuBQL::gpuBuilder method).
//
// Same splitting rule as gpuBuilder_impl (cuBQL/builder/cuda/sm_builder.h:
// 147-426): a node with more than makeLeafThreshold prims is split at the
// middle of its prims' centroid bounds along the widest axis (prims with
// centre >= pos go right); a node whose centroid bounds are flat or too thin
// to split (dim == -1) deals its prims to the two sides alternately.
//
// Different mechanics, B200-first.  The reference re-reads every prim at
// every level, grows child counts and centroid boxes with global atomics
// and syncs the host once per level down to the leaves.  Here:
//   * prims live as float4 (centre xyz, primID) in one of two buffers and
//     are partitioned stably, so every node owns a contiguous range and the
//     final prim order is the in-order leaf order;
//   * node slots follow from the partition: the children of a node split at
//     prim position m go to slots 2m, 2m+1 (root at 0) -- no allocation
//     counters; one scan over the used split positions compacts the slots at
//     the end (children of the k-th used split at nodes 2+2k, 2+2k+1; node 1
//     stays unused, as in the reference);
//   * nodes with more than warpMax prims (256..4096, chosen from the prim
//     count) are split level by level over the whole GPU in tiles of
//     SM_TILE prims: k_sm_tiles + one scan (tile offsets; one block,
//     k_sm_tiles_scan, up to SM_FUSED_MAX nodes), k_sm_count (right-side
//     count per tile), one scan + k_sm_children (one block,
//     k_sm_scan_children), k_sm_scatter (stable scatter that also reduces the
//     children's centroid bounds per tile and merges them with one
//     atomicMin/Max per tile -- min/max is order-independent, so the result
//     is deterministic), k_sm_classify (children to the next level's list or
//     to the warp tasks).  Lists and counts stay in device memory; the host
//     reads the counters only every SM_LEVELS_PER_CHECK levels;
//   * every subtree of at most warpMax prims is finished by one warp
//     of a persistent grid (k_sm_warp takes tasks from a counter), depth
//     first, smaller child first with the larger one on a per-warp
//     shared-memory stack; a node of up to 32 prims is held in
//     registers, one prim per lane, and its whole subtree is partitioned
//     with ballots and a 512-byte shared exchange buffer.
// Degenerate nodes send their k-th prim (primID order) to side
// (t0 + k) & 1, where t0 is the encoded centroid lower-z: that is the start
// value of the reference's tie-break counter, which aliases that field
// (sm_builder.h:82-103, 362-364), so child sizes match it exactly.  The
// partitions are stable, so "k-th in the node" is the k-th in primID order
// and leaves list their prims in ascending primID order, like the
// reference's final (nodeID, primID) sort (sm_builder.h:565-605).
#include <algorithm>
#include <climits>
#include <cfloat>
#include <cstring>
#include <vector>

#include "bq_internal.cuh"
#include "bq_refit.cuh"

namespace bq {

namespace {

// Warp subtrees hold at most warpMax prims: the largest power of two in
// [SM_WARP_MIN, SM_WARP_MAX] that still leaves SM_WARP_TASKS subtrees per SM,
// so small inputs do not end their global levels with a handful of warps
// busy and large ones do not pay for extra global levels.
constexpr uint32_t SM_WARP_MIN = 256;
constexpr uint32_t SM_WARP_MAX = 4096;
constexpr uint32_t SM_WARP_TASKS = 32;
constexpr uint32_t SM_TILE = 4096;      // prims per tile in the global levels
constexpr int SM_BLOCK = 256;           // global-level kernels
constexpr int SM_SCAT_GROUP = 4;        // chunks of SM_BLOCK prims k_sm_scatter loads at once
constexpr int SMW_BLOCK = 128;          // warp-phase kernel
constexpr int SMW_WARPS = SMW_BLOCK / 32;
constexpr int SMW_STACK = 24;           // >= log2(SM_WARP_MAX) + 1
constexpr int SM_LEVELS_PER_CHECK = 2;  // global levels between two host looks at the counters
constexpr int SM_SCAN_THREADS = BQ_SCAN_THREADS;  // one-block scans of a level's node and tile arrays
constexpr uint32_t SM_FUSED_MAX = BQ_SCAN_SMEM_MAX;

// A node still to be split: prim range [b, e) in buffer `parity`, its slot,
// and its prims' centroid bounds (encoded, see enc_f).
struct SmNode {
  uint32_t b, e, slot, parity;
  int32_t lo[3], hi[3];
};
static_assert(sizeof(SmNode) == 40, "SmNode size");

struct SmTile {
  uint32_t node, begin, end;
};

struct SmSplit {
  int dim;
  float pos;
  uint32_t tb;
};

// box center (lower + upper) / 2, as a multiply by 0.5: the same float
__device__ __forceinline__ float ctr2(float lo, float hi) { return __fmul_rn(__fadd_rn(lo, hi), 0.5f); }

// selectSplits (sm_builder.h:192-219)
__device__ __forceinline__ SmSplit choose_split(const SmNode &nd)
{
  float widestWidth = 0.f, wLo = 0.f, wHi = 0.f, wCtr = 0.f;
  int widestDim = -1;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const float l = dec_f(nd.lo[d]), h = dec_f(nd.hi[d]);
    const float width = __fsub_rn(h, l);
    if (width <= widestWidth) continue;
    const float c = __fmul_rn(0.5f, __fadd_rn(h, l));
    widestWidth = width; widestDim = d; wLo = l; wHi = h; wCtr = c;
  }
  SmSplit s;
  s.dim = (widestDim < 0 || wCtr == wLo || wCtr == wHi) ? -1 : widestDim;
  s.pos = wCtr;
  s.tb = (uint32_t)nd.lo[2];
  return s;
}

__device__ __forceinline__ uint32_t side_of(const float4 c, uint32_t rankInNode, const SmSplit &s)
{
  if (s.dim < 0) return (s.tb + rankInNode) & 1u;
  const float v = s.dim == 0 ? c.x : (s.dim == 1 ? c.y : c.z);
  return v >= s.pos ? 1u : 0u;
}

// running encoded min/max of the two children, without dynamic indexing
struct SideBounds {
  int32_t lo0[3], hi0[3], lo1[3], hi1[3];
  __device__ __forceinline__ void init()
  {
#pragma unroll
    for (int d = 0; d < 3; d++) { lo0[d] = lo1[d] = INT_MAX; hi0[d] = hi1[d] = INT_MIN; }
  }
  __device__ __forceinline__ void add(const float4 c, uint32_t side)
  {
    const int32_t e[3] = {enc_f(c.x), enc_f(c.y), enc_f(c.z)};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo0[d] = side ? lo0[d] : min(lo0[d], e[d]);
      hi0[d] = side ? hi0[d] : max(hi0[d], e[d]);
      lo1[d] = side ? min(lo1[d], e[d]) : lo1[d];
      hi1[d] = side ? max(hi1[d], e[d]) : hi1[d];
    }
  }
  __device__ __forceinline__ void warp_reduce()
  {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      lo0[d] = __reduce_min_sync(0xffffffffu, lo0[d]);
      hi0[d] = __reduce_max_sync(0xffffffffu, hi0[d]);
      lo1[d] = __reduce_min_sync(0xffffffffu, lo1[d]);
      hi1[d] = __reduce_max_sync(0xffffffffu, hi1[d]);
    }
  }
};

__device__ __forceinline__ void internal_node(Node *out, uint32_t *used, uint32_t slot, uint32_t m)
{
  out[slot] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(2ull * m, 0));
  used[m] = 1;
}

__device__ __forceinline__ void child_pair(const SmNode &nd, uint32_t m, const SideBounds &sb, SmNode &c0, SmNode &c1)
{
  c0.b = nd.b; c0.e = m; c0.slot = 2 * m; c0.parity = nd.parity ^ 1u;
  c1.b = m; c1.e = nd.e; c1.slot = 2 * m + 1; c1.parity = nd.parity ^ 1u;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    c0.lo[d] = sb.lo0[d]; c0.hi[d] = sb.hi0[d];
    c1.lo[d] = sb.lo1[d]; c1.hi[d] = sb.hi1[d];
  }
}

// ------------------------------------------------------------------
// set-up: valid prims compacted (primID order) as float4, invalid ones
// listed after them in primIDs, root centroid bounds
// ------------------------------------------------------------------
__global__ void k_sm_valid(const bq_box3f *__restrict__ boxes, uint32_t n, uint32_t *__restrict__ valid)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 a = *reinterpret_cast<const float2 *>(boxes + i);
  const float2 b = *(reinterpret_cast<const float2 *>(boxes + i) + 1);
  valid[i] = (a.x <= b.y) ? 1u : 0u;  // initPrims: lower.x <= upper.x (sm_builder.h:134)
}

// grid-stride over the prims with blocks of 256 (the block reduction needs
// every thread); root bounds merged once per block
__global__ void __launch_bounds__(256) k_sm_init(const bq_box3f *__restrict__ boxes, uint32_t n,
                                                 const uint32_t *__restrict__ vpos, const uint32_t *nvPtr,
                                                 float4 *__restrict__ pc, uint32_t *__restrict__ primIDs,
                                                 int32_t *rootLoHi)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  int32_t lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const bq_box3f b = boxes[i];
    const uint32_t p = vpos[i];
    if (b.lower[0] <= b.upper[0]) {
      const float4 c = make_float4(ctr2(b.lower[0], b.upper[0]), ctr2(b.lower[1], b.upper[1]),
                                   ctr2(b.lower[2], b.upper[2]), __uint_as_float((uint32_t)i));
      pc[p] = c;
      const int32_t e[3] = {enc_f(c.x), enc_f(c.y), enc_f(c.z)};
#pragma unroll
      for (int d = 0; d < 3; d++) { lo[d] = min(lo[d], e[d]); hi[d] = max(hi[d], e[d]); }
    } else {
      primIDs[nv + ((uint32_t)i - p)] = (uint32_t)i;  // invalid prims after all valid ones, ascending
    }
  }
  block_merge_bounds<256>(lo, hi, rootLoHi);
}

// ------------------------------------------------------------------
// global levels (nodes with more than warpMax prims)
// ------------------------------------------------------------------
// Device-side state of the global levels.  The big-node lists ping-pong
// between two buffers; their counts, the current level's tile count and
// the warp-phase task list live here, so levels run without the host.
struct SmCtl {
  uint32_t bigCount[2];  // nodes in big list 0 / 1
  uint32_t numTiles;     // tiles of the current level (scan total)
  uint32_t scanLen;      // numTiles + 1
  uint32_t taskCount;    // subtrees waiting for the warp phase
  uint32_t grab;         // warp-phase task counter
  uint32_t err;          // DEV_ERR_RANGE on a broken capacity bound
  uint32_t pad;
};

// tiles of a level: node k owns tiles [first[k], first[k+1]) (last: numTiles)
struct SmTileInfo {
  uint32_t node, begin, end;
};
__device__ __forceinline__ uint32_t first_end(const uint32_t *__restrict__ first, uint32_t K, uint32_t T, uint32_t k)
{
  return k + 1 < K ? first[k + 1] : T;
}
__device__ __forceinline__ SmTileInfo tile_info(const SmNode *__restrict__ nodes, const uint32_t *__restrict__ first,
                                                uint32_t K, uint32_t t)
{
  uint32_t lo = 0, hi = K;  // last node whose first tile is <= t
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (first[m] <= t) lo = m; else hi = m;
  }
  SmTileInfo r;
  r.node = lo;
  r.begin = nodes[lo].b + (t - first[lo]) * SM_TILE;
  r.end = min(nodes[lo].e, r.begin + SM_TILE);
  return r;
}

// tiles per big node of the current list
__global__ void k_sm_tiles(const SmNode *__restrict__ nodes, SmCtl *ctl, int cur, uint32_t cap,
                           uint32_t *__restrict__ tileCount)
{
  griddep_wait();
  const uint32_t K = ctl->bigCount[cur];
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0 && K > cap) atomicOr(&ctl->err, DEV_ERR_RANGE);
  if (k == 0) ctl->bigCount[cur ^ 1] = 0;  // the list this level's k_sm_classify fills (last read a level ago)
  if (k >= K || k >= cap) return;
  tileCount[k] = (nodes[k].e - nodes[k].b + SM_TILE - 1) / SM_TILE;
}

// k_sm_tiles and the scan of its counts in one block (the level's big
// nodes, at most cap <= SM_FUSED_MAX, counted in shared memory)
__global__ void __launch_bounds__(SM_SCAN_THREADS) k_sm_tiles_scan(const SmNode *__restrict__ nodes, SmCtl *ctl,
                                                                   int cur, uint32_t cap, uint32_t maxTiles,
                                                                   uint32_t *__restrict__ first)
{
  griddep_wait();
  extern __shared__ uint32_t sVal[];  // cap entries
  __shared__ uint32_t sWarp[33];
  uint32_t K = ctl->bigCount[cur];
  if (K > cap) {
    if (threadIdx.x == 0) atomicOr(&ctl->err, DEV_ERR_RANGE);
    K = cap;
  }
  if (threadIdx.x == 0) ctl->bigCount[cur ^ 1] = 0;  // the list this level's k_sm_classify fills (last read a level ago)
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) sVal[k] = (nodes[k].e - nodes[k].b + SM_TILE - 1) / SM_TILE;
  __syncthreads();
  const uint32_t T = block_scan_smem(sVal, K, sWarp);
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) first[k] = sVal[k];
  if (threadIdx.x == 0) {
    if (T >= maxTiles) atomicOr(&ctl->err, DEV_ERR_RANGE);
    ctl->numTiles = min(T, maxTiles - 1);
  }
}

// right-side count per tile; the blocks walk the level's tiles
__global__ void __launch_bounds__(SM_BLOCK) k_sm_count(const SmNode *__restrict__ nodes,
                                                       const uint32_t *__restrict__ first, SmCtl *ctl, int cur,
                                                       uint32_t maxTiles, const float4 *__restrict__ buf0,
                                                       const float4 *__restrict__ buf1, uint32_t *__restrict__ tileRight)
{
  griddep_wait();
  __shared__ uint32_t sCnt[SM_BLOCK / 32];
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (T >= maxTiles) atomicOr(&ctl->err, DEV_ERR_RANGE);
    else tileRight[T] = 0;  // the scan's total slot
    ctl->scanLen = min(T, maxTiles - 1) + 1;
  }
  for (uint32_t tile = blockIdx.x; tile < T && tile < maxTiles - 1; tile += gridDim.x) {  // whole block
    const SmTileInfo t = tile_info(nodes, first, K, tile);
    const SmNode nd = nodes[t.node];
    const SmSplit sp = choose_split(nd);
    const float4 *src = nd.parity ? buf1 : buf0;
    uint32_t c = 0;
#pragma unroll 4
    for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += SM_BLOCK) c += side_of(src[i], i - nd.b, sp);
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) sCnt[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t s = 0;
      for (int w = 0; w < SM_BLOCK / 32; w++) s += sCnt[w];
      tileRight[tile] = s;
    }
    __syncthreads();
  }
}

// per node: the split position, the internal node, the two child records
// (bounds start empty; k_sm_scatter fills them)
__global__ void k_sm_children(const SmNode *__restrict__ nodes, const SmCtl *ctl, int cur, uint32_t cap,
                              const uint32_t *__restrict__ first, const uint32_t *__restrict__ rightScan,
                              Node *__restrict__ out, uint32_t *__restrict__ used, SmNode *__restrict__ next)
{
  griddep_wait();
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K || k >= cap) return;
  const SmNode nd = nodes[k];
  const uint32_t nR = rightScan[first_end(first, K, T, k)] - rightScan[first[k]];
  const uint32_t m = nd.e - nR;  // left child is [b, m)
  internal_node(out, used, nd.slot, m);
  SideBounds sb;
  sb.init();
  SmNode c0, c1;
  child_pair(nd, m, sb, c0, c1);
  next[2 * k] = c0;
  next[2 * k + 1] = c1;
}

// the scan of the tiles' right counts and k_sm_children in one block
// (numTiles + 1 <= SM_FUSED_MAX entries in shared memory)
__global__ void __launch_bounds__(SM_SCAN_THREADS) k_sm_scan_children(const SmNode *__restrict__ nodes,
                                                                      const SmCtl *ctl, int cur, uint32_t cap,
                                                                      const uint32_t *__restrict__ first,
                                                                      uint32_t *__restrict__ tileRight,
                                                                      Node *__restrict__ out,
                                                                      uint32_t *__restrict__ used,
                                                                      SmNode *__restrict__ next)
{
  griddep_wait();
  extern __shared__ uint32_t sScan[];  // numTiles + 1 entries
  __shared__ uint32_t sWarp[33];
  const uint32_t K = min(ctl->bigCount[cur], cap), T = ctl->numTiles;
  for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) sScan[i] = tileRight[i];
  __syncthreads();
  const uint32_t total = block_scan_smem(sScan, T, sWarp);
  for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) tileRight[i] = sScan[i];
  if (threadIdx.x == 0) {
    tileRight[T] = total;
    sScan[T] = total;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
    const SmNode nd = nodes[k];
    const uint32_t nR = sScan[first_end(first, K, T, k)] - sScan[first[k]];
    const uint32_t m = nd.e - nR;  // left child is [b, m)
    internal_node(out, used, nd.slot, m);
    SideBounds sb;
    sb.init();
    SmNode c0, c1;
    child_pair(nd, m, sb, c0, c1);
    next[2 * k] = c0;
    next[2 * k + 1] = c1;
  }
}

// one tile of k_sm_scatter: the stable scatter of its prims and the
// children's centroid bounds (one atomicMin/Max per component)
__device__ __forceinline__ void scatter_tile(const SmNode *__restrict__ nodes, const uint32_t *__restrict__ first,
                                             uint32_t K, uint32_t T, uint32_t tile,
                                             const uint32_t *__restrict__ rightScan, float4 *buf0, float4 *buf1,
                                             SmNode *next, uint32_t *sWarp, int32_t (*sRed)[SM_BLOCK / 32])
{
  const SmTileInfo t = tile_info(nodes, first, K, tile);
  const SmNode nd = nodes[t.node];
  const SmSplit sp = choose_split(nd);
  const float4 *src = nd.parity ? buf1 : buf0;
  float4 *dst = nd.parity ? buf0 : buf1;
  const uint32_t nodeRight0 = rightScan[first[t.node]];
  const uint32_t m = nd.e - (rightScan[first_end(first, K, T, t.node)] - nodeRight0);
  uint32_t rBefore = rightScan[tile] - nodeRight0;  // this node's rights before the tile
  uint32_t lBefore = (t.begin - nd.b) - rBefore;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  SideBounds sb;
  sb.init();
  // SM_SCAT_GROUP chunks of SM_BLOCK prims per round: their loads are in
  // flight together and one barrier pair ranks all of them
  for (uint32_t base = t.begin; base < t.end; base += SM_BLOCK * SM_SCAT_GROUP) {
    float4 c[SM_SCAT_GROUP];
    uint32_t side[SM_SCAT_GROUP], bal[SM_SCAT_GROUP];
#pragma unroll
    for (int g = 0; g < SM_SCAT_GROUP; g++) {
      const uint32_t i = base + g * SM_BLOCK + threadIdx.x;
      c[g] = i < t.end ? src[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int g = 0; g < SM_SCAT_GROUP; g++) {
      const uint32_t i = base + g * SM_BLOCK + threadIdx.x;
      const bool valid = i < t.end;
      side[g] = valid ? side_of(c[g], i - nd.b, sp) : 0u;
      bal[g] = __ballot_sync(0xffffffffu, valid && side[g]);
      if (lane == 0) sWarp[g * (SM_BLOCK / 32) + warp] = __popc(bal[g]);
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < SM_SCAT_GROUP; g++) {
      const uint32_t cb = base + g * SM_BLOCK;
      if (cb >= t.end) break;  // the same for the whole block
      uint32_t rw = 0, rtot = 0;
#pragma unroll
      for (int w = 0; w < SM_BLOCK / 32; w++) {
        const uint32_t x = sWarp[g * (SM_BLOCK / 32) + w];
        rw += (w < warp) ? x : 0u;
        rtot += x;
      }
      if (cb + threadIdx.x < t.end) {
        const uint32_t rMine = rw + __popc(bal[g] & lt);  // rights of this chunk before me
        dst[side[g] ? m + rBefore + rMine : nd.b + lBefore + (threadIdx.x - rMine)] = c[g];
        sb.add(c[g], side[g]);
      }
      const uint32_t chunk = min((uint32_t)SM_BLOCK, t.end - cb);
      rBefore += rtot;
      lBefore += chunk - rtot;
    }
    __syncthreads();
  }
  sb.warp_reduce();
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      sRed[d][warp] = sb.lo0[d]; sRed[3 + d][warp] = sb.hi0[d];
      sRed[6 + d][warp] = sb.lo1[d]; sRed[9 + d][warp] = sb.hi1[d];
    }
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    const int j = threadIdx.x, comp = j % 6;
    const bool isMin = comp < 3;
    int32_t v = isMin ? INT_MAX : INT_MIN;
    for (int w = 0; w < SM_BLOCK / 32; w++) v = isMin ? min(v, sRed[j][w]) : max(v, sRed[j][w]);
    SmNode *child = next + 2 * t.node + (j / 6);
    if (isMin) {
      if (v != INT_MAX) atomicMin(&child->lo[comp], v);
    } else {
      if (v != INT_MIN) atomicMax(&child->hi[comp - 3], v);
    }
  }
  __syncthreads();  // sWarp and sRed are reused by the block's next tile
}

// 4 blocks per SM (at most 64 registers): the four chunks' loads in flight
// pay more than a fifth block would
__global__ void __launch_bounds__(SM_BLOCK, 4) k_sm_scatter(const SmNode *__restrict__ nodes,
                                                         const uint32_t *__restrict__ first, const SmCtl *ctl,
                                                         int cur, uint32_t maxTiles,
                                                         const uint32_t *__restrict__ rightScan, float4 *buf0,
                                                         float4 *buf1, SmNode *next)
{
  griddep_wait();
  __shared__ uint32_t sWarp[SM_SCAT_GROUP * SM_BLOCK / 32];
  __shared__ int32_t sRed[12][SM_BLOCK / 32];
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  for (uint32_t tile = blockIdx.x; tile < T && tile < maxTiles - 1; tile += gridDim.x)  // whole block
    scatter_tile(nodes, first, K, T, tile, rightScan, buf0, buf1, next, sWarp, sRed);
}

// ------------------------------------------------------------------
// warp phase: whole subtrees of at most warpMax prims
// ------------------------------------------------------------------
__device__ __forceinline__ void leaf_node(Node *out, uint32_t slot, uint32_t b, uint32_t count)
{
  out[slot] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(b, count));
}

// A node of 2..32 prims: lane j holds the prim at position nd.b + j, the
// whole subtree is built in registers.  Stack entries go to stk[0..].
__device__ void sm_small_subtree(const SmNode &root, const float4 *src, int thr, float4 *xbuf, SmNode *stk,
                                 int stackLeft, Node *__restrict__ out, uint32_t *__restrict__ primIDs,
                                 uint32_t *__restrict__ used, uint32_t *err)
{
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t base = root.b, cnt = root.e - root.b;
  float4 c = lane < (int)cnt ? src[base + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t pos = base + lane;
  SmNode cur = root;
  int sp = 0;
  while (true) {
    const uint32_t count = cur.e - cur.b;
    if ((int64_t)count <= thr) {
      if (lane == 0) leaf_node(out, cur.slot, cur.b, count);
      if (sp == 0) break;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    const SmSplit spl = choose_split(cur);
    const bool in = pos >= cur.b && pos < cur.e;
    const uint32_t side = in ? side_of(c, pos - cur.b, spl) : 0u;
    const uint32_t balR = __ballot_sync(0xffffffffu, in && side);
    const uint32_t balL = __ballot_sync(0xffffffffu, in && !side);
    const uint32_t m = cur.e - __popc(balR);
    // a child of at most thr prims is a leaf: written here, never split, so
    // its centroid bounds are not needed
    const bool leafL = (int64_t)(m - cur.b) <= thr, leafR = (int64_t)(cur.e - m) <= thr;
    SideBounds sb;
    sb.init();
    if (!(leafL && leafR)) {
      if (in) sb.add(c, side);
      sb.warp_reduce();
    }
    const uint32_t dest = !in ? (uint32_t)lane
                              : (side ? (m - base) + __popc(balR & lt) : (cur.b - base) + __popc(balL & lt));
    xbuf[dest] = c;
    __syncwarp();
    c = xbuf[lane];
    __syncwarp();
    SmNode c0, c1;
    child_pair(cur, m, sb, c0, c1);
    if (lane == 0) {
      internal_node(out, used, cur.slot, m);
      if (leafL) leaf_node(out, c0.slot, c0.b, c0.e - c0.b);
      if (leafR) leaf_node(out, c1.slot, c1.b, c1.e - c1.b);
    }
    if (leafL && leafR) {
      if (sp == 0) break;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    if (leafL || leafR) {
      cur = leafL ? c1 : c0;
      continue;
    }
    const bool leftSmaller = (m - cur.b) <= (cur.e - m);
    if (sp >= stackLeft) {  // unreachable: the stacked child is always the larger one
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      break;
    }
    if (lane == 0) stk[sp] = leftSmaller ? c1 : c0;
    sp++;
    cur = leftSmaller ? c0 : c1;
  }
  if (lane < (int)cnt) primIDs[base + lane] = __float_as_uint(c.w);
  __syncwarp();
}

// one subtree of at most warpMax prims, by the calling warp; stk and
// xbuf are the warp's shared-memory stack and exchange buffer
__device__ void sm_warp_task(SmNode cur, int thr, float4 *buf0, float4 *buf1, Node *__restrict__ out,
                             uint32_t *__restrict__ primIDs, uint32_t *__restrict__ used, uint32_t *err, SmNode *stk,
                             float4 *xbuf)
{
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  int sp = 0;
  while (true) {
    const uint32_t count = cur.e - cur.b;
    const float4 *src = cur.parity ? buf1 : buf0;
    float4 *dst = cur.parity ? buf0 : buf1;
    if ((int64_t)count <= thr || count <= 32) {
      if ((int64_t)count <= thr) {  // leaf: its prims are final
        for (uint32_t i = cur.b + lane; i < cur.e; i += 32) primIDs[i] = __float_as_uint(src[i].w);
        if (lane == 0) leaf_node(out, cur.slot, cur.b, count);
      } else {
        sm_small_subtree(cur, src, thr, xbuf, stk + sp, SMW_STACK - sp, out, primIDs, used, err);
      }
      if (sp == 0) return;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    const SmSplit spl = choose_split(cur);
    // pass 1: right-side count
    uint32_t nR = 0;
#pragma unroll 4
    for (uint32_t i = cur.b + lane; i < cur.e; i += 32) nR += side_of(src[i], i - cur.b, spl);
    nR = __reduce_add_sync(0xffffffffu, nR);
    const uint32_t m = cur.e - nR;
    // pass 2: stable scatter + children's bounds, 128 prims per round
    uint32_t lB = 0, rB = 0;
    SideBounds sb;
    sb.init();
    for (uint32_t base = cur.b; base < cur.e; base += 128) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t i = base + 32u * u + lane;
        v[u] = i < cur.e ? src[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const uint32_t i = base + 32u * u + lane;
        const bool valid = i < cur.e;
        const uint32_t s = valid ? side_of(v[u], i - cur.b, spl) : 0u;
        const uint32_t balR = __ballot_sync(0xffffffffu, valid && s);
        const uint32_t balL = __ballot_sync(0xffffffffu, valid && !s);
        if (valid) {
          dst[s ? m + rB + __popc(balR & lt) : cur.b + lB + __popc(balL & lt)] = v[u];
          sb.add(v[u], s);
        }
        rB += __popc(balR);
        lB += __popc(balL);
      }
    }
    sb.warp_reduce();
    if (lane == 0) internal_node(out, used, cur.slot, m);
    SmNode c0, c1;
    child_pair(cur, m, sb, c0, c1);
    const bool leftSmaller = (m - cur.b) <= (cur.e - m);
    if (sp >= SMW_STACK) {  // unreachable: the stacked child is always the larger one
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      return;
    }
    if (lane == 0) stk[sp] = leftSmaller ? c1 : c0;
    sp++;
    cur = leftSmaller ? c0 : c1;
    __syncwarp();  // this warp's scatter is visible to its own next pass
  }
}

// persistent grid: each warp takes the next waiting subtree until none is left
__global__ void __launch_bounds__(SMW_BLOCK) k_sm_warp(const SmNode *__restrict__ tasks, SmCtl *ctl, uint32_t taskCap,
                                                       int thr, float4 *buf0, float4 *buf1, Node *__restrict__ out,
                                                       uint32_t *__restrict__ primIDs, uint32_t *__restrict__ used)
{
  griddep_wait();
  __shared__ SmNode sStack[SMW_WARPS][SMW_STACK];
  __shared__ float4 sX[SMW_WARPS][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const uint32_t numTasks = min(ctl->taskCount, taskCap);
  while (true) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&ctl->grab, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= numTasks) return;  // whole warp
    sm_warp_task(tasks[t], thr, buf0, buf1, out, primIDs, used, &ctl->err, sStack[wb], sX[wb]);
    __syncwarp();
  }
}

// children of the level's big nodes: to the next big list or to the tasks
__global__ void k_sm_classify(const SmNode *__restrict__ next, SmCtl *ctl, int cur, uint32_t cap, int thr,
                              uint32_t warpMax, SmNode *__restrict__ bigNext, SmNode *__restrict__ tasks,
                              uint32_t taskCap)
{
  griddep_wait();
  const uint32_t K = min(ctl->bigCount[cur], cap);
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 2 * K) return;
  const SmNode c = next[j];
  const uint32_t size = c.e - c.b;
  if (size > warpMax && (int64_t)size > thr) {
    const uint32_t at = atomicAdd(&ctl->bigCount[cur ^ 1], 1u);
    if (at < cap) bigNext[at] = c;
    else atomicOr(&ctl->err, DEV_ERR_RANGE);  // cannot happen: big nodes are disjoint and above warpMax
  } else {
    const uint32_t at = atomicAdd(&ctl->taskCount, 1u);
    if (at < taskCap) tasks[at] = c;
    else atomicOr(&ctl->err, DEV_ERR_RANGE);  // the host flushes the tasks before this can happen
  }
}

// ------------------------------------------------------------------
// slot compaction: split m's children move from 2m, 2m+1 to 2+2*rank[m]
// ------------------------------------------------------------------
__device__ __forceinline__ Node sm_remap(const Node &c, const uint32_t *__restrict__ rank)
{
  const uint64_t a = node_admin(c);
  if (admin_count(a)) return c;
  const uint32_t cm = (uint32_t)(admin_offset(a) >> 1);
  return make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(2ull + 2ull * rank[cm], 0));
}

// an inner node written at index q is its children's parent
__device__ __forceinline__ void sm_link_children(const Node &c, uint32_t q, uint32_t *__restrict__ parent)
{
  const uint64_t a = node_admin(c);
  if (admin_count(a)) return;
  const uint64_t o = admin_offset(a);
  parent[o] = q;
  parent[o + 1] = q;
}

// Also writes what the refit's climb needs, which the generic refit would
// find with two more passes over the nodes: every node's parent and a zero
// arrival counter (the climb is k_refit_climb of bq_refit.cuh).
__global__ void k_sm_compact(const Node *__restrict__ full, const uint32_t *__restrict__ used,
                             const uint32_t *__restrict__ rank, uint32_t nv, Node *__restrict__ out,
                             uint32_t *__restrict__ parent, uint32_t *__restrict__ counter, uint32_t *__restrict__ err)
{
  griddep_wait();
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) {
    const Node root = sm_remap(full[0], rank);
    out[0] = root;
    out[1] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0);
    parent[0] = RF_NO_PARENT;
    parent[1] = RF_NO_PARENT;
    counter[0] = 0;
    counter[1] = 0;
    *err = 0;
    sm_link_children(root, 0, parent);
    return;
  }
  if (m >= nv || !used[m]) return;
  const uint32_t pair = 2u + 2u * rank[m];
#pragma unroll
  for (uint32_t side = 0; side < 2; side++) {
    const Node c = sm_remap(full[2ull * m + side], rank);
    out[pair + side] = c;
    counter[pair + side] = 0;
    sm_link_children(c, pair + side, parent);
  }
}

} // namespace

int build_spatial_median(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
{
  int thr = cfg ? cfg->makeLeafThreshold : 0;
  if (thr == 0) thr = 1;  // gpu_builder.h:60-63
  if (thr < 1 || thr > 65535)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "makeLeafThreshold must be in [0, 65535] (16-bit leaf count)");
  bvh->nodes = nullptr; bvh->primIDs = nullptr; bvh->numNodes = 0; bvh->numPrims = 0;
  if (n == 0) return BQ_OK;  // gpu_builder.h:39

  TempSet tmp(al);
  uint32_t *valid = nullptr, *vpos = nullptr, *ctl = nullptr, *used = nullptr;
  float4 *buf0 = nullptr, *buf1 = nullptr;
  BQ_TRY(tmp.get(&valid, n));
  BQ_TRY(tmp.get(&vpos, n));
  BQ_TRY(tmp.get(&ctl, 8));  // [0] valid count [1] device error bits [2..7] root centroid bounds
  BQ_TRY(tmp.get(&buf0, n));
  BQ_TRY(tmp.get(&buf1, n));
  BQ_TRY(tmp.get(&used, n));
  uint32_t *primIDs = nullptr;
  BQ_TRY(al.get(&primIDs, n));
  auto fail = [&](int code) {
    al.free_bytes(primIDs);
    return code;
  };
  int s;
  cudaError_t ce;
  const int32_t ctlInit[8] = {0, 0, INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  if ((ce = cudaMemcpyAsync(ctl, ctlInit, 32, cudaMemcpyHostToDevice, al.s)) != cudaSuccess ||
      (ce = cudaMemsetAsync(used, 0, sizeof(uint32_t) * n, al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "spatial median set-up"));
  {
    ProfScope ps("sm.setup", al.s, 5);
    launch_pdl(k_sm_valid, dim3(div_up(n, 256)), dim3(256), 0, al.s, boxes, n, valid);
    if ((s = exclusive_scan_u32(valid, vpos, n, nullptr, ctl, al)) != BQ_OK) return fail(s);
    launch_pdl(k_sm_init, dim3(std::min(div_up(n, 256), num_sms() * 8)), dim3(256), 0, al.s, boxes, n, vpos, ctl,
               buf0, primIDs, (int32_t *)(ctl + 2));
  }
  int32_t hctl[8];
  if ((ce = cudaMemcpyAsync(hctl, ctl, 32, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "spatial median set-up"));
  const uint32_t nv = (uint32_t)hctl[0];
  if (nv == 0) {  // nothing to build over
    al.free_bytes(primIDs);
    return BQ_OK;
  }
  Node *full = nullptr;
  if ((s = tmp.get(&full, 2ull * nv)) != BQ_OK) return fail(s);

  // ---- global levels, driven from device memory ----
  // Big nodes (more than warpMax prims) of one level are disjoint, so a
  // level holds at most cap of them and at most maxTiles tiles.  The host
  // looks at the counters first when perfectly balanced splits would be
  // done, then every SM_LEVELS_PER_CHECK levels; a level with no big node
  // left costs only its (empty) launches.  Every level adds at most 2 * cap
  // warp tasks, which bounds the task list between two looks.
  // warp subtrees small enough that every SM gets several of them
  uint32_t warpMax = SM_WARP_MIN;
  while (warpMax < SM_WARP_MAX && (uint64_t)warpMax * 2 * num_sms() * SM_WARP_TASKS <= nv) warpMax *= 2;
  const uint32_t cap = nv / (warpMax + 1) + 1;
  const uint32_t maxTiles = nv / SM_TILE + cap + 2;
  int nextCheck = 1;
  while (nextCheck < 62 && ((uint64_t)warpMax << nextCheck) < nv) nextCheck++;
  const uint32_t taskCap =
      std::max<uint32_t>(16 * cap, 4096) + 2 * cap * (uint32_t)std::max(nextCheck, SM_LEVELS_PER_CHECK);
  SmCtl *sc = nullptr;
  SmNode *bigList[2] = {nullptr, nullptr}, *next = nullptr, *tasks = nullptr;
  uint32_t *tileCount = nullptr, *first = nullptr, *tileRight = nullptr;
  if ((s = tmp.get(&sc, 1)) != BQ_OK || (s = tmp.get(&bigList[0], cap)) != BQ_OK ||
      (s = tmp.get(&bigList[1], cap)) != BQ_OK || (s = tmp.get(&next, 2ull * cap)) != BQ_OK ||
      (s = tmp.get(&tasks, taskCap)) != BQ_OK || (s = tmp.get(&tileCount, cap)) != BQ_OK ||
      (s = tmp.get(&first, cap)) != BQ_OK || (s = tmp.get(&tileRight, maxTiles)) != BQ_OK)
    return fail(s);
  SmNode root;
  root.b = 0; root.e = nv; root.slot = 0; root.parity = 0;
  for (int d = 0; d < 3; d++) { root.lo[d] = hctl[2 + d]; root.hi[d] = hctl[5 + d]; }
  const bool rootBig = nv > warpMax && (int64_t)nv > thr;
  SmCtl hsc{};
  hsc.bigCount[0] = rootBig ? 1u : 0u;
  hsc.taskCount = rootBig ? 0u : 1u;
  if ((ce = cudaMemcpyAsync(rootBig ? bigList[0] : tasks, &root, sizeof(root), cudaMemcpyHostToDevice, al.s)) !=
          cudaSuccess ||
      (ce = cudaMemcpyAsync(sc, &hsc, sizeof(hsc), cudaMemcpyHostToDevice, al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "spatial median set-up"));
  const int warpGrid = num_sms() * 8;
  // the level's tile kernels walk the tiles with at most 8 blocks per SM; with
  // at most SM_FUSED_MAX nodes and tiles a level's two scans run inside one
  // block each (5 launches per level instead of 11)
  const int levelGrid = std::max(1, std::min<int>((int)maxTiles, num_sms() * 8));
  const bool fused = cap <= SM_FUSED_MAX && maxTiles <= SM_FUSED_MAX;
  if (fused) {
    if ((ce = cudaFuncSetAttribute(k_sm_tiles_scan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(uint32_t) * cap))) != cudaSuccess ||
        (ce = cudaFuncSetAttribute(k_sm_scan_children, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(uint32_t) * maxTiles))) != cudaSuccess)
      return fail(cuda_error(ce, "spatial median set-up"));
  }
  auto warp_phase = [&]() -> int {  // every waiting subtree, then an empty task list
    ProfScope ps("sm.warps", al.s);
    launch_pdl(k_sm_warp, dim3(warpGrid), dim3(SMW_BLOCK), 0, al.s, tasks, sc, taskCap, thr, buf0, buf1, full,
               primIDs, used);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->taskCount, 0, 2 * sizeof(uint32_t), al.s);  // taskCount, grab
    return e == cudaSuccess ? BQ_OK : cuda_error(e, "k_sm_warp");
  };
  int cur = 0;
  for (int level = 0; rootBig; level++) {
    {
      ProfScope ps("sm.level", al.s, fused ? 5 : 11);
      if (fused) {
        launch_pdl(k_sm_tiles_scan, dim3(1), dim3(SM_SCAN_THREADS), sizeof(uint32_t) * cap, al.s, bigList[cur], sc,
                   cur, cap, maxTiles, first);
      } else {
        launch_pdl(k_sm_tiles, dim3(div_up(cap, 128)), dim3(128), 0, al.s, bigList[cur], sc, cur, cap, tileCount);
        if ((s = exclusive_scan_u32(tileCount, first, cap, &sc->bigCount[cur], &sc->numTiles, al)) != BQ_OK)
          return fail(s);
      }
      launch_pdl(k_sm_count, dim3(levelGrid), dim3(SM_BLOCK), 0, al.s, bigList[cur], first, sc, cur, maxTiles, buf0,
                 buf1, tileRight);
      if (fused) {
        launch_pdl(k_sm_scan_children, dim3(1), dim3(SM_SCAN_THREADS), sizeof(uint32_t) * maxTiles, al.s,
                   bigList[cur], sc, cur, cap, first, tileRight, full, used, next);
      } else {
        if ((s = exclusive_scan_u32(tileRight, tileRight, maxTiles, &sc->scanLen, nullptr, al)) != BQ_OK)
          return fail(s);
        launch_pdl(k_sm_children, dim3(div_up(cap, 128)), dim3(128), 0, al.s, bigList[cur], sc, cur, cap, first,
                   tileRight, full, used, next);
      }
      launch_pdl(k_sm_scatter, dim3(levelGrid), dim3(SM_BLOCK), 0, al.s, bigList[cur], first, sc, cur, maxTiles,
                 tileRight, buf0, buf1, next);
      launch_pdl(k_sm_classify, dim3(div_up(2ull * cap, 128)), dim3(128), 0, al.s, next, sc, cur, cap, thr, warpMax,
                 bigList[cur ^ 1], tasks, taskCap);
      if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_error(ce, "spatial median level"));
    }
    cur ^= 1;
    if (level + 1 < nextCheck) continue;
    nextCheck = level + 1 + SM_LEVELS_PER_CHECK;
    if ((ce = cudaMemcpyAsync(&hsc, sc, sizeof(hsc), cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "spatial median levels"));
    if (hsc.err) return fail(set_error(BQ_ERR_CUDA, "spatial-median level failed a capacity check"));
    if (hsc.bigCount[cur] == 0) break;
    // the next SM_LEVELS_PER_CHECK levels add at most 2 * cap tasks each
    if (hsc.taskCount + 2ull * SM_LEVELS_PER_CHECK * cap > taskCap && (s = warp_phase()) != BQ_OK) return fail(s);
  }
  // ---- warp phase ----
  if ((s = warp_phase()) != BQ_OK) return fail(s);
  // ---- slot compaction ----
  uint32_t *rank = nullptr;
  if ((s = tmp.get(&rank, nv)) != BQ_OK) return fail(s);
  {
    ProfScope ps("sm.rank", al.s, 3);
    if ((s = exclusive_scan_u32(used, rank, nv, nullptr, ctl + 2, al)) != BQ_OK) return fail(s);
  }
  uint32_t hres[2], herr = 0;
  if ((ce = cudaMemcpyAsync(hres, ctl + 1, 8, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(&herr, &sc->err, 4, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "spatial median"));
  if (hres[0] || herr) return fail(set_error(BQ_ERR_CUDA, "spatial-median build failed a range or capacity check"));
  const uint32_t numNodes = 2 + 2 * hres[1];
  Node *nodes = nullptr;
  uint32_t *rfParent = nullptr;  // parent[numNodes], counter[numNodes], err[1]
  if ((s = tmp.get(&rfParent, 2ull * numNodes + 1)) != BQ_OK) return fail(s);
  uint32_t *rfCounter = rfParent + numNodes, *rfErr = rfParent + 2ull * numNodes;
  if ((s = al.get(&nodes, numNodes)) != BQ_OK) return fail(s);
  {
    ProfScope ps("sm.compact", al.s);
    launch_pdl(k_sm_compact, dim3(div_up(nv, 256)), dim3(256), 0, al.s, full, used, rank, nv, nodes, rfParent,
               rfCounter, rfErr);
  }
  {
    // the bottom-up boxes (sm_builder.h:616-693), over the links written above
    ProfScope ps("refit", al.s);
    launch_pdl(k_refit_climb, dim3(div_up(numNodes, 128)), dim3(128), 0, al.s, nodes, numNodes, primIDs, n, boxes,
               rfParent, rfCounter, rfErr);
  }
  if ((ce = cudaGetLastError()) != cudaSuccess) {
    al.free_bytes(nodes);
    return fail(cuda_error(ce, "spatial median refit"));
  }
  bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
  bvh->numNodes = numNodes;
  bvh->primIDs = primIDs;
  bvh->numPrims = n;  // sm_builder.h:584: invalid prims stay listed after the valid ones
  return BQ_OK;
}

} // namespace bq
