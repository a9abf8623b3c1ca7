// bq_sah.cu -- binned SAH BVH builder (the cuBQL::cuda::sahBuilder method,
// also gpuBuilder with BuildConfig::SAH).
//
// Same splitting rule as sahBuilder_impl (cuBQL/builder/cuda/sah_builder.h:
// 22-538): a node with more than makeLeafThreshold prims bins its prims'
// centroids into 16 bins per axis over its centroid bounds (bin boxes are
// the union of the prim boxes, AtomicBox-encoded, empty = +-FLT_MAX);
// evaluateSAH (:61-104) compares the leaf cost area*count with every split
// lArea*lCount + rArea*rCount (surfaceArea = sx*sy + sx*sz + sy*sz) and
// takes the first strictly cheapest; prims whose bin along the split axis
// is >= the split bin go right.  Leaves list their prims in ascending
// primID order, as the reference's final (nodeID, primID) sort.
//
// Mechanics as the spatial-median builder (bq_sm.cu): prims live as 32-byte
// records (box, primID) in two buffers and are partitioned stably, so every
// node owns a contiguous range; children of the split at prim position m
// take slots 2m, 2m+1 and one scan compacts the slots at the end.
//   * nodes of more than warpMax prims (128..4096, about 64 subtrees per SM
//     below it) are split level by level over
//     the whole GPU in tiles of SAH_TILE prims: k_sah_bin (each warp bins
//     into its own shared-memory bins, the block merges them, writes the
//     tile's 48 bin counts and merges the bins into the node's with global
//     min/max/add atomics -- order-independent, so deterministic),
//     k_sah_decide (one warp per node evaluates the 48 candidates in
//     parallel), k_sah_tile_right (right count per tile from its bin
//     counts), one scan, k_sah_children, k_sah_scatter (stable scatter that
//     also reduces the children's centroid bounds), k_sah_classify;
//   * every subtree of at most warpMax prims is finished by one warp of a
//     persistent grid, depth first, smaller child first; a subtree of at
//     most 32 prims stays in registers (one prim per lane).
// The reference can make a leaf of more than 65535 prims (its 16-bit count
// then wraps); here such a node is split in two halves by position.
//
// Compiled twice: as itself (SAH) and, through bq_elh.cu with BQ_HEUR 1,
// as the edge-length-heuristic builder (8 bins, edge-length measure).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <vector>

#include "bq_internal.cuh"

namespace bq {
int refit(const bq_bvh3f *bvh, const bq_box3f *boxes, Alloc &al, bool check);

namespace {

// BQ_HEUR selects the heuristic of this translation unit: 0 = SAH (this
// file), 1 = ELH (bq_elh.cu includes this file with BQ_HEUR 1).
#ifndef BQ_HEUR
#define BQ_HEUR 0
#endif
constexpr int HEUR = BQ_HEUR;
constexpr int SAH_BINS = HEUR ? 8 : 16;      // bins per axis (SAHBins / ELHBins::numBins)
constexpr int SAH_NB = 3 * SAH_BINS;         // bins per node (3 axes)
constexpr int SAH_SEG = 32 / SAH_BINS;       // axes per warp pass in the evaluation
constexpr int SAH_PASSES = (3 + SAH_SEG - 1) / SAH_SEG;
constexpr int SAH_W = 7;                     // words per bin: lo[3], hi[3], count
constexpr uint32_t SAH_WARP_MIN = 128;       // warp subtrees: at most warpMax prims, warpMax in
constexpr uint32_t SAH_WARP_CAP = 4096;      // [SAH_WARP_MIN, SAH_WARP_CAP], about 64 tasks per SM
constexpr uint32_t SAH_TILE = 4096;          // prims per tile in the global levels
constexpr int SAH_BLOCK = 256;
constexpr int SAHW_BLOCK = 128;
constexpr int SAHW_WARPS = SAHW_BLOCK / 32;
constexpr int SAHW_STACK = 24;
constexpr int SAH_LEVELS_PER_CHECK = 2;
constexpr uint32_t SAH_MAX_LEAF = 65535;     // 16-bit leaf count

enum { DEC_LEAF = -1, DEC_HALVES = -2 };

struct __align__(16) SahPrim {
  float4 a;  // lower xyz, primID bits
  float4 b;  // upper xyz, unused
};

struct SahNode {
  uint32_t b, e, slot, parity;
  int32_t lo[3], hi[3];  // encoded centroid bounds
};
static_assert(sizeof(SahNode) == 40, "SahNode size");

struct SahDec {
  int dim;  // 0..2 split axis, DEC_LEAF, DEC_HALVES
  int bin;  // first bin of the right side
};

__device__ __forceinline__ float sah_ctr(float l, float h) { return __fmul_rn(0.5f, __fadd_rn(l, h)); }

// The cost measure of a box.  SAH: surfaceArea(box3f) (cuBQL/math/box.h:
// 198-205) with the contraction nvcc gives it in the reference's device
// code (pinned against its kernels).  ELH: edgeLengths (cuBQL/builder/
// cuda/elh_builder.h:66-76), a sum from 0 with no product to contract.
__device__ __forceinline__ float sah_area(float lx, float ly, float lz, float hx, float hy, float hz)
{
  const float sx = __fsub_rn(hx, lx), sy = __fsub_rn(hy, ly), sz = __fsub_rn(hz, lz);
  if (HEUR) return __fadd_rn(__fadd_rn(__fadd_rn(0.f, sx), sy), sz);
  return __fmaf_rn(sy, sz, __fmaf_rn(sx, sy, __fmul_rn(sx, sz)));
}

// binPrims (:170-180) / updatePrims (:300-306); ELH divides by hi - lo
// alone (elh_builder.h:213-217, 347-351)
__device__ __forceinline__ int sah_bin(float c, float lo, float hi)
{
  if (!(hi > lo)) return 0;
  const float den = HEUR ? __fsub_rn(hi, lo) : __fadd_rn(__fsub_rn(hi, lo), 1e-20f);
  const float rel = __fdiv_rn(__fsub_rn(c, lo), den);
  const int b = __float2int_rz(__fmul_rn(rel, (float)SAH_BINS));
  return max(0, min(SAH_BINS - 1, b));
}

__device__ __forceinline__ float prim_coord(const SahPrim &p, int d, bool upper)
{
  if (upper) return d == 0 ? p.b.x : (d == 1 ? p.b.y : p.b.z);
  return d == 0 ? p.a.x : (d == 1 ? p.a.y : p.a.z);
}

__device__ __forceinline__ float prim_ctr(const SahPrim &p, int d)
{
  return d == 0 ? sah_ctr(p.a.x, p.b.x) : (d == 1 ? sah_ctr(p.a.y, p.b.y) : sah_ctr(p.a.z, p.b.z));
}

__device__ __forceinline__ uint32_t side_of(const SahPrim &p, uint32_t rankInNode, uint32_t count, const SahDec &dec,
                                            float lo, float hi)
{
  if (dec.dim == DEC_HALVES) return rankInNode >= count / 2 ? 1u : 0u;
  return sah_bin(prim_ctr(p, dec.dim), lo, hi) >= dec.bin ? 1u : 0u;
}

__device__ __forceinline__ void bins_clear(int32_t *bins, int tid, int nthreads)
{
  for (int w = tid; w < SAH_NB * SAH_W; w += nthreads) {
    const int k = w % SAH_W;
    bins[w] = k < 3 ? enc_f(FLT_MAX) : (k < 6 ? enc_f(-FLT_MAX) : 0);
  }
}

// add one prim to shared or global bins (3 axes)
__device__ __forceinline__ void bins_add(int32_t *bins, const SahPrim &p, const float clo[3], const float chi[3])
{
  const int32_t e[6] = {enc_f(p.a.x), enc_f(p.a.y), enc_f(p.a.z), enc_f(p.b.x), enc_f(p.b.y), enc_f(p.b.z)};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int32_t *x = bins + (d * SAH_BINS + sah_bin(prim_ctr(p, d), clo[d], chi[d])) * SAH_W;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      atomicMin(x + k, e[k]);
      atomicMax(x + 3 + k, e[3 + k]);
    }
    atomicAdd(x + 6, 1);
  }
}

// evaluateSAH / evaluateELH by one warp over per-lane bins.  In pass p,
// lane L holds bin L % B of axis p * (32 / B) + L / B (B bins per axis;
// lanes of a missing fourth axis propose nothing): for SAH axes 0 and 1,
// then axis 2 (b*); for ELH all three axes in one pass.  Unions and counts
// by B-lane scans; the first strictly cheapest candidate in (axis, bin)
// order wins if it is cheaper than the leaf, as in the reference's serial
// loop.  Empty bins are (+FLT_MAX, -FLT_MAX), as AtomicBox leaves them.
__device__ __forceinline__ SahDec sah_evaluate_lanes(const float aLo[3], const float aHi[3], int aCnt,
                                                     const float bLo[3], const float bHi[3], int bCnt)
{
  const int lane = threadIdx.x & 31, b = lane % SAH_BINS;
  float leafCost = INFINITY;
  float best = INFINITY;
  int bestIdx = INT_MAX;
#pragma unroll
  for (int pass = 0; pass < SAH_PASSES; pass++) {
    float plo[3], phi[3], slo[3], shi[3];
    int pc = pass ? bCnt : aCnt, sc = pc;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      plo[k] = slo[k] = pass ? bLo[k] : aLo[k];
      phi[k] = shi[k] = pass ? bHi[k] : aHi[k];
    }
    // inclusive prefix (bins 0..b) and suffix (bins b..15) unions / counts
#pragma unroll
    for (int o = 1; o < SAH_BINS; o <<= 1) {
      const int pcu = __shfl_up_sync(0xffffffffu, pc, o, SAH_BINS);
      const int scd = __shfl_down_sync(0xffffffffu, sc, o, SAH_BINS);
      if (b >= o) pc += pcu;
      if (b + o < SAH_BINS) sc += scd;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const float a0 = __shfl_up_sync(0xffffffffu, plo[k], o, SAH_BINS);
        const float a1 = __shfl_up_sync(0xffffffffu, phi[k], o, SAH_BINS);
        const float a2 = __shfl_down_sync(0xffffffffu, slo[k], o, SAH_BINS);
        const float a3 = __shfl_down_sync(0xffffffffu, shi[k], o, SAH_BINS);
        if (b >= o) { plo[k] = fminf(plo[k], a0); phi[k] = fmaxf(phi[k], a1); }
        if (b + o < SAH_BINS) { slo[k] = fminf(slo[k], a2); shi[k] = fmaxf(shi[k], a3); }
      }
    }
    // exclusive prefix: the union of bins 0..b-1 (b == 0: the empty box)
    float elo[3], ehi[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float a0 = __shfl_up_sync(0xffffffffu, plo[k], 1, SAH_BINS);
      const float a1 = __shfl_up_sync(0xffffffffu, phi[k], 1, SAH_BINS);
      elo[k] = b > 0 ? a0 : INFINITY;
      ehi[k] = b > 0 ? a1 : -INFINITY;
    }
    const int pcu = __shfl_up_sync(0xffffffffu, pc, 1, SAH_BINS);
    const int lCount = b > 0 ? pcu : 0;
    const int rCount = sc;
    const float rArea = sah_area(slo[0], slo[1], slo[2], shi[0], shi[1], shi[2]);
    const float lArea = sah_area(elo[0], elo[1], elo[2], ehi[0], ehi[1], ehi[2]);
    if (pass == 0) leafCost = __shfl_sync(0xffffffffu, __fmul_rn(rArea, (float)rCount), 0);  // rAreas[0]*rCount
    const int dim = pass * SAH_SEG + lane / SAH_BINS;
    float cost = INFINITY;
    if (lCount > 0 && rCount > 0 && dim < 3) {
      cost = __fmaf_rn(lArea, (float)lCount, __fmul_rn(rArea, (float)rCount));
      if (cost != cost) cost = INFINITY;  // NaN never wins (cost < best is false)
    }
    const int idx = dim * SAH_BINS + b;
    if (cost < best || (cost == best && cost != INFINITY && idx < bestIdx)) {
      best = cost;
      bestIdx = idx;
    }
  }
  // warp arg-min, first index among equal costs
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bestIdx, o);
    if (ob < best || (ob == best && oi < bestIdx)) {
      best = ob;
      bestIdx = oi;
    }
  }
  // the reference starts from the leaf cost when that is below +inf
  const float start = leafCost < INFINITY ? leafCost : INFINITY;
  SahDec dec;
  if (bestIdx != INT_MAX && best < start) {
    dec.dim = bestIdx / SAH_BINS;
    dec.bin = bestIdx % SAH_BINS;
  } else {
    dec.dim = DEC_LEAF;
    dec.bin = 0;
  }
  return dec;
}

// evaluation over 3*B encoded bins (bins[(d*B+b)*7 + ...], shared or global)
__device__ __forceinline__ SahDec sah_evaluate(const int32_t *bins)
{
  const int lane = threadIdx.x & 31, b = lane % SAH_BINS;
  const int da = lane / SAH_BINS, db = SAH_SEG + lane / SAH_BINS;  // axes of passes 0 and 1
  float aLo[3], aHi[3], bLo[3], bHi[3];
  int aCnt = 0, bCnt = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) { aLo[k] = bLo[k] = FLT_MAX; aHi[k] = bHi[k] = -FLT_MAX; }
  if (da < 3) {
    const int32_t *xa = bins + (da * SAH_BINS + b) * SAH_W;
#pragma unroll
    for (int k = 0; k < 3; k++) { aLo[k] = dec_f(xa[k]); aHi[k] = dec_f(xa[3 + k]); }
    aCnt = xa[6];
  }
  if (SAH_PASSES > 1 && db < 3) {
    const int32_t *xb = bins + (db * SAH_BINS + b) * SAH_W;
#pragma unroll
    for (int k = 0; k < 3; k++) { bLo[k] = dec_f(xb[k]); bHi[k] = dec_f(xb[3 + k]); }
    bCnt = xb[6];
  }
  return sah_evaluate_lanes(aLo, aHi, aCnt, bLo, bHi, bCnt);
}

// running encoded min/max of the two children's centroids
struct SideBounds {
  int32_t lo0[3], hi0[3], lo1[3], hi1[3];
  __device__ __forceinline__ void init()
  {
#pragma unroll
    for (int d = 0; d < 3; d++) { lo0[d] = lo1[d] = INT_MAX; hi0[d] = hi1[d] = INT_MIN; }
  }
  __device__ __forceinline__ void add(const SahPrim &p, uint32_t side)
  {
    const int32_t e[3] = {enc_f(sah_ctr(p.a.x, p.b.x)), enc_f(sah_ctr(p.a.y, p.b.y)), enc_f(sah_ctr(p.a.z, p.b.z))};
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

__device__ __forceinline__ void leaf_node(Node *out, uint32_t slot, uint32_t b, uint32_t count)
{
  out[slot] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(b, count));
}

__device__ __forceinline__ void child_pair(const SahNode &nd, uint32_t m, const SideBounds &sb, SahNode &c0,
                                           SahNode &c1)
{
  c0.b = nd.b; c0.e = m; c0.slot = 2 * m; c0.parity = nd.parity ^ 1u;
  c1.b = m; c1.e = nd.e; c1.slot = 2 * m + 1; c1.parity = nd.parity ^ 1u;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    c0.lo[d] = sb.lo0[d]; c0.hi[d] = sb.hi0[d];
    c1.lo[d] = sb.lo1[d]; c1.hi[d] = sb.hi1[d];
  }
}

__device__ __forceinline__ void node_bounds(const SahNode &nd, float lo[3], float hi[3])
{
#pragma unroll
  for (int d = 0; d < 3; d++) { lo[d] = dec_f(nd.lo[d]); hi[d] = dec_f(nd.hi[d]); }
}

// ------------------------------------------------------------------
// set-up: valid prims compacted (primID order) as records, invalid ones
// listed after them in primIDs, root centroid bounds
// ------------------------------------------------------------------
__global__ void k_sah_valid(const bq_box3f *__restrict__ boxes, uint32_t n, uint32_t *__restrict__ valid)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  valid[i] = (boxes[i].lower[0] <= boxes[i].upper[0]) ? 1u : 0u;  // initPrims (:139)
}

__global__ void __launch_bounds__(256) k_sah_init(const bq_box3f *__restrict__ boxes, uint32_t n,
                                                  const uint32_t *__restrict__ vpos, const uint32_t *nvPtr,
                                                  SahPrim *__restrict__ recs, uint32_t *__restrict__ primIDs,
                                                  int32_t *rootLoHi)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  int32_t lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const bq_box3f b = boxes[i];
    const uint32_t p = vpos[i];
    if (b.lower[0] <= b.upper[0]) {
      SahPrim r;
      r.a = make_float4(b.lower[0], b.lower[1], b.lower[2], __uint_as_float((uint32_t)i));
      r.b = make_float4(b.upper[0], b.upper[1], b.upper[2], 0.f);
      recs[p] = r;
      const int32_t e[3] = {enc_f(sah_ctr(b.lower[0], b.upper[0])), enc_f(sah_ctr(b.lower[1], b.upper[1])),
                            enc_f(sah_ctr(b.lower[2], b.upper[2]))};
#pragma unroll
      for (int d = 0; d < 3; d++) { lo[d] = min(lo[d], e[d]); hi[d] = max(hi[d], e[d]); }
    } else {
      primIDs[nv + ((uint32_t)i - p)] = (uint32_t)i;
    }
  }
  block_merge_bounds<256>(lo, hi, rootLoHi);
}

// ------------------------------------------------------------------
// global levels (nodes with more than warpMax prims)
// ------------------------------------------------------------------
struct SahCtl {
  uint32_t bigCount[2];
  uint32_t numTiles;
  uint32_t scanLen;
  uint32_t taskCount;
  uint32_t grab;
  uint32_t err;
  uint32_t pad;
};

struct TileInfo {
  uint32_t node, begin, end;
};
__device__ __forceinline__ uint32_t first_end(const uint32_t *__restrict__ first, uint32_t K, uint32_t T, uint32_t k)
{
  return k + 1 < K ? first[k + 1] : T;
}
__device__ __forceinline__ TileInfo tile_info(const SahNode *__restrict__ nodes, const uint32_t *__restrict__ first,
                                              uint32_t K, uint32_t t)
{
  uint32_t lo = 0, hi = K;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (first[m] <= t) lo = m; else hi = m;
  }
  TileInfo r;
  r.node = lo;
  r.begin = nodes[lo].b + (t - first[lo]) * SAH_TILE;
  r.end = min(nodes[lo].e, r.begin + SAH_TILE);
  return r;
}

// tiles per big node; clears the node's global bins
__global__ void k_sah_tiles(const SahNode *__restrict__ nodes, SahCtl *ctl, int cur, uint32_t cap,
                            uint32_t *__restrict__ tileCount, int32_t *__restrict__ nodeBins)
{
  griddep_wait();
  const uint32_t K = ctl->bigCount[cur];
  const uint32_t k = blockIdx.x;
  if (k == 0 && threadIdx.x == 0 && K > cap) atomicOr(&ctl->err, DEV_ERR_RANGE);
  if (k >= K || k >= cap) return;
  bins_clear(nodeBins + (size_t)k * SAH_NB * SAH_W, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) tileCount[k] = (nodes[k].e - nodes[k].b + SAH_TILE - 1) / SAH_TILE;
}

// per tile: per-warp shared bins, merged per block; the tile's 48 counts
// to tileCnt, the bins into the node's with global atomics
__global__ void __launch_bounds__(SAH_BLOCK) k_sah_bin(const SahNode *__restrict__ nodes,
                                                       const uint32_t *__restrict__ first, SahCtl *ctl, int cur,
                                                       uint32_t maxTiles, const SahPrim *__restrict__ buf0,
                                                       const SahPrim *__restrict__ buf1,
                                                       uint32_t *__restrict__ tileCnt, int32_t *__restrict__ nodeBins)
{
  griddep_wait();
  constexpr int WARPS = SAH_BLOCK / 32;
  __shared__ int32_t sBins[WARPS][SAH_NB * SAH_W];
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  if (blockIdx.x >= T || blockIdx.x >= maxTiles - 1) return;  // whole block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  bins_clear(sBins[warp], lane, 32);
  __syncwarp();
  const TileInfo t = tile_info(nodes, first, K, blockIdx.x);
  const SahNode nd = nodes[t.node];
  float clo[3], chi[3];
  node_bounds(nd, clo, chi);
  const SahPrim *src = nd.parity ? buf1 : buf0;
  for (uint32_t i = t.begin + threadIdx.x; i < t.end; i += SAH_BLOCK) bins_add(sBins[warp], src[i], clo, chi);
  __syncthreads();
  int32_t *nb = nodeBins + (size_t)t.node * SAH_NB * SAH_W;
  for (int w = threadIdx.x; w < SAH_NB * SAH_W; w += SAH_BLOCK) {
    const int k = w % SAH_W;
    int32_t v = sBins[0][w];
    for (int j = 1; j < WARPS; j++) {
      const int32_t x = sBins[j][w];
      v = k < 3 ? min(v, x) : (k < 6 ? max(v, x) : v + x);
    }
    if (k == 6) {
      tileCnt[(size_t)blockIdx.x * SAH_NB + w / SAH_W] = (uint32_t)v;
      if (v) atomicAdd(nb + w, v);
    } else if (k < 3) {
      if (v != enc_f(FLT_MAX)) atomicMin(nb + w, v);
    } else {
      if (v != enc_f(-FLT_MAX)) atomicMax(nb + w, v);
    }
  }
}

// one warp per big node: the split decision; a leaf writes its node and
// its final primIDs
__global__ void k_sah_decide(const SahNode *__restrict__ nodes, const SahCtl *ctl, int cur, uint32_t cap, int thr,
                             const int32_t *__restrict__ nodeBins, SahDec *__restrict__ decs,
                             const SahPrim *__restrict__ buf0, const SahPrim *__restrict__ buf1,
                             Node *__restrict__ out, uint32_t *__restrict__ primIDs)
{
  griddep_wait();
  const uint32_t K = min(ctl->bigCount[cur], cap);
  const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= K) return;  // whole warp
  const SahNode nd = nodes[k];
  const uint32_t count = nd.e - nd.b;
  SahDec dec;
  if ((int64_t)count > thr) {
    dec = sah_evaluate(nodeBins + (size_t)k * SAH_NB * SAH_W);
  } else {
    dec.dim = DEC_LEAF;
    dec.bin = 0;
  }
  if (dec.dim == DEC_LEAF && count > SAH_MAX_LEAF) dec.dim = DEC_HALVES;
  if (dec.dim == DEC_LEAF) {
    const SahPrim *src = nd.parity ? buf1 : buf0;
    for (uint32_t i = nd.b + lane; i < nd.e; i += 32) primIDs[i] = __float_as_uint(src[i].a.w);
    if (lane == 0) leaf_node(out, nd.slot, nd.b, count);
  }
  if (lane == 0) decs[k] = dec;
}

// the scan of the level's tile counts in one block (at most
// BQ_SCAN_SMEM_MAX nodes, counted in shared memory)
__global__ void __launch_bounds__(BQ_SCAN_THREADS) k_sah_tiles_scan(SahCtl *ctl, int cur, uint32_t cap,
                                                                    uint32_t maxTiles,
                                                                    const uint32_t *__restrict__ tileCount,
                                                                    uint32_t *__restrict__ first)
{
  griddep_wait();
  extern __shared__ uint32_t sVal[];  // cap entries
  __shared__ uint32_t sWarp[33];
  const uint32_t K = min(ctl->bigCount[cur], cap);
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) sVal[k] = tileCount[k];
  __syncthreads();
  const uint32_t T = block_scan_smem(sVal, K, sWarp);
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) first[k] = sVal[k];
  if (threadIdx.x == 0) {
    if (T >= maxTiles) atomicOr(&ctl->err, DEV_ERR_RANGE);
    ctl->numTiles = min(T, maxTiles - 1);
  }
}

// right-side count of a tile from its bin counts
__device__ __forceinline__ uint32_t sah_tile_right(const SahNode *__restrict__ nodes, const uint32_t *__restrict__ first,
                                                   uint32_t K, uint32_t t, const SahDec *__restrict__ decs,
                                                   const uint32_t *__restrict__ tileCnt)
{
  const TileInfo ti = tile_info(nodes, first, K, t);
  const SahDec dec = decs[ti.node];
  uint32_t r = 0;
  if (dec.dim >= 0) {
    for (int b = dec.bin; b < SAH_BINS; b++) r += tileCnt[(size_t)t * SAH_NB + dec.dim * SAH_BINS + b];
  } else if (dec.dim == DEC_HALVES) {
    const SahNode nd = nodes[ti.node];
    const uint32_t half = nd.b + (nd.e - nd.b) / 2;  // positions >= half go right
    r = ti.end > max(ti.begin, half) ? ti.end - max(ti.begin, half) : 0u;
  }
  return r;
}

// per split node: the split position, the internal node, the two child
// records (bounds start empty); leaves get an empty pair
__device__ __forceinline__ void sah_node_children(const SahNode *__restrict__ nodes, uint32_t K, uint32_t T, uint32_t k,
                                                  const uint32_t *__restrict__ first, const uint32_t *rightScan,
                                                  const SahDec *__restrict__ decs, Node *__restrict__ out,
                                                  uint32_t *__restrict__ used, SahNode *__restrict__ next,
                                                  uint32_t *err)
{
  const SahNode nd = nodes[k];
  SahNode c0, c1;
  if (decs[k].dim == DEC_LEAF) {
    c0.b = c0.e = c1.b = c1.e = 0;
    next[2 * k] = c0;
    next[2 * k + 1] = c1;
    return;
  }
  const uint32_t nR = rightScan[first_end(first, K, T, k)] - rightScan[first[k]];
  const uint32_t m = nd.e - nR;
  if (nR == 0 || m == nd.b) atomicOr(err, DEV_ERR_RANGE);  // a chosen split always has both sides
  internal_node(out, used, nd.slot, m);
  SideBounds sb;
  sb.init();
  child_pair(nd, m, sb, c0, c1);
  next[2 * k] = c0;
  next[2 * k + 1] = c1;
}

// k_sah_tile_right, the scan of its counts and k_sah_children in one block
// (numTiles + 1 <= BQ_SCAN_SMEM_MAX entries in shared memory)
__global__ void __launch_bounds__(BQ_SCAN_THREADS) k_sah_right_children(const SahNode *__restrict__ nodes,
                                                                        const uint32_t *__restrict__ first,
                                                                        SahCtl *ctl, int cur, uint32_t cap,
                                                                        const SahDec *__restrict__ decs,
                                                                        const uint32_t *__restrict__ tileCnt,
                                                                        uint32_t *__restrict__ tileRight,
                                                                        Node *__restrict__ out,
                                                                        uint32_t *__restrict__ used,
                                                                        SahNode *__restrict__ next)
{
  griddep_wait();
  extern __shared__ uint32_t sScan[];  // numTiles + 1 entries
  __shared__ uint32_t sWarp[33];
  const uint32_t K = min(ctl->bigCount[cur], cap), T = ctl->numTiles;
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) sScan[t] = sah_tile_right(nodes, first, K, t, decs, tileCnt);
  __syncthreads();
  const uint32_t total = block_scan_smem(sScan, T, sWarp);
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) tileRight[t] = sScan[t];
  if (threadIdx.x == 0) {
    tileRight[T] = total;
    sScan[T] = total;
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
    sah_node_children(nodes, K, T, k, first, sScan, decs, out, used, next, &ctl->err);
}

// right-side count of every tile from its bin counts
__global__ void k_sah_tile_right(const SahNode *__restrict__ nodes, const uint32_t *__restrict__ first, SahCtl *ctl,
                                 int cur, uint32_t maxTiles, const SahDec *__restrict__ decs,
                                 const uint32_t *__restrict__ tileCnt, uint32_t *__restrict__ tileRight)
{
  griddep_wait();
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    if (T >= maxTiles) atomicOr(&ctl->err, DEV_ERR_RANGE);
    else tileRight[T] = 0;
    ctl->scanLen = min(T, maxTiles - 1) + 1;
  }
  if (t >= T || t >= maxTiles - 1) return;
  tileRight[t] = sah_tile_right(nodes, first, K, t, decs, tileCnt);
}

// sah_node_children for every big node of the level
__global__ void k_sah_children(const SahNode *__restrict__ nodes, const SahCtl *ctl, int cur, uint32_t cap,
                               const uint32_t *__restrict__ first, const uint32_t *__restrict__ rightScan,
                               const SahDec *__restrict__ decs, Node *__restrict__ out, uint32_t *__restrict__ used,
                               SahNode *__restrict__ next, uint32_t *err)
{
  griddep_wait();
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K || k >= cap) return;
  sah_node_children(nodes, K, T, k, first, rightScan, decs, out, used, next, err);
}

__global__ void __launch_bounds__(SAH_BLOCK) k_sah_scatter(const SahNode *__restrict__ nodes,
                                                           const uint32_t *__restrict__ first, const SahCtl *ctl,
                                                           int cur, uint32_t maxTiles,
                                                           const uint32_t *__restrict__ rightScan,
                                                           const SahDec *__restrict__ decs, SahPrim *buf0,
                                                           SahPrim *buf1, SahNode *next)
{
  griddep_wait();
  __shared__ uint32_t sWarp[SAH_BLOCK / 32];
  __shared__ int32_t sRed[12][SAH_BLOCK / 32];
  const uint32_t K = ctl->bigCount[cur], T = ctl->numTiles;
  if (blockIdx.x >= T || blockIdx.x >= maxTiles - 1) return;  // whole block
  const TileInfo t = tile_info(nodes, first, K, blockIdx.x);
  const SahDec dec = decs[t.node];
  if (dec.dim == DEC_LEAF) return;  // whole block
  const SahNode nd = nodes[t.node];
  const uint32_t count = nd.e - nd.b;
  const float lo = dec.dim >= 0 ? dec_f(nd.lo[dec.dim]) : 0.f, hi = dec.dim >= 0 ? dec_f(nd.hi[dec.dim]) : 0.f;
  const SahPrim *src = nd.parity ? buf1 : buf0;
  SahPrim *dst = nd.parity ? buf0 : buf1;
  const uint32_t nodeRight0 = rightScan[first[t.node]];
  const uint32_t m = nd.e - (rightScan[first_end(first, K, T, t.node)] - nodeRight0);
  uint32_t rBefore = rightScan[blockIdx.x] - nodeRight0;
  uint32_t lBefore = (t.begin - nd.b) - rBefore;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  SideBounds sb;
  sb.init();
  for (uint32_t base = t.begin; base < t.end; base += SAH_BLOCK) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < t.end;
    SahPrim p;
    uint32_t side = 0;
    if (valid) {
      p = src[i];
      side = side_of(p, i - nd.b, count, dec, lo, hi);
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, valid && side);
    if (lane == 0) sWarp[warp] = __popc(bal);
    __syncthreads();
    uint32_t rw = 0, rtot = 0;
#pragma unroll
    for (int w = 0; w < SAH_BLOCK / 32; w++) {
      const uint32_t x = sWarp[w];
      rw += (w < warp) ? x : 0u;
      rtot += x;
    }
    if (valid) {
      const uint32_t rMine = rw + __popc(bal & lt);
      dst[side ? m + rBefore + rMine : nd.b + lBefore + (threadIdx.x - rMine)] = p;
      sb.add(p, side);
    }
    const uint32_t chunk = min((uint32_t)SAH_BLOCK, t.end - base);
    rBefore += rtot;
    lBefore += chunk - rtot;
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
    for (int w = 0; w < SAH_BLOCK / 32; w++) v = isMin ? min(v, sRed[j][w]) : max(v, sRed[j][w]);
    SahNode *child = next + 2 * t.node + (j / 6);
    if (isMin) {
      if (v != INT_MAX) atomicMin(&child->lo[comp], v);
    } else {
      if (v != INT_MIN) atomicMax(&child->hi[comp - 3], v);
    }
  }
}

// ------------------------------------------------------------------
// warp phase: whole subtrees of at most warpMax prims
// ------------------------------------------------------------------
// A subtree of at most 32 prims: lane j holds the prim at position
// root.b + j in registers for the whole subtree.  A node's bins are
// gathered by broadcasting its prims to the lanes that own the bins (no
// shared atomics); partitions go through the 32-entry exchange buffer.
__device__ void sah_small_subtree(const SahNode &root, const SahPrim *src, int thr, SahPrim *xbuf, SahNode *stk,
                                  int stackLeft, Node *__restrict__ out, uint32_t *__restrict__ primIDs,
                                  uint32_t *__restrict__ used, uint32_t *err)
{
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t base = root.b, cnt = root.e - root.b;
  SahPrim p;
  if (lane < (int)cnt) p = src[base + lane];
  else p.a = p.b = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint32_t pos = base + lane;
  const int dimA = lane / SAH_BINS, dimB = SAH_SEG + lane / SAH_BINS, binL = lane % SAH_BINS;
  SahNode cur = root;
  int sp = 0;
  while (true) {
    const uint32_t count = cur.e - cur.b;
    const bool in = pos >= cur.b && pos < cur.e;
    float clo[3], chi[3];
    node_bounds(cur, clo, chi);
    int mb[3] = {0, 0, 0};
    if (in) {
#pragma unroll
      for (int d = 0; d < 3; d++) mb[d] = sah_bin(prim_ctr(p, d), clo[d], chi[d]);
    }
    SahDec dec;
    dec.dim = DEC_LEAF;
    dec.bin = 0;
    if ((int64_t)count > thr && count > 1) {  // one prim cannot be split: a leaf
      float aLo[3], aHi[3], bLo[3], bHi[3];
#pragma unroll
      for (int k = 0; k < 3; k++) { aLo[k] = bLo[k] = FLT_MAX; aHi[k] = bHi[k] = -FLT_MAX; }
      int aCnt = 0, bCnt = 0;
      for (uint32_t j = cur.b - base; j < cur.e - base; j++) {
        const float l0 = __shfl_sync(0xffffffffu, p.a.x, j), l1 = __shfl_sync(0xffffffffu, p.a.y, j);
        const float l2 = __shfl_sync(0xffffffffu, p.a.z, j), h0 = __shfl_sync(0xffffffffu, p.b.x, j);
        const float h1 = __shfl_sync(0xffffffffu, p.b.y, j), h2 = __shfl_sync(0xffffffffu, p.b.z, j);
        const int j0 = __shfl_sync(0xffffffffu, mb[0], j), j1 = __shfl_sync(0xffffffffu, mb[1], j);
        const int j2 = __shfl_sync(0xffffffffu, mb[2], j);
        const int ja = dimA == 0 ? j0 : (dimA == 1 ? j1 : (dimA == 2 ? j2 : -1));
        const int jb = dimB == 0 ? j0 : (dimB == 1 ? j1 : (dimB == 2 ? j2 : -1));
        if (ja == binL) {
          aLo[0] = fminf(aLo[0], l0); aLo[1] = fminf(aLo[1], l1); aLo[2] = fminf(aLo[2], l2);
          aHi[0] = fmaxf(aHi[0], h0); aHi[1] = fmaxf(aHi[1], h1); aHi[2] = fmaxf(aHi[2], h2);
          aCnt++;
        }
        if (SAH_PASSES > 1 && jb == binL) {
          bLo[0] = fminf(bLo[0], l0); bLo[1] = fminf(bLo[1], l1); bLo[2] = fminf(bLo[2], l2);
          bHi[0] = fmaxf(bHi[0], h0); bHi[1] = fmaxf(bHi[1], h1); bHi[2] = fmaxf(bHi[2], h2);
          bCnt++;
        }
      }
      dec = sah_evaluate_lanes(aLo, aHi, aCnt, bLo, bHi, bCnt);
    }
    if (dec.dim == DEC_LEAF) {
      if (lane == 0) leaf_node(out, cur.slot, cur.b, count);
      if (sp == 0) break;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    const int myBin = dec.dim == 0 ? mb[0] : (dec.dim == 1 ? mb[1] : mb[2]);
    const uint32_t side = in ? (myBin >= dec.bin ? 1u : 0u) : 0u;
    const uint32_t balR = __ballot_sync(0xffffffffu, in && side);
    const uint32_t balL = __ballot_sync(0xffffffffu, in && !side);
    const uint32_t m = cur.e - __popc(balR);
    if (balR == 0 || balL == 0) {  // unreachable: a chosen split has prims on both sides
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      break;
    }
    // a child of at most thr prims, or of one, is a leaf: written here, never
    // evaluated, so its bounds are not needed
    const uint32_t nL = m - cur.b, nR = cur.e - m;
    const bool leafL = (int64_t)nL <= thr || nL == 1, leafR = (int64_t)nR <= thr || nR == 1;
    SideBounds sb;
    sb.init();
    if (!(leafL && leafR)) {
      if (in) sb.add(p, side);
      sb.warp_reduce();
    }
    const uint32_t dest = !in ? (uint32_t)lane
                              : (side ? (m - base) + __popc(balR & lt) : (cur.b - base) + __popc(balL & lt));
    xbuf[dest] = p;
    __syncwarp();
    p = xbuf[lane];
    __syncwarp();
    SahNode c0, c1;
    child_pair(cur, m, sb, c0, c1);
    if (lane == 0) {
      internal_node(out, used, cur.slot, m);
      if (leafL) leaf_node(out, c0.slot, c0.b, nL);
      if (leafR) leaf_node(out, c1.slot, c1.b, nR);
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
    const bool leftSmaller = nL <= nR;
    if (sp >= stackLeft) {  // unreachable: the stacked child is always the larger one
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      break;
    }
    if (lane == 0) stk[sp] = leftSmaller ? c1 : c0;
    sp++;
    cur = leftSmaller ? c0 : c1;
  }
  if (lane < (int)cnt) primIDs[base + lane] = __float_as_uint(p.a.w);
  __syncwarp();
}

__device__ void sah_warp_task(SahNode cur, int thr, SahPrim *buf0, SahPrim *buf1, Node *__restrict__ out,
                              uint32_t *__restrict__ primIDs, uint32_t *__restrict__ used, uint32_t *err,
                              SahNode *stk, int32_t *bins, SahPrim *xbuf)
{
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  int sp = 0;
  while (true) {
    const uint32_t count = cur.e - cur.b;
    const SahPrim *src = cur.parity ? buf1 : buf0;
    SahPrim *dst = cur.parity ? buf0 : buf1;
    if ((int64_t)count > thr && count <= 32) {
      sah_small_subtree(cur, src, thr, xbuf, stk + sp, SAHW_STACK - sp, out, primIDs, used, err);
      if (sp == 0) return;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    SahDec dec;
    dec.dim = DEC_LEAF;
    dec.bin = 0;
    float clo[3], chi[3];
    node_bounds(cur, clo, chi);
    if ((int64_t)count > thr) {
      bins_clear(bins, lane, 32);
      __syncwarp();
      for (uint32_t i = cur.b + lane; i < cur.e; i += 32) bins_add(bins, src[i], clo, chi);
      __syncwarp();
      dec = sah_evaluate(bins);
      __syncwarp();  // bins are read before the next node clears them
    }
    if (dec.dim == DEC_LEAF) {  // counts here are at most max(warpMax, thr) <= 65535
      for (uint32_t i = cur.b + lane; i < cur.e; i += 32) primIDs[i] = __float_as_uint(src[i].a.w);
      if (lane == 0) leaf_node(out, cur.slot, cur.b, count);
      if (sp == 0) return;
      __syncwarp();
      cur = stk[--sp];
      __syncwarp();
      continue;
    }
    const float lo = clo[dec.dim], hi = chi[dec.dim];
    // pass 1: right-side count
    uint32_t nR = 0;
    for (uint32_t i = cur.b + lane; i < cur.e; i += 32) nR += side_of(src[i], i - cur.b, count, dec, lo, hi);
    nR = __reduce_add_sync(0xffffffffu, nR);
    const uint32_t m = cur.e - nR;
    if (nR == 0 || m == cur.b) {  // unreachable: a chosen split has prims on both sides
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      return;
    }
    // pass 2: stable scatter + children's centroid bounds
    uint32_t lB = 0, rB = 0;
    SideBounds sb;
    sb.init();
    for (uint32_t base = cur.b; base < cur.e; base += 32) {
      const uint32_t i = base + lane;
      const bool valid = i < cur.e;
      SahPrim p;
      uint32_t sd = 0;
      if (valid) {
        p = src[i];
        sd = side_of(p, i - cur.b, count, dec, lo, hi);
      }
      const uint32_t balR = __ballot_sync(0xffffffffu, valid && sd);
      const uint32_t balL = __ballot_sync(0xffffffffu, valid && !sd);
      if (valid) {
        dst[sd ? m + rB + __popc(balR & lt) : cur.b + lB + __popc(balL & lt)] = p;
        sb.add(p, sd);
      }
      rB += __popc(balR);
      lB += __popc(balL);
    }
    sb.warp_reduce();
    if (lane == 0) internal_node(out, used, cur.slot, m);
    SahNode c0, c1;
    child_pair(cur, m, sb, c0, c1);
    const bool leftSmaller = (m - cur.b) <= (cur.e - m);
    if (sp >= SAHW_STACK) {  // unreachable: the stacked child is always the larger one
      if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
      return;
    }
    if (lane == 0) stk[sp] = leftSmaller ? c1 : c0;
    sp++;
    cur = leftSmaller ? c0 : c1;
    __syncwarp();  // this warp's scatter is visible to its own next pass
  }
}

__global__ void __launch_bounds__(SAHW_BLOCK) k_sah_warp(const SahNode *__restrict__ tasks, SahCtl *ctl,
                                                         uint32_t taskCap, int thr, SahPrim *buf0, SahPrim *buf1,
                                                         Node *__restrict__ out, uint32_t *__restrict__ primIDs,
                                                         uint32_t *__restrict__ used)
{
  griddep_wait();
  __shared__ SahNode sStack[SAHW_WARPS][SAHW_STACK];
  __shared__ int32_t sBins[SAHW_WARPS][SAH_NB * SAH_W];
  __shared__ SahPrim sX[SAHW_WARPS][32];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const uint32_t numTasks = min(ctl->taskCount, taskCap);
  while (true) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&ctl->grab, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= numTasks) return;  // whole warp
    sah_warp_task(tasks[t], thr, buf0, buf1, out, primIDs, used, &ctl->err, sStack[wb], sBins[wb], sX[wb]);
    __syncwarp();
  }
}

// children of the level's split nodes: to the next big list or to the tasks
__global__ void k_sah_classify(const SahNode *__restrict__ next, SahCtl *ctl, int cur, uint32_t cap, int thr,
                               uint32_t warpMax, SahNode *__restrict__ bigNext, SahNode *__restrict__ tasks,
                               uint32_t taskCap)
{
  griddep_wait();
  const uint32_t K = min(ctl->bigCount[cur], cap);
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 2 * K) return;
  const SahNode c = next[j];
  const uint32_t size = c.e - c.b;
  if (size == 0) return;  // the node became a leaf
  if (size > warpMax && (int64_t)size > thr) {
    const uint32_t at = atomicAdd(&ctl->bigCount[cur ^ 1], 1u);
    if (at < cap) bigNext[at] = c;
    else atomicOr(&ctl->err, DEV_ERR_RANGE);
  } else {
    const uint32_t at = atomicAdd(&ctl->taskCount, 1u);
    if (at < taskCap) tasks[at] = c;
    else atomicOr(&ctl->err, DEV_ERR_RANGE);
  }
}

// ------------------------------------------------------------------
// slot compaction: split m's children move from 2m, 2m+1 to 2+2*rank[m]
// ------------------------------------------------------------------
__device__ __forceinline__ Node sah_remap(const Node &c, const uint32_t *__restrict__ rank)
{
  const uint64_t a = node_admin(c);
  if (admin_count(a)) return c;
  const uint32_t cm = (uint32_t)(admin_offset(a) >> 1);
  return make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(2ull + 2ull * rank[cm], 0));
}

__global__ void k_sah_compact(const Node *__restrict__ full, const uint32_t *__restrict__ used,
                              const uint32_t *__restrict__ rank, uint32_t nv, Node *__restrict__ out)
{
  griddep_wait();
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) {
    out[0] = sah_remap(full[0], rank);
    out[1] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0);
    return;
  }
  if (m >= nv || !used[m]) return;
  const uint64_t pair = 2ull + 2ull * rank[m];
  out[pair] = sah_remap(full[2ull * m], rank);
  out[pair + 1] = sah_remap(full[2ull * m + 1], rank);
}

} // namespace
} // namespace bq

namespace bq {

#if BQ_HEUR == 0
int build_sah(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
#else
int build_elh(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
#endif
{
  const int thr = cfg ? cfg->makeLeafThreshold : 0;  // 0 and 1 build the same tree
  if (thr < 0 || thr > 65535)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "makeLeafThreshold must be in [0, 65535] (16-bit leaf count)");
  bvh->nodes = nullptr; bvh->primIDs = nullptr; bvh->numNodes = 0; bvh->numPrims = 0;
  if (n == 0) return BQ_OK;

  TempSet tmp(al);
  uint32_t *valid = nullptr, *vpos = nullptr, *ctl = nullptr, *used = nullptr;
  SahPrim *buf0 = nullptr, *buf1 = nullptr;
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
    return fail(cuda_error(ce, "sah set-up"));
  {
    ProfScope ps(HEUR ? "elh.setup" : "sah.setup", al.s, 5);
    launch_pdl(k_sah_valid, dim3(div_up(n, 256)), dim3(256), 0, al.s, boxes, n, valid);
    if ((s = exclusive_scan_u32(valid, vpos, n, nullptr, ctl, al)) != BQ_OK) return fail(s);
    launch_pdl(k_sah_init, dim3(std::min(div_up(n, 256), num_sms() * 8)), dim3(256), 0, al.s, boxes, n, vpos, ctl,
               buf0, primIDs, (int32_t *)(ctl + 2));
  }
  int32_t hctl[8];
  if ((ce = cudaMemcpyAsync(hctl, ctl, 32, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "sah set-up"));
  const uint32_t nv = (uint32_t)hctl[0];
  if (nv == 0) {
    al.free_bytes(primIDs);
    return BQ_OK;
  }
  Node *full = nullptr;
  if ((s = tmp.get(&full, 2ull * nv)) != BQ_OK) return fail(s);

  // ---- global levels, driven from device memory (as the spatial-median
  // builder: big nodes of a level are disjoint, so at most cap of them and
  // maxTiles tiles; the host looks at the counters every few levels) ----
  // warp subtrees small enough for about 64 of them per SM, so the warp
  // phase has work for every warp
  uint32_t warpMax = SAH_WARP_MIN;
  while (warpMax < SAH_WARP_CAP && (uint64_t)warpMax * 2 * num_sms() * 64 <= nv) warpMax *= 2;
  const uint32_t cap = nv / (warpMax + 1) + 1;
  const uint32_t maxTiles = nv / SAH_TILE + cap + 2;
  int nextCheck = 1;
  while (nextCheck < 62 && ((uint64_t)warpMax << nextCheck) < nv) nextCheck++;
  const uint32_t taskCap =
      std::max<uint32_t>(16 * cap, 4096) + 2 * cap * (uint32_t)std::max(nextCheck, SAH_LEVELS_PER_CHECK);
  SahCtl *sc = nullptr;
  SahNode *bigList[2] = {nullptr, nullptr}, *next = nullptr, *tasks = nullptr;
  uint32_t *tileCount = nullptr, *first = nullptr, *tileRight = nullptr, *tileCnt = nullptr;
  int32_t *nodeBins = nullptr;
  SahDec *decs = nullptr;
  if ((s = tmp.get(&sc, 1)) != BQ_OK || (s = tmp.get(&bigList[0], cap)) != BQ_OK ||
      (s = tmp.get(&bigList[1], cap)) != BQ_OK || (s = tmp.get(&next, 2ull * cap)) != BQ_OK ||
      (s = tmp.get(&tasks, taskCap)) != BQ_OK || (s = tmp.get(&tileCount, cap)) != BQ_OK ||
      (s = tmp.get(&first, cap)) != BQ_OK || (s = tmp.get(&tileRight, maxTiles)) != BQ_OK ||
      (s = tmp.get(&tileCnt, (size_t)maxTiles * SAH_NB)) != BQ_OK ||
      (s = tmp.get(&nodeBins, (size_t)cap * SAH_NB * SAH_W)) != BQ_OK || (s = tmp.get(&decs, cap)) != BQ_OK)
    return fail(s);
  SahNode root;
  root.b = 0; root.e = nv; root.slot = 0; root.parity = 0;
  for (int d = 0; d < 3; d++) { root.lo[d] = hctl[2 + d]; root.hi[d] = hctl[5 + d]; }
  const bool rootBig = nv > warpMax && (int64_t)nv > thr;
  SahCtl hsc{};
  hsc.bigCount[0] = rootBig ? 1u : 0u;
  hsc.taskCount = rootBig ? 0u : 1u;
  if ((ce = cudaMemcpyAsync(rootBig ? bigList[0] : tasks, &root, sizeof(root), cudaMemcpyHostToDevice, al.s)) !=
          cudaSuccess ||
      (ce = cudaMemcpyAsync(sc, &hsc, sizeof(hsc), cudaMemcpyHostToDevice, al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "sah set-up"));
  const int warpGrid = num_sms() * 8;
  // with at most BQ_SCAN_SMEM_MAX big nodes and tiles a level's two scans run
  // inside one block each (7 launches per level instead of 12)
  const bool fused = cap <= BQ_SCAN_SMEM_MAX && maxTiles <= BQ_SCAN_SMEM_MAX;
  if (fused) {
    if ((ce = cudaFuncSetAttribute(k_sah_tiles_scan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(uint32_t) * cap))) != cudaSuccess ||
        (ce = cudaFuncSetAttribute(k_sah_right_children, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(uint32_t) * maxTiles))) != cudaSuccess)
      return fail(cuda_error(ce, "sah set-up"));
  }
  auto warp_phase = [&]() -> int {
    ProfScope ps(HEUR ? "elh.warps" : "sah.warps", al.s);
    launch_pdl(k_sah_warp, dim3(warpGrid), dim3(SAHW_BLOCK), 0, al.s, tasks, sc, taskCap, thr, buf0, buf1, full,
               primIDs, used);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->taskCount, 0, 2 * sizeof(uint32_t), al.s);  // taskCount, grab
    return e == cudaSuccess ? BQ_OK : cuda_error(e, "k_sah_warp");
  };
  int cur = 0;
  for (int level = 0; rootBig; level++) {
    {
      ProfScope ps(HEUR ? "elh.level" : "sah.level", al.s, fused ? 7 : 12);
      launch_pdl(k_sah_tiles, dim3(cap), dim3(128), 0, al.s, bigList[cur], sc, cur, cap, tileCount, nodeBins);
      if (fused) {
        launch_pdl(k_sah_tiles_scan, dim3(1), dim3(BQ_SCAN_THREADS), sizeof(uint32_t) * cap, al.s, sc, cur, cap,
                   maxTiles, tileCount, first);
      } else if ((s = exclusive_scan_u32(tileCount, first, cap, &sc->bigCount[cur], &sc->numTiles, al)) != BQ_OK) {
        return fail(s);
      }
      launch_pdl(k_sah_bin, dim3(maxTiles), dim3(SAH_BLOCK), 0, al.s, bigList[cur], first, sc, cur, maxTiles, buf0,
                 buf1, tileCnt, nodeBins);
      launch_pdl(k_sah_decide, dim3(div_up(cap, 4)), dim3(128), 0, al.s, bigList[cur], sc, cur, cap, thr, nodeBins,
                 decs, buf0, buf1, full, primIDs);
      if (fused) {
        launch_pdl(k_sah_right_children, dim3(1), dim3(BQ_SCAN_THREADS), sizeof(uint32_t) * maxTiles, al.s,
                   bigList[cur], first, sc, cur, cap, decs, tileCnt, tileRight, full, used, next);
      } else {
        launch_pdl(k_sah_tile_right, dim3(div_up(maxTiles, 128)), dim3(128), 0, al.s, bigList[cur], first, sc, cur,
                   maxTiles, decs, tileCnt, tileRight);
        if ((s = exclusive_scan_u32(tileRight, tileRight, maxTiles, &sc->scanLen, nullptr, al)) != BQ_OK)
          return fail(s);
        launch_pdl(k_sah_children, dim3(div_up(cap, 128)), dim3(128), 0, al.s, bigList[cur], sc, cur, cap, first,
                   tileRight, decs, full, used, next, &sc->err);
      }
      launch_pdl(k_sah_scatter, dim3(maxTiles), dim3(SAH_BLOCK), 0, al.s, bigList[cur], first, sc, cur, maxTiles,
                 tileRight, decs, buf0, buf1, next);
      launch_pdl(k_sah_classify, dim3(div_up(2ull * cap, 128)), dim3(128), 0, al.s, next, sc, cur, cap, thr, warpMax,
                 bigList[cur ^ 1], tasks, taskCap);
      if ((ce = cudaMemsetAsync(&sc->bigCount[cur], 0, sizeof(uint32_t), al.s)) != cudaSuccess ||
          (ce = cudaGetLastError()) != cudaSuccess)
        return fail(cuda_error(ce, "sah level"));
    }
    cur ^= 1;
    if (level + 1 < nextCheck) continue;
    nextCheck = level + 1 + SAH_LEVELS_PER_CHECK;
    if ((ce = cudaMemcpyAsync(&hsc, sc, sizeof(hsc), cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "sah levels"));
    if (hsc.err) return fail(set_error(BQ_ERR_CUDA, "sah level failed a range or capacity check"));
    if (hsc.bigCount[cur] == 0) break;
    if (hsc.taskCount + 2ull * SAH_LEVELS_PER_CHECK * cap > taskCap && (s = warp_phase()) != BQ_OK) return fail(s);
  }
  if ((s = warp_phase()) != BQ_OK) return fail(s);
  // ---- slot compaction ----
  uint32_t *rank = nullptr;
  if ((s = tmp.get(&rank, nv)) != BQ_OK) return fail(s);
  {
    ProfScope ps(HEUR ? "elh.rank" : "sah.rank", al.s, 3);
    if ((s = exclusive_scan_u32(used, rank, nv, nullptr, ctl + 2, al)) != BQ_OK) return fail(s);
  }
  uint32_t hres[2], herr = 0;
  if ((ce = cudaMemcpyAsync(hres, ctl + 1, 8, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaMemcpyAsync(&herr, &sc->err, 4, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "sah"));
  if (hres[0] || herr) return fail(set_error(BQ_ERR_CUDA, "sah build failed a range or capacity check"));
  const uint32_t numNodes = 2 + 2 * hres[1];
  Node *nodes = nullptr;
  if ((s = al.get(&nodes, numNodes)) != BQ_OK) return fail(s);
  {
    ProfScope ps(HEUR ? "elh.compact" : "sah.compact", al.s);
    launch_pdl(k_sah_compact, dim3(div_up(nv, 256)), dim3(256), 0, al.s, full, used, rank, nv, nodes);
  }
  bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
  bvh->numNodes = numNodes;
  bvh->primIDs = primIDs;
  bvh->numPrims = n;
  if ((s = refit(bvh, boxes, al, false)) != BQ_OK) {
    al.free_bytes(nodes);
    bvh->nodes = nullptr; bvh->numNodes = 0; bvh->primIDs = nullptr; bvh->numPrims = 0;
    return fail(s);
  }
  return BQ_OK;
}

} // namespace bq
