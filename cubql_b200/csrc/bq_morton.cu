// bq_morton.cu -- Morton (radix) BVH builder with 63-bit keys.
//
// Builds the same tree as cuBQL::cuda::radixBuilder<float,3>
// (cuBQL/builder/cuda/radix.h:591-771), without its per-level host loop:
//
//   k_bounds      centroid bounds and valid count of each block's chunk
//                 (radix.h:185-241 fillBuildState/finishBuildState)
//   k_keygen      every block first reduces those partials to the global
//                 bounds, the quantizer and its own compaction offset; then
//                 stable compaction of valid prims, 63-bit Morton keys
//                 (radix.h:41-62 Quantizer, 283-421 key generation) and the
//                 digit histograms of the top key bits
//   onesweep sort stable (key, primID) sort on the top key bits only:
//                 bits [39, 63) in 3 digit passes up to 2^24 prims, bits
//                 [31, 63) in 4 passes above, instead of 8 (bq_sort.cu)
//   k_fix_runs    runs of equal top bits are then ordered by the low bits,
//                 stably, from shared memory: runs of 2..4 prims (on
//                 uniform data nearly all runs) by one thread each, runs
//                 of 5..32 by one warp each, grouped by size so that warps
//                 do not diverge; longer runs, if they hold differing
//                 keys, by one segmented composite-key sort of just their
//                 prims ((run, low bits) keys) -- a run of identical keys
//                 is already in order.  The result is the full stable
//                 63-bit order, as cub's SortPairs gives.  The same kernel
//                 writes the split levels: one byte per
//                 adjacent key pair, the level at which the reference's
//                 top-down split would separate them (k_run_levels writes
//                 those inside the longer runs)
//   agglomerate   bottom-up construction of topology and boxes
//                 (bq_agglom.cuh: per-chunk in shared memory, then the few
//                 chunk-crossing nodes device-wide)
//
// Why the bottom-up pass gives the reference's tree: createNodes/findSplit
// (radix.h:446-570) split a key range [b,e) at the first key that has the
// highest bit in which keys[b] and keys[e-1] differ.  That bit flips exactly
// once inside the range, so the split is the unique adjacent pair whose
// highest differing bit is the largest in the range: the tree is the
// Cartesian (max-rooted) tree of the adjacent-pair "delta" array.  Runs of
// equal keys are split at (b+e)/2 recursively (radix.h:455-465); giving
// each split position inside a run the value 63 - (its depth in that
// midpoint recursion), below every real delta (64 + bit index), keeps the
// Cartesian-tree characterisation exact.  A Cartesian tree can be built
// bottom-up: a node covering [l,r] is the child of the split at whichever
// boundary (l or r+1) carries the smaller delta.  Each thread starts at one
// leaf and climbs; at every parent the first arriving thread parks its
// range end in a slot and stops, the second merges both children and goes
// on, so every node is written exactly once and nothing waits.
//
// Node numbering: the children of the split between sorted positions s-1
// and s go to nodes[2s], nodes[2s+1] (node 0 = root, node 1 unused), which
// is a valid BinaryBVH layout with 2*numValid nodes.  It differs from the
// reference's numbering, which its atomic allocation makes
// run-dependent anyway; trees are compared after BFS renumbering.
//
// Leaf thresholds above 1 (radix.h:525-530) first build the full tree, then
// collapse every subtree of at most `thr` prims into one leaf with a scan
// over the kept inner nodes.
#include <algorithm>
#include <climits>
#include <cfloat>

#include "bq_agglom.cuh"

namespace bq {
namespace {

constexpr int MB_BLOCK = 256;
constexpr int MB_UNROLL = 4;
// The global sort covers key bits [SB, 63): SB = 39 (24 bits, 3 passes) up
// to 2^24 prims, SB = 31 (32 bits, 4 passes) above, so that runs of equal
// sorted bits stay short (on uniform data about n / 2^(63-SB) prims each);
// the bits below SB are ordered inside those runs.
constexpr int MB_SB3 = 39, MB_SB4 = 31;
constexpr int MB_MAX_HIST_PASSES = 4;
template <int SB>
constexpr int hist_passes() { return (63 - SB + 7) / 8; }
template <int SB>
constexpr uint64_t low_mask() { return (1ull << SB) - 1; }
template <int SB>
__device__ __forceinline__ uint32_t key_hi(uint64_t k) { return (uint32_t)(k >> SB); }
constexpr uint32_t MB_THREAD_RUN = 32;  // longest run of equal top bits one thread orders

struct __align__(16) Partial {
  int32_t lo[3], hi[3];
  uint32_t cnt, pad;
};

__device__ __forceinline__ void load_box(const bq_box3f *boxes, uint64_t i, float &lx, float &ly, float &lz,
                                         float &hx, float &hy, float &hz)
{
  const float2 *p = reinterpret_cast<const float2 *>(boxes + i);
  const float2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  lx = a.x; ly = a.y; lz = b.x; hx = b.y; hy = c.x; hz = c.y;
}

// box.center() = (lower+upper)/2 (cuBQL/math/box.h:146-147)
// (lower + upper) / 2 as a multiply by 0.5: x / 2 and x * 0.5 round the same
// real number, so both give the same float (the divide costs a dozen
// instructions more)
__device__ __forceinline__ float ctr(float lo, float hi) { return __fmul_rn(__fadd_rn(lo, hi), 0.5f); }

// ------------------------------------------------------------------
// pass 1: bounds
// ------------------------------------------------------------------
__global__ void __launch_bounds__(MB_BLOCK) k_bounds(const bq_box3f *__restrict__ boxes, uint32_t n, uint32_t chunk,
                                                     Partial *__restrict__ partials, uint32_t *__restrict__ hist,
                                                     int histWords, uint32_t *__restrict__ zero, uint64_t zeroWords,
                                                     uint32_t *__restrict__ ctl, int ctlWords)
{
  griddep_wait();  // the previous work on the stream (its memory may be reused here) is done
  // the build state and run statistics, the digit histograms and the sort's
  // look-back state (16-byte aligned), zeroed here rather than by memset
  // launches of their own
  {
    if (blockIdx.x == 0)
      for (int i = threadIdx.x; i < ctlWords; i += MB_BLOCK) ctl[i] = 0u;
    uint4 *z4 = reinterpret_cast<uint4 *>(zero);
    const uint64_t n4 = zeroWords / 4;
    for (uint64_t i = (uint64_t)blockIdx.x * MB_BLOCK + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * MB_BLOCK)
      z4[i] = make_uint4(0u, 0u, 0u, 0u);
    if (blockIdx.x == 0 && threadIdx.x < (zeroWords & 3)) zero[n4 * 4 + threadIdx.x] = 0u;
    for (int i = blockIdx.x * MB_BLOCK + threadIdx.x; i < histWords; i += gridDim.x * MB_BLOCK) hist[i] = 0;
  }
  __shared__ int32_t sLo[3][MB_BLOCK / 32], sHi[3][MB_BLOCK / 32];
  __shared__ uint32_t sCnt[MB_BLOCK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = min((uint64_t)n, begin + chunk);
  int32_t lo0 = INT_MAX, lo1 = INT_MAX, lo2 = INT_MAX, hi0 = INT_MIN, hi1 = INT_MIN, hi2 = INT_MIN;
  uint32_t cnt = 0;
  for (uint64_t i0 = begin + threadIdx.x; i0 < end; i0 += (uint64_t)MB_BLOCK * MB_UNROLL) {
    float b[MB_UNROLL][6];
#pragma unroll
    for (int u = 0; u < MB_UNROLL; u++) {
      uint64_t i = i0 + (uint64_t)u * MB_BLOCK;
      if (i < end) load_box(boxes, i, b[u][0], b[u][1], b[u][2], b[u][3], b[u][4], b[u][5]);
      else b[u][0] = 1.f, b[u][3] = 0.f;  // empty
    }
#pragma unroll
    for (int u = 0; u < MB_UNROLL; u++) {
      if (!(b[u][0] > b[u][3])) {  // box.empty() is lower.x > upper.x (box.h:139)
        int32_t cx = enc_f(ctr(b[u][0], b[u][3])), cy = enc_f(ctr(b[u][1], b[u][4])), cz = enc_f(ctr(b[u][2], b[u][5]));
        lo0 = min(lo0, cx); lo1 = min(lo1, cy); lo2 = min(lo2, cz);
        hi0 = max(hi0, cx); hi1 = max(hi1, cy); hi2 = max(hi2, cz);
        cnt++;
      }
    }
  }
  lo0 = __reduce_min_sync(0xffffffffu, lo0); lo1 = __reduce_min_sync(0xffffffffu, lo1);
  lo2 = __reduce_min_sync(0xffffffffu, lo2); hi0 = __reduce_max_sync(0xffffffffu, hi0);
  hi1 = __reduce_max_sync(0xffffffffu, hi1); hi2 = __reduce_max_sync(0xffffffffu, hi2);
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if (lane == 0) {
    sLo[0][warp] = lo0; sLo[1][warp] = lo1; sLo[2][warp] = lo2;
    sHi[0][warp] = hi0; sHi[1][warp] = hi1; sHi[2][warp] = hi2;
    sCnt[warp] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p;
    for (int d = 0; d < 3; d++) { p.lo[d] = INT_MAX; p.hi[d] = INT_MIN; }
    p.cnt = 0;
    p.pad = 0;
    for (int w = 0; w < MB_BLOCK / 32; w++) {
      for (int d = 0; d < 3; d++) { p.lo[d] = min(p.lo[d], sLo[d][w]); p.hi[d] = max(p.hi[d], sHi[d][w]); }
      p.cnt += sCnt[w];
    }
    partials[blockIdx.x] = p;
  }
}

// The global centroid bounds, the quantizer (Quantizer<float,3>::init,
// radix.h:46-53) and this block's compaction offset, reduced from the
// per-block partials of k_bounds by every block of k_keygen (gridDim.x x
// 32 B from L2): k_bounds then has no serial last block.  Block 0 also
// records them in *st for the later kernels and the host.
struct KeyQuant {
  float bias[3], scale;
  uint32_t before, total;  // valid prims of the blocks before this one; of all blocks
};
__device__ __forceinline__ KeyQuant reduce_partials(const Partial *__restrict__ partials, BuildState *st)
{
  __shared__ int32_t sLo[3][MB_BLOCK / 32], sHi[3][MB_BLOCK / 32];
  __shared__ uint32_t sTot[MB_BLOCK / 32], sBefore[MB_BLOCK / 32];
  __shared__ KeyQuant sQ;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  uint32_t tot = 0, before = 0;
  for (uint32_t b = threadIdx.x; b < gridDim.x; b += MB_BLOCK) {
    const int4 *pp = reinterpret_cast<const int4 *>(partials + b);
    const int4 q0 = __ldg(pp), q1 = __ldg(pp + 1);  // lo[3] hi[0] | hi[1] hi[2] cnt pad
    lo[0] = min(lo[0], q0.x); lo[1] = min(lo[1], q0.y); lo[2] = min(lo[2], q0.z);
    hi[0] = max(hi[0], q0.w); hi[1] = max(hi[1], q1.x); hi[2] = max(hi[2], q1.y);
    tot += (uint32_t)q1.z;
    if (b < blockIdx.x) before += (uint32_t)q1.z;
  }
  for (int d = 0; d < 3; d++) {
    lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
    hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
  }
  tot = __reduce_add_sync(0xffffffffu, tot);
  before = __reduce_add_sync(0xffffffffu, before);
  if (lane == 0) {
    for (int d = 0; d < 3; d++) { sLo[d][warp] = lo[d]; sHi[d][warp] = hi[d]; }
    sTot[warp] = tot;
    sBefore[warp] = before;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    KeyQuant q;
    q.total = 0;
    q.before = 0;
    for (int w = 0; w < MB_BLOCK / 32; w++) { q.total += sTot[w]; q.before += sBefore[w]; }
    int32_t a[3], b[3];
    float sz[3];
    for (int d = 0; d < 3; d++) {
      a[d] = INT_MAX;
      b[d] = INT_MIN;
      for (int w = 0; w < MB_BLOCK / 32; w++) { a[d] = min(a[d], sLo[d][w]); b[d] = max(b[d], sHi[d][w]); }
      if (q.total == 0) { a[d] = enc_f(FLT_MAX); b[d] = enc_f(-FLT_MAX); }  // AtomicBox::set_empty
      q.bias[d] = dec_f(a[d]);
      sz[d] = __fsub_rn(dec_f(b[d]), q.bias[d]);
    }
    const float ext = fmaxf(fmaxf(sz[0], sz[1]), sz[2]);
    q.scale = __fmul_rn(2097152.0f, __fdiv_rn(1.0f, fmaxf(ext, 1e-20f)));
    sQ = q;
    if (blockIdx.x == 0) {
      for (int d = 0; d < 3; d++) { st->cbLo[d] = a[d]; st->cbHi[d] = b[d]; st->bias[d] = q.bias[d]; }
      st->scale = q.scale;
      st->numValid = q.total;
    }
  }
  __syncthreads();
  return sQ;
}

// ------------------------------------------------------------------
// pass 2: keys, compaction, digit histograms
// ------------------------------------------------------------------
template <int SB>
__global__ void __launch_bounds__(MB_BLOCK) k_keygen(const bq_box3f *__restrict__ boxes, uint32_t n, uint32_t chunk,
                                                     const Partial *__restrict__ partials, BuildState *st,
                                                     uint64_t *__restrict__ keys, uint32_t *__restrict__ ids,
                                                     uint32_t *__restrict__ hist)
{
  griddep_wait();
  constexpr int PASSES = hist_passes<SB>();
  __shared__ uint32_t sHist[PASSES * 256];
  __shared__ uint32_t sWarpCnt[MB_UNROLL][MB_BLOCK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < PASSES * 256; i += MB_BLOCK) sHist[i] = 0;
  const KeyQuant q = reduce_partials(partials, st);
  const float bx = q.bias[0], by = q.bias[1], bz = q.bias[2], sc = q.scale;
  uint32_t running = q.before;
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = min((uint64_t)n, begin + chunk);
  // every box of the chunk valid (the common case): prim i goes to position
  // running + (i - begin), with no compaction ballots or barriers
  const bool allValid = __ldg(&partials[blockIdx.x].cnt) == (uint32_t)(end - begin);
  __syncthreads();
  if (allValid) {
#pragma unroll 4
    for (uint64_t i = begin + threadIdx.x; i < end; i += MB_BLOCK) {
      float lx, ly, lz, hx, hy, hz;
      load_box(boxes, i, lx, ly, lz, hx, hy, hz);
      const float cx = ctr(lx, hx), cy = ctr(ly, hy), cz = ctr(lz, hz);
      const uint64_t key = spread21(quant_cell(cx, bx, sc, 2097151u)) |
                           (spread21(quant_cell(cy, by, sc, 2097151u)) << 1) |
                           (spread21(quant_cell(cz, bz, sc, 2097151u)) << 2);
      const uint32_t pos = running + (uint32_t)(i - begin);
      keys[pos] = key;
      ids[pos] = (uint32_t)i;
#pragma unroll
      for (int p = 0; p < PASSES; p++)
        atomicAdd(&sHist[p * 256 + ((key >> (SB + 8 * p)) & 0xff)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < PASSES * 256; i += MB_BLOCK)
      if (sHist[i]) atomicAdd(&hist[i], sHist[i]);
    return;
  }
  const uint32_t lt = (1u << lane) - 1u;
  for (uint64_t i0 = begin; i0 < end; i0 += (uint64_t)MB_BLOCK * MB_UNROLL) {
    float b[MB_UNROLL][6];
    bool valid[MB_UNROLL];
    uint32_t wpre[MB_UNROLL];
#pragma unroll
    for (int u = 0; u < MB_UNROLL; u++) {
      uint64_t i = i0 + (uint64_t)u * MB_BLOCK + threadIdx.x;
      valid[u] = false;
      if (i < end) {
        load_box(boxes, i, b[u][0], b[u][1], b[u][2], b[u][3], b[u][4], b[u][5]);
        valid[u] = !(b[u][0] > b[u][3]);
      }
      uint32_t bal = __ballot_sync(0xffffffffu, valid[u]);
      wpre[u] = __popc(bal & lt);
      if (lane == 0) sWarpCnt[u][warp] = __popc(bal);
    }
    __syncthreads();
    uint32_t base[MB_UNROLL];
    uint32_t acc = running;
#pragma unroll
    for (int u = 0; u < MB_UNROLL; u++) {
      uint32_t wb = 0, tot = 0;
#pragma unroll
      for (int w = 0; w < MB_BLOCK / 32; w++) {
        uint32_t c = sWarpCnt[u][w];
        wb += (w < warp) ? c : 0;
        tot += c;
      }
      base[u] = acc + wb;
      acc += tot;
    }
    running = acc;
    __syncthreads();
#pragma unroll
    for (int u = 0; u < MB_UNROLL; u++) {
      if (!valid[u]) continue;
      const float cx = ctr(b[u][0], b[u][3]), cy = ctr(b[u][1], b[u][4]), cz = ctr(b[u][2], b[u][5]);
      const uint64_t key = spread21(quant_cell(cx, bx, sc, 2097151u)) |
                           (spread21(quant_cell(cy, by, sc, 2097151u)) << 1) |
                           (spread21(quant_cell(cz, bz, sc, 2097151u)) << 2);
      const uint32_t pos = base[u] + wpre[u];
      keys[pos] = key;
      ids[pos] = (uint32_t)(i0 + (uint64_t)u * MB_BLOCK + threadIdx.x);
#pragma unroll
      for (int p = 0; p < PASSES; p++)
        atomicAdd(&sHist[p * 256 + ((key >> (SB + 8 * p)) & 0xff)], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < PASSES * 256; i += MB_BLOCK)
    if (sHist[i]) atomicAdd(&hist[i], sHist[i]);
}

// ------------------------------------------------------------------
// runs of equal top key bits: order them by the low bits, stably
// ------------------------------------------------------------------
struct RunStats {
  uint32_t count, elems, maxSize, pad;
};

// one past the last index j >= i with key_hi(keys[j]) == hi (key_hi(keys[i]) == hi)
template <int SB>
__device__ __forceinline__ uint32_t hi_run_end(const uint64_t *__restrict__ keys, uint32_t i, uint32_t hi, uint32_t n)
{
  uint32_t step = 1, lo = i + 1, up = n;
  while (lo < up) {
    const uint32_t probe = lo - 1 + min(step, up - lo + 1);
    if (probe >= up || key_hi<SB>(keys[probe]) != hi) { up = min(probe, up); break; }
    lo = probe + 1;
    step <<= 1;
  }
  while (lo < up) {
    const uint32_t m = lo + ((up - lo) >> 1);
    if (key_hi<SB>(keys[m]) == hi) lo = m + 1; else up = m;
  }
  return lo;
}

// split level of two different keys (highest differing bit + 64)
__device__ __forceinline__ uint8_t key_level(uint64_t a, uint64_t b) { return (uint8_t)(64 + (63 - __clzll(a ^ b))); }

// level of split position s inside the run [r0, r1) of equal keys: 63 minus
// its depth in the (b+e)/2 recursion of radix.h:455-465
__device__ __forceinline__ uint8_t equal_run_level(uint64_t r0, uint64_t r1, uint64_t s)
{
  int depth = 0;
  while (true) {
    const uint64_t m = (r0 + r1) / 2;
    if (s == m) break;
    if (s < m) r1 = m; else r0 = m;
    depth++;
  }
  return (uint8_t)(63 - depth);
}

// Every sorted position: the split level of the pair (i, i+1), and the
// low-bit order inside runs of equal top bits.
// One block covers FT_TILE consecutive positions, staged in shared memory
// with FT_HALO positions after them:
//   A. per position: the split level of a pair that lies across
//      two runs (their highest differing bit is a top bit, so it does not
//      depend on the order inside the runs) and, at the first position of a
//      run, the run's size class -- 2, 3..4 or more prims -- appended to
//      that class's list;
//   B. the block then orders the listed runs class by class, so a warp
//      runs one code path at a time: pairs and runs of 3..4 by one thread
//      each in registers, runs of 5..32 by one warp each (a lane per prim
//      takes its rank), all from shared memory; longer runs are listed for
//      the segmented sort.
// A run belongs to the tile holding its first position, including the part
// of it that lies in the next tile; that tile reads only the top bits of
// those prims, which the reordering leaves unchanged, and writes none of
// their keys, ids or inner levels.
constexpr int FT_BLOCK = 256;
constexpr int FT_ITEMS = 4;
constexpr uint32_t FT_TILE = FT_BLOCK * FT_ITEMS;
constexpr uint32_t FT_HALO = 32;  // a run of up to 32 prims begun in the tile is staged whole

// the pair / three-or-four run starting at sorted position i, keys r[] and
// ids src[] in their current order: order it on the low bits (stable) and
// write the levels of the pairs inside it
__device__ __forceinline__ void order_run2(uint64_t a, uint64_t b, uint64_t i, const uint32_t *src, uint64_t *keys,
                                           uint32_t *ids, uint8_t *__restrict__ delta)
{
  if (a > b) {
    const uint32_t ia = src[0], ib = src[1];
    keys[i] = b; keys[i + 1] = a;
    ids[i] = ib; ids[i + 1] = ia;
  }
  delta[i] = a != b ? key_level(a, b) : (uint8_t)63;  // equal: the midpoint of [i, i+2)
}

__device__ __forceinline__ void order_run34(uint64_t r[4], uint32_t size, uint64_t i, const uint32_t *src,
                                            uint64_t *keys, uint32_t *ids, uint8_t *__restrict__ delta)
{
  if (size == 3) r[3] = ~0ull;  // above every key: stays last
  uint32_t d[4] = {0u, 1u, 2u, 3u};
  bool moved = false;
#pragma unroll
  for (int pass = 0; pass < 3; pass++)  // bubble sort: swaps on > only, so stable
#pragma unroll
    for (int j = 0; j < 3; j++)
      if (r[j] > r[j + 1]) {
        const uint64_t t = r[j]; r[j] = r[j + 1]; r[j + 1] = t;
        const uint32_t u = d[j]; d[j] = d[j + 1]; d[j + 1] = u;
        moved = true;
      }
  if (moved) {
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = (uint32_t)j < size ? src[d[j]] : 0u;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if ((uint32_t)j < size && d[j] != (uint32_t)j) {
        keys[i + j] = r[j];
        ids[i + j] = v[j];
      }
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    if ((uint32_t)j + 1 >= size) break;
    if (r[j] != r[j + 1]) {
      delta[i + j] = key_level(r[j], r[j + 1]);
    } else {
      int e0 = j, e1 = j + 2;  // the run of keys equal to r[j] (constant indices only)
#pragma unroll
      for (int t = 2; t >= 0; t--)
        if (t < j && e0 == t + 1 && r[t] == r[j]) e0 = t;
#pragma unroll
      for (int t = 2; t < 4; t++)
        if (t >= j + 2 && e1 == t && (uint32_t)t < size && r[t] == r[j]) e1 = t + 1;
      delta[i + j] = equal_run_level(i + e0, i + e1, i + j + 1);
    }
  }
}

// a run of more than MB_THREAD_RUN prims starting at sorted position i: listed
// for sort_low_bits (its inner levels are written by k_run_levels)
template <int SB>
__device__ __forceinline__ void list_long_run(uint32_t i, uint32_t hi, uint32_t nv, const uint64_t *keys, RunStats *rs,
                                              uint4 *runs, uint32_t maxRuns)
{
  const uint32_t size = hi_run_end<SB>(keys, i, hi, nv) - i;
  const uint32_t slotIdx = atomicAdd(&rs->count, 1u);
  if (slotIdx < maxRuns) runs[slotIdx] = make_uint4(i, size, hi, 0);
  else atomicOr(&rs->pad, 1u);  // cannot happen: maxRuns = nv / (MB_THREAD_RUN + 1) + 1
  atomicAdd(&rs->elems, size);
  atomicMax(&rs->maxSize, size);
}

// 8 blocks per SM (32 registers): the kernel is latency-bound, and occupancy
// pays more than the few spilled bytes cost
template <int SB>
__global__ void __launch_bounds__(FT_BLOCK, 8) k_fix_runs(uint64_t *keys, uint32_t *ids, const uint32_t *nvPtr,
                                                       uint8_t *__restrict__ delta,
                                                       RunStats *rs, uint4 *runs, uint32_t maxRuns)
{
  griddep_wait();
  __shared__ uint64_t sK[FT_TILE + FT_HALO + 1];  // [0]: position base-1, [1+j]: base+j
  __shared__ uint16_t sR2[FT_TILE / 2], sR34[FT_TILE / 3 + 1], sRL[FT_TILE / 5 + 1];
  __shared__ uint32_t sCnt[3];
  __shared__ uint64_t sSorted[FT_BLOCK / 32][32];  // per warp: a run of 5..32 keys in order
  const uint32_t nv = *nvPtr;
  const uint64_t base = (uint64_t)blockIdx.x * FT_TILE;
  if (base >= nv) return;
  const uint32_t len = (uint32_t)min((uint64_t)FT_TILE, nv - base);
  const uint32_t lenH = (uint32_t)min((uint64_t)(FT_TILE + FT_HALO), nv - base);  // staged positions
  const int t = threadIdx.x, lane = t & 31;
  const uint32_t lt = (1u << lane) - 1u;

  for (uint32_t j = t; j < lenH; j += FT_BLOCK) sK[j + 1] = keys[base + j];
  if (t == 0) sK[0] = base > 0 ? keys[base - 1] : 0ull;
  if (t < 3) sCnt[t] = 0u;
  __syncthreads();

  // A. levels across runs; runs begun here, by size class
#pragma unroll
  for (int u = 0; u < FT_ITEMS; u++) {
    const uint32_t j = u * FT_BLOCK + t;
    int cls = -1;
    if (j < len) {
      const uint64_t k = sK[j + 1];
      const uint32_t hi = key_hi<SB>(k);
      const bool hasNext = j + 1 < lenH;
      const uint64_t kn = sK[j + 2];
      const bool nextSame = hasNext && key_hi<SB>(kn) == hi;
      if (hasNext && !nextSame) delta[base + j] = key_level(k, kn);
      const bool prevSame = (j > 0 || base > 0) && key_hi<SB>(sK[j]) == hi;
      if (nextSame && !prevSame) {
        uint32_t size = 2;
        while (size < 5 && j + size < lenH && key_hi<SB>(sK[j + size + 1]) == hi) size++;
        cls = size == 2 ? 0 : size < 5 ? 1 : 2;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const uint32_t m = __ballot_sync(0xffffffffu, cls == c);
      if (m == 0) continue;
      uint32_t at = 0;
      if (lane == __ffs(m) - 1) at = atomicAdd(&sCnt[c], (uint32_t)__popc(m));
      at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
      if (cls == c) {
        uint16_t *list = c == 0 ? sR2 : c == 1 ? sR34 : sRL;
        list[at + __popc(m & lt)] = (uint16_t)j;
      }
    }
  }
  __syncthreads();

  // B. order the listed runs, one class at a time
  const uint32_t n2 = sCnt[0], n34 = sCnt[1], nL = sCnt[2];
  for (uint32_t r = t; r < n2; r += FT_BLOCK) {
    const uint32_t j = sR2[r];
    order_run2(sK[j + 1], sK[j + 2], base + j, ids + base + j, keys, ids, delta);
  }
  for (uint32_t r = t; r < n34; r += FT_BLOCK) {
    const uint32_t j = sR34[r];
    const uint32_t hi = key_hi<SB>(sK[j + 1]);
    const uint32_t size = j + 3 < lenH && key_hi<SB>(sK[j + 4]) == hi ? 4u : 3u;
    uint64_t rk[4] = {sK[j + 1], sK[j + 2], sK[j + 3], size == 4 ? sK[j + 4] : 0ull};
    order_run34(rk, size, base + j, ids + base + j, keys, ids, delta);
  }
  // runs of 5..32 prims: one warp each, a lane per prim; longer ones are listed
  const int warp = t >> 5;
  uint64_t *scratch = sSorted[warp];
  for (uint32_t r = warp; r < nL; r += FT_BLOCK / 32) {
    const uint32_t j = sRL[r];
    const uint32_t hi = key_hi<SB>(sK[j + 1]);
    const uint32_t m = __ballot_sync(0xffffffffu, j + lane < lenH && key_hi<SB>(sK[j + lane + 1]) == hi);
    if (m == 0xffffffffu && j + 32 < lenH && key_hi<SB>(sK[j + 33]) == hi) {
      if (lane == 0) list_long_run<SB>((uint32_t)(base + j), hi, nv, keys, rs, runs, maxRuns);
      continue;
    }
    const uint32_t size = m == 0xffffffffu ? 32u : (uint32_t)__ffs(~m) - 1u;
    const bool in = (uint32_t)lane < size;
    const uint64_t k = in ? sK[j + lane + 1] : ~0ull;
    uint32_t rank = 0;
    for (uint32_t q = 0; q < size; q++) {
      const uint64_t x = __shfl_sync(0xffffffffu, k, (int)q);
      rank += (x < k || (x == k && q < (uint32_t)lane)) ? 1u : 0u;
    }
    const uint64_t i0 = base + j;
    if (__ballot_sync(0xffffffffu, in && rank != (uint32_t)lane)) {
      const uint32_t id = in ? ids[i0 + lane] : 0u;
      __syncwarp();
      if (in && rank != (uint32_t)lane) {
        keys[i0 + rank] = k;
        ids[i0 + rank] = id;
      }
    }
    if (in) scratch[rank] = k;
    __syncwarp();
    const uint64_t sk = in ? scratch[lane] : 0ull;
    __syncwarp();
    const uint64_t skPrev = __shfl_up_sync(0xffffffffu, sk, 1), skNext = __shfl_down_sync(0xffffffffu, sk, 1);
    const uint32_t eqStart = __ballot_sync(0xffffffffu, in && (lane == 0 || sk != skPrev));
    if ((uint32_t)lane + 1 < size) {
      if (sk != skNext) {
        delta[i0 + lane] = key_level(sk, skNext);
      } else {  // the run of keys equal to sk: [e0, e1)
        const uint32_t e0 = 31u - __clz(eqStart & ((2u << lane) - 1u));
        const uint32_t above = eqStart & ~((2u << lane) - 1u);
        const uint32_t e1 = above ? (uint32_t)__ffs(above) - 1u : size;
        delta[i0 + lane] = equal_run_level(i0 + e0, i0 + e1, i0 + lane + 1);
      }
    }
  }
}

__global__ void k_run_sizes(const uint4 *__restrict__ runs, uint32_t numRuns, uint32_t *__restrict__ sizes)
{
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < numRuns) sizes[r] = runs[r].y;
}

// the run of compacted slot t: last run whose offset is <= t
__device__ __forceinline__ uint32_t run_of(const uint32_t *__restrict__ off, uint32_t numRuns, uint32_t t)
{
  uint32_t lo = 0, hi = numRuns;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (__ldg(off + m) <= t) lo = m; else hi = m;
  }
  return lo;
}

// long run r (of R) holds differing keys: mixed[r] = 1 (every writer stores 1)
__global__ void k_run_mixed(const uint4 *__restrict__ runs, const uint32_t *__restrict__ off, uint32_t R, uint32_t P,
                            const uint64_t *__restrict__ keys, uint32_t *__restrict__ mixed)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P) return;
  const uint32_t r = run_of(off, R, t);
  const uint4 run = runs[r];
  if (keys[run.x + (t - off[r])] != keys[run.x]) mixed[r] = 1u;
}

// the mixed runs, compacted in run order, and their sizes
__global__ void k_run_pick(const uint4 *__restrict__ runs, const uint32_t *__restrict__ mixed,
                           const uint32_t *__restrict__ rank, uint32_t R, uint4 *__restrict__ runsM,
                           uint32_t *__restrict__ sizesM)
{
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R || !mixed[r]) return;
  runsM[rank[r]] = runs[r];
  sizesM[rank[r]] = runs[r].y;
}

// cnt[0] runs (cnt[1] prims, both on the device): composite (run, low bits) keys
template <int SB>
__global__ void k_run_gather(const uint4 *__restrict__ runs, const uint32_t *__restrict__ off,
                             const uint32_t *__restrict__ cnt, const uint64_t *__restrict__ keys,
                             const uint32_t *__restrict__ ids, uint64_t *__restrict__ kk, uint32_t *__restrict__ vv)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt[1]) return;
  const uint32_t r = run_of(off, cnt[0], t);
  const uint32_t pos = runs[r].x + (t - off[r]);
  kk[t] = ((uint64_t)r << SB) | (keys[pos] & low_mask<SB>());
  vv[t] = ids[pos];
}

template <int SB>
__global__ void k_run_scatter(const uint4 *__restrict__ runs, const uint32_t *__restrict__ off,
                              const uint32_t *__restrict__ cnt, const uint64_t *__restrict__ kk,
                              const uint32_t *__restrict__ vv, uint64_t *__restrict__ keys, uint32_t *__restrict__ ids)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt[1]) return;
  const uint64_t k = kk[t];
  const uint32_t r = (uint32_t)(k >> SB);
  const uint4 run = runs[r];
  const uint32_t pos = run.x + (t - off[r]);
  keys[pos] = ((uint64_t)run.z << SB) | (k & low_mask<SB>());
  ids[pos] = vv[t];
}

// Split levels of the pairs inside the long runs (the pairs at their ends,
// which lie across runs, were written by k_fix_runs).  A run
// of identical keys is split at (b+e)/2 recursively (radix.h:455-465); in a
// mixed run, equal neighbours are looked up inside the run.
__global__ void k_run_levels(const uint4 *__restrict__ runs, const uint32_t *__restrict__ off, uint32_t R,
                             uint32_t P, const uint32_t *__restrict__ mixed, const uint64_t *__restrict__ keys,
                             uint8_t *__restrict__ delta)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P) return;
  const uint32_t r = run_of(off, R, t);
  const uint4 run = runs[r];
  const uint32_t pos = run.x + (t - off[r]), end = run.x + run.y;
  if (pos + 1 >= end) return;
  if (!mixed[r]) {
    delta[pos] = equal_run_level(run.x, end, (uint64_t)pos + 1);
    return;
  }
  const uint64_t a = keys[pos], b = keys[pos + 1];
  if (a != b) {
    delta[pos] = key_level(a, b);
  } else {
    const uint32_t r0 = run_begin(keys, run.x, pos, a);
    const uint32_t r1 = run_end(keys, pos + 1, end, a);
    delta[pos] = equal_run_level(r0, r1, (uint64_t)pos + 1);
  }
}

// ------------------------------------------------------------------
// leaf threshold > 1: collapse small subtrees of the full tree
// ------------------------------------------------------------------
__global__ void k_kept(const uint2 *__restrict__ ranges, const uint32_t *nvPtr, int thr, uint32_t *__restrict__ kept)
{
  const uint32_t nv = *nvPtr;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x + 1;  // split positions 1..nv-1
  if (s >= nv) return;
  const uint2 rg = ranges[s];
  kept[s - 1] = (rg.y - rg.x + 1 > (uint32_t)thr) ? 1u : 0u;
}

__global__ void k_collapse(const Node *__restrict__ full, const uint2 *__restrict__ ranges,
                           const uint32_t *__restrict__ kept, const uint32_t *__restrict__ rank, const uint32_t *nvPtr,
                           int thr, Node *__restrict__ out)
{
  const uint32_t nv = *nvPtr;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    Node root = full[0];
    uint64_t a;
    if (nv > (uint32_t)thr) {
      const uint32_t s0 = (uint32_t)(admin_offset(node_admin(root)) >> 1);
      a = make_admin(2ull + 2ull * rank[s0 - 1], 0);
    } else {
      a = make_admin(0, nv);
    }
    out[0] = make_node(root.a.x, root.a.y, root.a.z, root.a.w, root.b.x, root.b.y, a);
    out[1] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0);
  }
  const uint32_t s = t + 1;
  if (s >= nv || !kept[s - 1]) return;
  const uint2 rg = ranges[s];
  const uint64_t base = 2ull + 2ull * rank[s - 1];
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const Node c = full[2ull * s + side];
    const uint32_t cl = side ? s : rg.x, cr = side ? rg.y : s - 1;
    const uint32_t sz = cr - cl + 1;
    uint64_t a;
    if (sz > (uint32_t)thr) {
      const uint32_t cs = (uint32_t)(admin_offset(node_admin(c)) >> 1);
      a = make_admin(2ull + 2ull * rank[cs - 1], 0);
    } else {
      a = make_admin(cl, sz);
    }
    out[base + side] = make_node(c.a.x, c.a.y, c.a.z, c.a.w, c.b.x, c.b.y, a);
  }
}

} // namespace

// ------------------------------------------------------------------
// low-bit order inside runs of equal top bits (after the top-bit sort)
// ------------------------------------------------------------------
namespace {
// Orders the runs of equal top bits of at most MB_THREAD_RUN prims and writes
// every split level (k_fix_runs); longer runs are listed in `runs`
// and counted in *rs (zeroed by the caller) for long_runs.  Nothing waits
// here.
template <int SB>
int fix_runs(uint64_t *keys, uint32_t *ids, uint32_t n, const uint32_t *nvDev, uint8_t *delta, RunStats *rs,
             uint4 *runs, uint32_t maxRuns, Alloc &al)
{
  ProfScope ps("morton.runs", al.s);
  BQ_CUDA(launch_pdl(k_fix_runs<SB>, dim3(div_up(n, FT_TILE)), dim3(FT_BLOCK), 0, al.s, keys, ids, nvDev, delta, rs,
                     runs, maxRuns));
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

// The runs longer than MB_THREAD_RUN (h: their statistics, read back).
// Those holding differing keys get one stable sort of (run, low bits) over
// just their prims, written back into each run's range; runs of identical
// keys are already in order (the sort of the top bits is stable).  Then the
// levels inside all of them.
template <int SB>
int long_runs(const RunStats &h, const uint4 *runs, uint64_t *keys, uint32_t *ids, uint64_t *spareKeys,
              uint32_t *spareIds, uint8_t *delta, uint32_t *err, Alloc &al)
{
  if (h.count == 0) return BQ_OK;
  TempSet tmp(al);
  const uint32_t R = h.count, P = h.elems;
  uint32_t *off = nullptr, *mixed = nullptr, *rank = nullptr, *sizesM = nullptr, *offM = nullptr, *cnt = nullptr;
  uint4 *runsM = nullptr;
  BQ_TRY(tmp.get(&off, R + 1ull));
  BQ_TRY(tmp.get(&mixed, R));
  BQ_TRY(tmp.get(&rank, R));
  BQ_TRY(tmp.get(&runsM, R));
  BQ_TRY(tmp.get(&sizesM, R));
  BQ_TRY(tmp.get(&offM, R));
  BQ_TRY(tmp.get(&cnt, 2));  // mixed runs, their prims
  uint64_t *kk[2] = {spareKeys, nullptr};
  uint32_t *vv[2] = {spareIds, nullptr};
  BQ_TRY(tmp.get(&kk[1], P));
  BQ_TRY(tmp.get(&vv[1], P));
  int runBits = 0;
  while (runBits < 32 && ((R - 1) >> runBits)) runBits++;
  if (runBits > 64 - SB) return set_error(BQ_ERR_UNSUPPORTED, "too many long runs of equal keys");
  BQ_CUDA(cudaMemsetAsync(mixed, 0, sizeof(uint32_t) * R, al.s));
  {
    ProfScope ps("morton.longruns", al.s, 6);
    k_run_sizes<<<div_up(R, 256), 256, 0, al.s>>>(runs, R, off);
    BQ_TRY(exclusive_scan_u32(off, off, R, nullptr, off + R, al));
    k_run_mixed<<<div_up(P, 256), 256, 0, al.s>>>(runs, off, R, P, keys, mixed);
    BQ_TRY(exclusive_scan_u32(mixed, rank, R, nullptr, cnt, al));
    k_run_pick<<<div_up(R, 256), 256, 0, al.s>>>(runs, mixed, rank, R, runsM, sizesM);
    BQ_TRY(exclusive_scan_u32(sizesM, offM, R, cnt, cnt + 1, al));
    k_run_gather<SB><<<div_up(P, 256), 256, 0, al.s>>>(runsM, offM, cnt, keys, ids, kk[0], vv[0]);
  }
  int ksel = 0;
  BQ_TRY(onesweep_sort_u64(kk, vv, P, cnt + 1, 0, SB + runBits, nullptr, &ksel, err, al));
  {
    ProfScope ps("morton.runlevels", al.s, 2);
    k_run_scatter<SB><<<div_up(P, 256), 256, 0, al.s>>>(runsM, offM, cnt, kk[ksel], vv[ksel], keys, ids);
    k_run_levels<<<div_up(P, 256), 256, 0, al.s>>>(runs, off, R, P, mixed, keys, delta);
  }
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}
} // namespace

// ------------------------------------------------------------------
// host entry
// ------------------------------------------------------------------
int build_morton63(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
{
  const int maxLeaf = cfg ? cfg->maxAllowedLeafSize : (1 << 15);
  const int mlt = cfg ? cfg->makeLeafThreshold : 0;
  const int thr = mlt > 0 ? std::min(mlt, maxLeaf) : 1;  // radix.h:599-602
  if (thr < 1 || thr > 65535)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "leaf threshold must be in [1, 65535] (16-bit leaf count)");
  bvh->nodes = nullptr; bvh->primIDs = nullptr; bvh->numNodes = 0; bvh->numPrims = 0;
  if (n == 0) return BQ_OK;

  const int sms = num_sms();
  int grid = std::max(1, std::min(div_up(n, MB_BLOCK * MB_UNROLL), sms * 4));
  uint32_t chunk = (uint32_t)div_up(div_up(n, grid), MB_BLOCK * MB_UNROLL) * (MB_BLOCK * MB_UNROLL);
  grid = div_up(n, chunk);

  TempSet tmp(al);
  // the build's state and the long-run statistics side by side, so that
  // one copy reads back everything the host needs
  struct Ctl {
    BuildState st;
    RunStats runs;
  };
  static_assert(sizeof(Ctl) % 4 == 0, "k_bounds zeroes the control block as words");
  // all temporaries of the build in one allocation (one call to the
  // allocator instead of a dozen before the first kernel can start)
  const bool wide4 = n > (1u << 24);  // more than 2^24 prims: sort 32 top bits in 4 passes instead of 24 in 3
  const int sb = wide4 ? MB_SB4 : MB_SB3;
  const int histWords = (wide4 ? hist_passes<MB_SB4>() : hist_passes<MB_SB3>()) * 256;
  const size_t sortCtlWords = onesweep_ctl_words(n, sb, 63);
  const uint32_t maxRuns = n / (MB_THREAD_RUN + 1) + 1;
  Ctl *ctl = nullptr;
  Partial *partials = nullptr;
  uint32_t *hist = nullptr, *slot = nullptr, *sortCtl = nullptr;
  uint64_t *keysA = nullptr, *keysB = nullptr;
  uint8_t *delta = nullptr;
  uint4 *runs = nullptr;
  uint2 *pending = nullptr;
  auto carve = [&](Carver &c) {
    c.take(&ctl, 1);
    c.take(&partials, grid);
    c.take(&hist, MB_MAX_HIST_PASSES * 256);
    c.take(&keysA, n);
    c.take(&keysB, n);
    c.take(&delta, n);
    c.take(&slot, n);
    c.take(&runs, maxRuns);
    c.take(&pending, 2ull * div_up(n, AGG_CHUNK));
    c.take(&sortCtl, sortCtlWords);
  };
  Carver sizing(nullptr);
  carve(sizing);
  char *arena = nullptr;
  BQ_TRY(tmp.get(&arena, sizing.off));
  Carver cut(arena);
  carve(cut);
  BuildState *st = &ctl->st;
  uint32_t *idsA = nullptr, *idsB = nullptr;
  Node *nodes = nullptr;
  BQ_TRY(al.get(&idsA, n));
  int s = al.get(&idsB, n);
  if (s != BQ_OK) { al.free_bytes(idsA); return s; }
  auto fail = [&](int code) {
    al.free_bytes(idsA); al.free_bytes(idsB); al.free_bytes(nodes);
    return code;
  };
  if (thr == 1) {
    if ((s = al.get(&nodes, 2ull * n)) != BQ_OK) return fail(s);
  }
  cudaError_t ce = cudaSuccess;

  {
    ProfScope ps("morton.bounds", al.s);
    ce = launch_pdl(k_bounds, dim3(grid), dim3(MB_BLOCK), 0, al.s, boxes, n, chunk, partials, hist, histWords, sortCtl,
                    (uint64_t)sortCtlWords, reinterpret_cast<uint32_t *>(ctl), (int)(sizeof(Ctl) / 4));
  }
  if (ce == cudaSuccess) {
    ProfScope ps("morton.keygen", al.s);
    if (wide4)
      ce = launch_pdl(k_keygen<MB_SB4>, dim3(grid), dim3(MB_BLOCK), 0, al.s, boxes, n, chunk, (const Partial *)partials,
                      st, keysA, idsA, hist);
    else
      ce = launch_pdl(k_keygen<MB_SB3>, dim3(grid), dim3(MB_BLOCK), 0, al.s, boxes, n, chunk, (const Partial *)partials,
                      st, keysA, idsA, hist);
  }
  if (ce == cudaSuccess) ce = cudaGetLastError();
  if (ce != cudaSuccess) return fail(cuda_error(ce, "k_bounds/k_keygen"));

  uint64_t *keys2[2] = {keysA, keysB};
  uint32_t *ids2[2] = {idsA, idsB};
  int sel = 0;
  if ((s = onesweep_sort_u64(keys2, ids2, n, &st->numValid, sb, 63, hist, &sel, &st->err, al, sortCtl)) != BQ_OK)
    return fail(s);
  uint64_t *keys = keys2[sel];
  uint32_t *ids = ids2[sel];
  uint32_t *idsOther = ids2[sel ^ 1];
  RunStats *rs = &ctl->runs;
  s = wide4 ? fix_runs<MB_SB4>(keys, ids, n, &st->numValid, delta, rs, runs, maxRuns, al)
            : fix_runs<MB_SB3>(keys, ids, n, &st->numValid, delta, rs, runs, maxRuns, al);
  if (s != BQ_OK) return fail(s);
  AggArgs ag{delta, slot, ids, boxes, nodes, nullptr, &st->numValid, nullptr, pending, nullptr, 0};
  // what the host reads back (one copy): the long-run statistics, the valid
  // count, the error word
  struct { RunStats runs; uint32_t nv, err; } h = {};
  Ctl *pinned = static_cast<Ctl *>(host_readback_buffer(sizeof(Ctl)));
  auto read_back = [&]() -> cudaError_t {
    Ctl local;
    Ctl &hc = pinned ? *pinned : local;
    cudaError_t e = cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, al.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(al.s);
    h.runs = hc.runs;
    h.nv = hc.st.numValid;
    h.err = hc.st.err;
    return e;
  };
  auto do_long_runs = [&]() -> int {
    return wide4 ? long_runs<MB_SB4>(h.runs, runs, keys, ids, keys2[sel ^ 1], idsOther, delta, &st->err, al)
                 : long_runs<MB_SB3>(h.runs, runs, keys, ids, keys2[sel ^ 1], idsOther, delta, &st->err, al);
  };
  // The one read-back of a build: the valid count, the sort's error word
  // and the long-run statistics, which decide what runs next.  Without long
  // runs nothing after this point can fail on the device, so the
  // agglomeration is left running on the stream (stream-ordered, like the
  // reference builder, which returns before its refit completes); with them
  // a second read-back collects the long-run sort's error word.
  if ((ce = read_back()) != cudaSuccess) return fail(cuda_error(ce, "build sync"));
  if (h.runs.pad) return fail(set_error(BQ_ERR_CUDA, "run list overflow in the Morton build"));
  if (h.err & DEV_ERR_TIMEOUT) return fail(set_error(BQ_ERR_TIMEOUT, "radix sort look-back timed out"));
  if (h.err) return fail(set_error(BQ_ERR_CUDA, "device-side range check failed in the Morton build"));
  const bool longRuns = h.runs.count > 0;
  if ((s = do_long_runs()) != BQ_OK) return fail(s);
  if (thr == 1) {
    if ((s = agglomerate<false>(ag, n, al.s, "morton.agg_local", "morton.agg_global")) != BQ_OK) return fail(s);
    if (longRuns && (ce = read_back()) != cudaSuccess) return fail(cuda_error(ce, "build sync"));
  } else {
    Node *full = nullptr;
    uint2 *ranges = nullptr;
    uint32_t *kept = nullptr, *rank = nullptr, *total = nullptr;
    TempSet tmp2(al);
    if ((s = tmp2.get(&full, 2ull * n)) != BQ_OK) return fail(s);
    if ((s = tmp2.get(&ranges, n)) != BQ_OK) return fail(s);
    if ((s = tmp2.get(&kept, n)) != BQ_OK) return fail(s);
    if ((s = tmp2.get(&rank, n)) != BQ_OK) return fail(s);
    if ((s = tmp2.get(&total, 1)) != BQ_OK) return fail(s);
    if ((ce = cudaMemsetAsync(kept, 0, sizeof(uint32_t) * n, al.s)) != cudaSuccess) return fail(cuda_error(ce, "memset"));
    ag.nodes = full;
    ag.ranges = ranges;
    if ((s = agglomerate<false>(ag, n, al.s, "morton.agg_local", "morton.agg_global")) != BQ_OK) return fail(s);
    k_kept<<<div_up(n, 256), 256, 0, al.s>>>(ranges, &st->numValid, thr, kept);
    if ((s = exclusive_scan_u32(kept, rank, n > 1 ? n - 1 : 1, nullptr, total, al)) != BQ_OK) return fail(s);
    // the number of kept inner nodes decides the output size
    uint32_t hostTotal = 0, hostNv = 0;
    cudaMemcpyAsync(&hostTotal, total, 4, cudaMemcpyDeviceToHost, al.s);
    cudaMemcpyAsync(&hostNv, &st->numValid, 4, cudaMemcpyDeviceToHost, al.s);
    if ((ce = cudaStreamSynchronize(al.s)) != cudaSuccess) return fail(cuda_error(ce, "build sync"));
    const uint64_t numNodes = hostNv > (uint32_t)thr ? 2ull + 2ull * hostTotal : 2ull;
    if ((s = al.get(&nodes, numNodes)) != BQ_OK) return fail(s);
    k_collapse<<<div_up(n, 256), 256, 0, al.s>>>(full, ranges, kept, rank, &st->numValid, thr, nodes);
    if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_error(ce, "k_collapse"));
    if (hostNv > 0) bvh->numNodes = (uint32_t)numNodes;
    if (longRuns && (ce = read_back()) != cudaSuccess) return fail(cuda_error(ce, "build sync"));
  }
  if (h.err & DEV_ERR_TIMEOUT) return fail(set_error(BQ_ERR_TIMEOUT, "radix sort look-back timed out"));
  if (h.err) return fail(set_error(BQ_ERR_CUDA, "device-side range check failed in the Morton build"));
  al.free_bytes(idsOther);
  if (h.nv == 0) {
    al.free_bytes(ids);
    al.free_bytes(nodes);
    bvh->numNodes = 0;
    return BQ_OK;
  }
  bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
  bvh->primIDs = ids;
  bvh->numPrims = h.nv;
  if (thr == 1) bvh->numNodes = 2 * h.nv;
  return BQ_OK;
}

} // namespace bq
