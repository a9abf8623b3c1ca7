// bq_rebin.cu -- rebinning Morton builder with 30-bit keys (the
// cuBQL::cuda::rebinRadixBuilder method, cuBQL/builder/cuda/
// rebinMortonBuilder.h:1161-1488).
//
// The reference's tree, restated so that it can be built bottom-up:
//   * keys are 30-bit Morton codes of the centroids quantised over the
//     centroid bounds (Quantizer<float,3>, :33-61); prims sorted by key;
//   * a node [b, e) with more than `thr` prims splits at the first key that
//     has the highest bit in which its first and last key differ (findSplit,
//     :566-590), i.e. at the highest-differing adjacent pair inside it;
//   * a node whose keys are all equal -- which is exactly a maximal run of
//     equal keys, since no split ever separates two equal keys -- gets new
//     keys quantised over its own centroid bounds (or its local index when
//     those bounds are a single point) and is split again:
//       - more than 32 prims: "broad phase" rebin, a stable sort of the new
//         keys (:1022-1063, :1306-1380);
//       - at most 32 prims: "thread phase", one thread recomputes the keys
//         and applies the reference's exchange sort (:756-764, :766-872),
//         which is not stable, so its exact swap order is kept; a node whose
//         new keys are still all equal becomes a leaf of any size.
// Here every adjacent pair gets a 16-bit split level that orders all these
// splits: a pair resolved at rebin depth d by key bit h gets
// 64 + (REBIN_MAX_DEPTH - d) * 32 + h (a deeper rebin happens inside a node
// of the shallower one, so its levels are lower), a pair split by the
// thread phase at recursion depth r inside its run gets 32 - r, and pairs
// never split get 0 (they lie inside leaves).  The tree is then the same
// max-rooted Cartesian tree as for the 63-bit builder, built by the shared
// bottom-up agglomeration (bq_agglom.cuh) and collapsed to the leaf
// threshold; thread-phase leaves above the threshold are flagged per pair.
//
// Deviation: the reference restarts the broad phase forever when a run's
// centroid bounds are not a single point but narrower than 1e-20 (all new
// keys equal again).  Here the rebin depth is capped at REBIN_MAX_DEPTH;
// a run still unresolved there is keyed by its local index, as if its
// bounds were a single point.
#include <algorithm>
#include <climits>
#include <cfloat>

#include "bq_agglom.cuh"
#include "bq_internal.cuh"

namespace bq {

namespace {

constexpr int REBIN_MAX_DEPTH = 40;
constexpr int REBIN_THREAD_MAX = 32;  // smallEnoughToLeaveBroadPhase (:629-636)

__host__ __device__ constexpr uint16_t broad_level(int depth, int bit)
{
  return (uint16_t)(64 + (REBIN_MAX_DEPTH - depth) * 32 + bit);
}

// box.center() = (lower+upper)/2 (cuBQL/math/box.h:146-147), as a multiply
// by 0.5 (the same float: both round the same real number)
__device__ __forceinline__ float3 rb_center(const bq_box3f *__restrict__ boxes, uint32_t id)
{
  const float2 *bp = reinterpret_cast<const float2 *>(boxes + id);
  const float2 p0 = __ldg(bp), p1 = __ldg(bp + 1), p2 = __ldg(bp + 2);
  return make_float3(__fmul_rn(__fadd_rn(p0.x, p1.y), 0.5f), __fmul_rn(__fadd_rn(p0.y, p2.x), 0.5f),
                     __fmul_rn(__fadd_rn(p1.x, p2.y), 0.5f));
}

// Quantizer<float,3>::init over [lo, hi] (rebinMortonBuilder.h:40-47):
// scale = 1024 * rcp(max(max extent, 1e-20))
struct Quant30 {
  float bx, by, bz, scale;
};
__device__ __forceinline__ Quant30 make_quant30(float lx, float ly, float lz, float hx, float hy, float hz)
{
  const float ext = fmaxf(fmaxf(__fsub_rn(hx, lx), __fsub_rn(hy, ly)), __fsub_rn(hz, lz));
  return Quant30{lx, ly, lz, __fmul_rn(1024.0f, __fdiv_rn(1.0f, fmaxf(ext, 1e-20f)))};
}
__device__ __forceinline__ uint32_t morton30(const float3 c, const Quant30 &q)
{
  return spread10(quant_cell(c.x, q.bx, q.scale, 1023u)) | (spread10(quant_cell(c.y, q.by, q.scale, 1023u)) << 1) |
         (spread10(quant_cell(c.z, q.bz, q.scale, 1023u)) << 2);
}

// ------------------------------------------------------------------
// initial keys
// ------------------------------------------------------------------
// grid-stride, blocks of 256; centroid bounds merged once per block
__global__ void __launch_bounds__(256) k_rb_valid(const bq_box3f *__restrict__ boxes, uint32_t n,
                                                  uint32_t *__restrict__ valid,
                                                  int32_t *bounds /* lo xyz, hi xyz, encoded */)
{
  griddep_wait();
  int32_t lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const bq_box3f b = boxes[i];
    const bool have = !(b.lower[0] > b.upper[0]);  // box.empty() tests lower.x > upper.x
    valid[i] = have ? 1u : 0u;
    if (have) {
      const float3 c = rb_center(boxes, (uint32_t)i);
      const int32_t e[3] = {enc_f(c.x), enc_f(c.y), enc_f(c.z)};
#pragma unroll
      for (int d = 0; d < 3; d++) { lo[d] = min(lo[d], e[d]); hi[d] = max(hi[d], e[d]); }
    }
  }
  block_merge_bounds<256>(lo, hi, bounds);
}

__global__ void k_rb_keys(const bq_box3f *__restrict__ boxes, uint32_t n, const uint32_t *__restrict__ valid,
                          const uint32_t *__restrict__ vpos, const int32_t *__restrict__ bounds,
                          uint32_t *__restrict__ keys, uint32_t *__restrict__ ids)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !valid[i]) return;
  const Quant30 q = make_quant30(dec_f(bounds[0]), dec_f(bounds[1]), dec_f(bounds[2]), dec_f(bounds[3]),
                                 dec_f(bounds[4]), dec_f(bounds[5]));
  const uint32_t p = vpos[i];
  keys[p] = morton30(rb_center(boxes, i), q);
  ids[p] = i;
}

__global__ void k_rb_levels0(const uint32_t *__restrict__ keys, const uint32_t *nvPtr, uint16_t *__restrict__ lev)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  if (i + 1 < nv) {
    const uint32_t x = keys[i] ^ keys[i + 1];
    lev[i] = x ? broad_level(0, 31 - __clz(x)) : (uint16_t)0;
  }
}

// ------------------------------------------------------------------
// runs: maximal ranges whose inner pairs are all unresolved (level 0)
// ------------------------------------------------------------------
__global__ void k_rb_run_flags(const uint16_t *__restrict__ lev, const uint32_t *nvPtr, uint32_t *__restrict__ flag)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  flag[i] = (i == 0 || lev[i - 1] != 0) ? 1u : 0u;
}

__global__ void k_rb_run_starts(const uint32_t *__restrict__ flag, const uint32_t *__restrict__ runIdx,
                                const uint32_t *nvPtr, uint32_t *__restrict__ starts)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  if (flag[i]) starts[runIdx[i]] = i;
  if (i == nv - 1) starts[runIdx[i] + flag[i]] = nv;
}

// per run: is it rebinned by the broad phase?
__global__ void k_rb_big(const uint32_t *__restrict__ starts, const uint32_t *numRunsPtr, uint32_t bigMin,
                         uint32_t *__restrict__ big, uint32_t *__restrict__ bigSize)
{
  griddep_wait();
  const uint32_t R = *numRunsPtr;
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const uint32_t size = starts[r + 1] - starts[r];
  const bool b = size > bigMin;
  big[r] = b ? 1u : 0u;
  bigSize[r] = b ? size : 0u;
}

struct RebinJob {
  uint32_t start, size, off;  // prim range [start, start+size); first compacted slot
  int32_t lo[3], hi[3];       // centroid bounds (encoded)
};

__global__ void k_rb_jobs(const uint32_t *__restrict__ starts, const uint32_t *numRunsPtr,
                          const uint32_t *__restrict__ big, const uint32_t *__restrict__ bigRank,
                          const uint32_t *__restrict__ bigOff, RebinJob *__restrict__ jobs,
                          uint32_t *__restrict__ jobOff)
{
  griddep_wait();
  const uint32_t R = *numRunsPtr;
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R || !big[r]) return;
  RebinJob j;
  j.start = starts[r];
  j.size = starts[r + 1] - starts[r];
  j.off = bigOff[r];
  for (int d = 0; d < 3; d++) { j.lo[d] = INT_MAX; j.hi[d] = INT_MIN; }
  jobs[bigRank[r]] = j;
  jobOff[bigRank[r]] = j.off;
}

// the job of compacted slot t: last job whose offset is <= t
__device__ __forceinline__ uint32_t job_of(const uint32_t *__restrict__ jobOff, uint32_t numJobs, uint32_t t)
{
  uint32_t lo = 0, hi = numJobs;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (__ldg(jobOff + m) <= t) lo = m; else hi = m;
  }
  return lo;
}

// rebinGrowDomains (:960-990): centroid bounds per job
__global__ void k_rb_domains(RebinJob *jobs, const uint32_t *__restrict__ jobOff, uint32_t numJobs,
                             uint32_t numSlots, const uint32_t *__restrict__ ids, const bq_box3f *__restrict__ boxes)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = t < numSlots;
  uint32_t q = 0;
  int32_t e[3] = {INT_MAX, INT_MAX, INT_MAX};
  if (in) {
    q = job_of(jobOff, numJobs, t);
    const RebinJob &j = jobs[q];
    const float3 c = rb_center(boxes, ids[j.start + (t - j.off)]);
    e[0] = enc_f(c.x); e[1] = enc_f(c.y); e[2] = enc_f(c.z);
  }
  const uint32_t q0 = __shfl_sync(0xffffffffu, q, 0);
  const bool uniform = __all_sync(0xffffffffu, !in || q == q0);
  if (uniform) {  // common case (jobs are large): one atomic per warp and component
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int32_t mn = __reduce_min_sync(0xffffffffu, in ? e[d] : INT_MAX);
      const int32_t mx = __reduce_max_sync(0xffffffffu, in ? e[d] : INT_MIN);
      if ((threadIdx.x & 31) == 0 && mn <= mx) {
        atomicMin(&jobs[q0].lo[d], mn);
        atomicMax(&jobs[q0].hi[d], mx);
      }
    }
  } else if (in) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      atomicMin(&jobs[q].lo[d], e[d]);
      atomicMax(&jobs[q].hi[d], e[d]);
    }
  }
}

// rebinCreateNewKeysAndPrimIDs (:1022-1063): composite (job, new key)
__global__ void k_rb_newkeys(const RebinJob *__restrict__ jobs, const uint32_t *__restrict__ jobOff,
                             uint32_t numJobs, uint32_t numSlots, const uint32_t *__restrict__ ids,
                             const bq_box3f *__restrict__ boxes, bool atDepthCap, uint64_t *__restrict__ kk,
                             uint32_t *__restrict__ vv)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numSlots) return;
  const uint32_t q = job_of(jobOff, numJobs, t);
  const RebinJob j = jobs[q];
  const uint32_t local = t - j.off;
  const uint32_t id = ids[j.start + local];
  const bool point = j.lo[0] == j.hi[0] && j.lo[1] == j.hi[1] && j.lo[2] == j.hi[2];
  uint32_t key = local;
  if (!point && !atDepthCap) {
    const Quant30 qz = make_quant30(dec_f(j.lo[0]), dec_f(j.lo[1]), dec_f(j.lo[2]), dec_f(j.hi[0]),
                                    dec_f(j.hi[1]), dec_f(j.hi[2]));
    key = morton30(rb_center(boxes, id), qz);
  }
  kk[t] = ((uint64_t)q << 32) | key;
  vv[t] = id;
}

// rebinWriteBackNewKeysAndPrimIDs (:1000-1020)
__global__ void k_rb_writeback(const RebinJob *__restrict__ jobs, const uint32_t *__restrict__ jobOff,
                               uint32_t numSlots, const uint64_t *__restrict__ kk, const uint32_t *__restrict__ vv,
                               uint32_t *__restrict__ keys, uint32_t *__restrict__ ids)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numSlots) return;
  const uint64_t k = kk[t];
  const uint32_t q = (uint32_t)(k >> 32);
  const uint32_t pos = jobs[q].start + (t - jobOff[q]);
  keys[pos] = (uint32_t)k;
  ids[pos] = vv[t];
}

__global__ void k_rb_newlevels(const RebinJob *__restrict__ jobs, const uint32_t *__restrict__ jobOff,
                               uint32_t numJobs, uint32_t numSlots, const uint32_t *__restrict__ keys, int depth,
                               uint16_t *__restrict__ lev)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numSlots) return;
  const uint32_t q = job_of(jobOff, numJobs, t);
  const RebinJob j = jobs[q];
  const uint32_t local = t - j.off;
  if (local + 1 >= j.size) return;
  const uint32_t pos = j.start + local;
  const uint32_t x = keys[pos] ^ keys[pos + 1];
  lev[pos] = x ? broad_level(depth, 31 - __clz(x)) : (uint16_t)0;
}

// ------------------------------------------------------------------
// thread phase (threadPhaseCreateNodes, :766-872): one thread per run of
// thr < size <= 32 equal keys
// ------------------------------------------------------------------
// If position i starts a run of at least two prims (level 0 between them),
// its size, counted up to `cap` + 1 at most; else 0.
__device__ __forceinline__ uint32_t run_size_at(const uint16_t *__restrict__ lev, uint32_t i, uint32_t nv, uint32_t cap)
{
  if (i + 1 >= nv || (i > 0 && lev[i - 1] == 0) || lev[i] != 0) return 0;
  uint32_t size = 2;
  while (size <= cap && i + size - 1 < nv - 1 && lev[i + size - 1] == 0) size++;
  return size;
}

// counts the runs the broad phase must rebin (more than bigMin prims)
__global__ void k_rb_detect(const uint16_t *__restrict__ lev, const uint32_t *nvPtr, uint32_t bigMin,
                            uint32_t *numBig)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  if (run_size_at(lev, i, nv, bigMin) > bigMin) atomicAdd(numBig, 1u);
}

// the run [start, start + size) of thr < size <= 32 prims, by one thread
__device__ void rb_thread_run(uint32_t start, uint32_t size, int thr, const bq_box3f *__restrict__ boxes,
                              uint32_t *__restrict__ ids, uint16_t *__restrict__ lev, uint8_t *__restrict__ forced,
                              uint32_t *numForced)
{
  if (size == 2) {
    // the common case (pairs of identical or near prims): the steps below
    // for two prims, each centroid read once
    const uint32_t i0 = ids[start], i1 = ids[start + 1];
    const float3 c0 = rb_center(boxes, i0), c1 = rb_center(boxes, i1);
    uint32_t k0 = 0, k1 = 1;  // a point domain keys by position
    if (!(c0.x == c1.x && c0.y == c1.y && c0.z == c1.z)) {
      const Quant30 q = make_quant30(fminf(c0.x, c1.x), fminf(c0.y, c1.y), fminf(c0.z, c1.z), fmaxf(c0.x, c1.x),
                                     fmaxf(c0.y, c1.y), fmaxf(c0.z, c1.z));
      k0 = morton30(c0, q);
      k1 = morton30(c1, q);
    }
    if (k1 < k0) {  // the exchange sort of two keys
      ids[start] = i1;
      ids[start + 1] = i0;
    }
    if (k0 == k1) {
      forced[start] = 1;
      atomicAdd(numForced, 1u);
    } else {
      lev[start] = (uint16_t)32;  // split at depth 0 of the run
    }
    return;
  }
  uint32_t key[REBIN_THREAD_MAX], id[REBIN_THREAD_MAX];
  for (uint32_t i = 0; i < size; i++) {
    key[i] = 0;  // the run's keys are all equal: only equality matters below
    id[i] = ids[start + i];
  }
  struct Item {
    uint8_t b, e, depth;
  };
  Item stack[REBIN_THREAD_MAX];
  int sp = 0;
  stack[sp++] = Item{0, (uint8_t)size, 0};
  while (sp > 0) {
    const Item it = stack[--sp];
    const uint32_t b = it.b, e = it.e;
    if ((int64_t)(e - b) <= thr) continue;  // leaf
    if (key[b] == key[e - 1]) {
      // no split with the current keys: new keys over this node's centroid bounds
      float lx = FLT_MAX, ly = FLT_MAX, lz = FLT_MAX, hx = -FLT_MAX, hy = -FLT_MAX, hz = -FLT_MAX;
      for (uint32_t i = b; i < e; i++) {
        const float3 c = rb_center(boxes, id[i]);
        lx = fminf(lx, c.x); ly = fminf(ly, c.y); lz = fminf(lz, c.z);
        hx = fmaxf(hx, c.x); hy = fmaxf(hy, c.y); hz = fmaxf(hz, c.z);
      }
      if (lx == hx && ly == hy && lz == hz) {
        for (uint32_t i = b; i < e; i++) key[i] = i - b;
      } else {
        const Quant30 q = make_quant30(lx, ly, lz, hx, hy, hz);
        for (uint32_t i = b; i < e; i++) key[i] = morton30(rb_center(boxes, id[i]), q);
      }
      for (uint32_t i = b; i < e; i++)  // bubbleSort (:756-764): exchange order matters, it is not stable
        for (uint32_t j = i + 1; j < e; j++)
          if (key[j] < key[i]) {
            const uint32_t tk = key[i]; key[i] = key[j]; key[j] = tk;
            const uint32_t ti = id[i]; id[i] = id[j]; id[j] = ti;
          }
      if (key[b] == key[e - 1]) {  // still no split: a leaf, whatever its size
        for (uint32_t i = b; i + 1 < e; i++) forced[start + i] = 1;
        atomicAdd(numForced, 1u);
        continue;
      }
    }
    // findSplit: first key with the highest differing bit set
    const uint32_t x = key[b] ^ key[e - 1];
    const uint32_t hb = 31 - __clz(x);
    uint32_t sp2 = b + 1;
    while (sp2 < e && !((key[sp2] ^ key[b]) >> hb)) sp2++;
    lev[start + sp2 - 1] = (uint16_t)(32 - it.depth);
    stack[sp++] = Item{(uint8_t)sp2, (uint8_t)e, (uint8_t)(it.depth + 1)};
    stack[sp++] = Item{(uint8_t)b, (uint8_t)sp2, (uint8_t)(it.depth + 1)};
  }
  for (uint32_t i = 0; i < size; i++) ids[start + i] = id[i];
}

// The thread phase runs as two kernels: the levels are read to find the
// runs before any run writes its new levels (a finder that ran beside the
// run work could mistake a half-written run for a new one).
// k_rb_find_runs: each warp looks at RT_ITEMS * 32 consecutive positions
// and appends the runs of thr < size <= 32 prims that start there (one
// atomic per warp); k_rb_thread then gives one listed run to each thread.
constexpr int RT_BLOCK = 128;
constexpr int RT_ITEMS = 4;
__global__ void __launch_bounds__(RT_BLOCK) k_rb_find_runs(const uint32_t *nvPtr, int thr,
                                                           const uint16_t *__restrict__ lev, uint2 *__restrict__ list,
                                                           uint32_t *listCount)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t warpBase = ((uint64_t)blockIdx.x * (RT_BLOCK / 32) + warp) * (RT_ITEMS * 32);
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t size[RT_ITEMS], bal[RT_ITEMS], total = 0;
#pragma unroll
  for (int u = 0; u < RT_ITEMS; u++) {
    const uint64_t i = warpBase + (uint64_t)u * 32 + lane;
    size[u] = i < nv ? run_size_at(lev, (uint32_t)i, nv, REBIN_THREAD_MAX) : 0u;
    const bool mine = (int64_t)size[u] > thr && size[u] <= (uint32_t)REBIN_THREAD_MAX;
    bal[u] = __ballot_sync(0xffffffffu, mine);
    total += __popc(bal[u]);
  }
  if (total == 0) return;  // whole warp
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(listCount, total);
  base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
  for (int u = 0; u < RT_ITEMS; u++) {
    if ((bal[u] >> lane) & 1u) list[base + __popc(bal[u] & lt)] = make_uint2((uint32_t)(warpBase + u * 32 + lane), size[u]);
    base += __popc(bal[u]);
  }
}

__global__ void __launch_bounds__(RT_BLOCK) k_rb_thread(const uint2 *__restrict__ list, const uint32_t *listCount,
                                                        uint32_t listCap, int thr, const bq_box3f *__restrict__ boxes,
                                                        uint32_t *__restrict__ ids, uint16_t *__restrict__ lev,
                                                        uint8_t *__restrict__ forced, uint32_t *numForced)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= min(*listCount, listCap)) return;
  const uint2 r = list[t];
  rb_thread_run(r.x, r.y, thr, boxes, ids, lev, forced, numForced);
}

// ------------------------------------------------------------------
// collapse to the leaf threshold (thread-phase leaves flagged in `forced`)
// ------------------------------------------------------------------
__global__ void k_rb_kept(const uint2 *__restrict__ ranges, const uint8_t *__restrict__ forced, const uint32_t *nvPtr,
                          int thr, uint32_t *__restrict__ kept)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x + 1;  // split positions 1..nv-1
  if (s >= nv) return;
  const uint2 rg = ranges[s];
  kept[s - 1] = (rg.y - rg.x + 1 > (uint32_t)thr && !forced[s - 1]) ? 1u : 0u;
}

// is the full-tree node c (covering [cl, cr]) a leaf of the final tree?
__device__ __forceinline__ bool rb_is_leaf(const Node &c, uint32_t sz, int thr, const uint8_t *__restrict__ forced)
{
  if (sz <= (uint32_t)thr) return true;
  const uint32_t cs = (uint32_t)(admin_offset(node_admin(c)) >> 1);
  return forced[cs - 1] != 0;
}

__global__ void k_rb_collapse(const Node *__restrict__ full, const uint2 *__restrict__ ranges,
                              const uint32_t *__restrict__ kept, const uint32_t *__restrict__ rank,
                              const uint8_t *__restrict__ forced, const uint32_t *nvPtr, int thr,
                              Node *__restrict__ out)
{
  griddep_wait();
  const uint32_t nv = *nvPtr;
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    const Node root = full[0];
    uint64_t a;
    if (nv == 1 || rb_is_leaf(root, nv, thr, forced)) {
      a = make_admin(0, nv);
    } else {
      const uint32_t s0 = (uint32_t)(admin_offset(node_admin(root)) >> 1);
      a = make_admin(2ull + 2ull * rank[s0 - 1], 0);
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
    if (sz == 1 || rb_is_leaf(c, sz, thr, forced)) {
      a = make_admin(cl, sz);
    } else {
      const uint32_t cs = (uint32_t)(admin_offset(node_admin(c)) >> 1);
      a = make_admin(2ull + 2ull * rank[cs - 1], 0);
    }
    out[base + side] = make_node(c.a.x, c.a.y, c.a.z, c.a.w, c.b.x, c.b.y, a);
  }
}

} // namespace

// ------------------------------------------------------------------
// host entry
// ------------------------------------------------------------------
int build_rebin_morton30(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
{
  const int maxLeaf = cfg ? cfg->maxAllowedLeafSize : (1 << 15);
  const int mlt = cfg ? cfg->makeLeafThreshold : 0;
  const int thr = mlt > 0 ? std::min(mlt, maxLeaf) : 1;  // rebinMortonBuilder.h:1174-1177
  if (thr < 1 || thr > 65535)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "leaf threshold must be in [1, 65535] (16-bit leaf count)");
  bvh->nodes = nullptr; bvh->primIDs = nullptr; bvh->numNodes = 0; bvh->numPrims = 0;
  if (n == 0) return BQ_OK;

  TempSet tmp(al);
  uint32_t *valid = nullptr, *vpos = nullptr, *ctl = nullptr, *slot = nullptr;
  uint32_t *keysA = nullptr, *keysB = nullptr, *idsB = nullptr;
  uint16_t *lev = nullptr;
  uint8_t *forced = nullptr;
  BQ_TRY(tmp.get(&valid, n));
  BQ_TRY(tmp.get(&vpos, n));
  BQ_TRY(tmp.get(&ctl, 16));  // [0] nv [1] err [2..7] bounds [8] runs [9] jobs [10] job prims [11] thread leaves
                              // [12] thread-phase runs
  BQ_TRY(tmp.get(&keysA, n));
  BQ_TRY(tmp.get(&keysB, n));
  BQ_TRY(tmp.get(&idsB, n));
  BQ_TRY(tmp.get(&lev, n));
  BQ_TRY(tmp.get(&forced, n));
  BQ_TRY(tmp.get(&slot, n));
  uint32_t *idsA = nullptr;
  Node *nodes = nullptr;
  BQ_TRY(al.get(&idsA, n));
  auto fail = [&](int code) {
    al.free_bytes(idsA);
    al.free_bytes(nodes);
    return code;
  };
  int s;
  cudaError_t ce;
  const int32_t ctlInit[8] = {0, 0, INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  if ((ce = cudaMemcpyAsync(ctl, ctlInit, 32, cudaMemcpyHostToDevice, al.s)) != cudaSuccess ||
      (ce = cudaMemsetAsync(forced, 0, n, al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "rebin set-up"));
  uint32_t *nvDev = ctl;
  int32_t *bounds = (int32_t *)(ctl + 2);
  {
    ProfScope ps("rebin.keys", al.s, 5);
    launch_pdl(k_rb_valid, dim3(std::min(div_up(n, 256), num_sms() * 8)), dim3(256), 0, al.s, boxes, n, valid,
               bounds);
    if ((s = exclusive_scan_u32(valid, vpos, n, nullptr, nvDev, al)) != BQ_OK) return fail(s);
    launch_pdl(k_rb_keys, dim3(div_up(n, 256)), dim3(256), 0, al.s, boxes, n, valid, vpos, bounds, keysA, idsA);
  }
  uint32_t *keys2[2] = {keysA, keysB};
  uint32_t *ids2[2] = {idsA, idsB};
  int sel = 0;
  if ((s = onesweep_sort_u32(keys2, ids2, n, nvDev, 0, 30, nullptr, &sel, ctl + 1, al)) != BQ_OK) return fail(s);
  uint32_t *keys = keys2[sel];
  uint32_t *ids = ids2[sel];
  if (sel) {  // keep the result in the caller-owned buffer
    if ((ce = cudaMemcpyAsync(idsA, idsB, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "copy"));
    ids = idsA;
  }
  {
    ProfScope ps("rebin.levels", al.s);
    launch_pdl(k_rb_levels0, dim3(div_up(n, 256)), dim3(256), 0, al.s, keys, nvDev, lev);
  }
  // ---- broad-phase rebinning ----
  uint32_t *flag = nullptr, *runIdx = nullptr, *starts = nullptr, *big = nullptr, *bigSize = nullptr;
  uint32_t *bigRank = nullptr, *bigOff = nullptr, *jobOff = nullptr, *vv[2] = {nullptr, nullptr};
  uint64_t *kk[2] = {nullptr, nullptr};
  RebinJob *jobs = nullptr;
  const uint32_t bigMin = (uint32_t)std::max(REBIN_THREAD_MAX, thr);
  uint32_t hnv = 0;
  for (int depth = 0;; depth++) {
    // one cheap pass decides whether any run still needs a broad-phase rebin
    if ((ce = cudaMemsetAsync(ctl + 9, 0, 4, al.s)) != cudaSuccess) return fail(cuda_error(ce, "memset"));
    {
      ProfScope ps("rebin.detect", al.s);
      launch_pdl(k_rb_detect, dim3(div_up(n, 256)), dim3(256), 0, al.s, lev, nvDev, bigMin, ctl + 9);
    }
    uint32_t h[10];
    if ((ce = cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "rebin runs"));
    hnv = h[0];
    if (h[1] & DEV_ERR_TIMEOUT) return fail(set_error(BQ_ERR_TIMEOUT, "radix sort look-back timed out"));
    if (h[1]) return fail(set_error(BQ_ERR_CUDA, "device-side range check failed in the rebin build"));
    if (hnv == 0 || h[9] == 0) break;
    // list the runs and the ones to rebin (their prims, compacted)
    if (!jobs) {
      if ((s = tmp.get(&flag, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&runIdx, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&starts, n + 1ull)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&big, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&bigSize, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&bigRank, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&bigOff, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&jobs, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&jobOff, n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&kk[0], n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&kk[1], n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&vv[0], n)) != BQ_OK) return fail(s);
      if ((s = tmp.get(&vv[1], n)) != BQ_OK) return fail(s);
    }
    {
      ProfScope ps("rebin.runs", al.s, 12);
      launch_pdl(k_rb_run_flags, dim3(div_up(n, 256)), dim3(256), 0, al.s, lev, nvDev, flag);
      if ((s = exclusive_scan_u32(flag, runIdx, n, nvDev, ctl + 8, al)) != BQ_OK) return fail(s);
      launch_pdl(k_rb_run_starts, dim3(div_up(n, 256)), dim3(256), 0, al.s, flag, runIdx, nvDev, starts);
      launch_pdl(k_rb_big, dim3(div_up(n, 256)), dim3(256), 0, al.s, starts, ctl + 8, bigMin, big, bigSize);
      if ((s = exclusive_scan_u32(big, bigRank, n, ctl + 8, ctl + 9, al)) != BQ_OK) return fail(s);
      if ((s = exclusive_scan_u32(bigSize, bigOff, n, ctl + 8, ctl + 10, al)) != BQ_OK) return fail(s);
    }
    uint32_t hj[2];
    if ((ce = cudaMemcpyAsync(hj, ctl + 9, sizeof(hj), cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "rebin runs"));
    const uint32_t numJobs = hj[0], numSlots = hj[1];
    const int next = depth + 1;
    const bool cap = next >= REBIN_MAX_DEPTH;
    ProfScope ps2("rebin.rebin", al.s, 5);
    launch_pdl(k_rb_jobs, dim3(div_up(n, 256)), dim3(256), 0, al.s, starts, ctl + 8, big, bigRank, bigOff, jobs,
               jobOff);
    launch_pdl(k_rb_domains, dim3(div_up(numSlots, 256)), dim3(256), 0, al.s, jobs, jobOff, numJobs, numSlots, ids,
               boxes);
    launch_pdl(k_rb_newkeys, dim3(div_up(numSlots, 256)), dim3(256), 0, al.s, jobs, jobOff, numJobs, numSlots, ids,
               boxes, cap, kk[0], vv[0]);
    int jobBits = 0;
    while (jobBits < 32 && (numJobs - 1) >> jobBits) jobBits++;
    int ksel = 0;
    if ((s = onesweep_sort_u64(kk, vv, numSlots, nullptr, 0, 32 + jobBits, nullptr, &ksel, ctl + 1, al)) != BQ_OK)
      return fail(s);
    launch_pdl(k_rb_writeback, dim3(div_up(numSlots, 256)), dim3(256), 0, al.s, jobs, jobOff, numSlots, kk[ksel],
               vv[ksel], keys, ids);
    launch_pdl(k_rb_newlevels, dim3(div_up(numSlots, 256)), dim3(256), 0, al.s, jobs, jobOff, numJobs, numSlots, keys,
               next, lev);
    if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_error(ce, "rebin"));
  }
  if (hnv == 0) {
    al.free_bytes(idsA);
    return BQ_OK;
  }
  // ---- thread phase ----
  if ((ce = cudaMemsetAsync(ctl + 11, 0, 4, al.s)) != cudaSuccess) return fail(cuda_error(ce, "memset"));
  if (thr < REBIN_THREAD_MAX) {
    ProfScope ps("rebin.thread", al.s, 2);
    // runs of at least two prims: at most hnv / 2 of them
    const uint32_t listCap = hnv / 2 + 1;
    uint2 *list = nullptr;
    if ((s = tmp.get(&list, listCap)) != BQ_OK) return fail(s);
    if ((ce = cudaMemsetAsync(ctl + 12, 0, 4, al.s)) != cudaSuccess) return fail(cuda_error(ce, "memset"));
    launch_pdl(k_rb_find_runs, dim3(div_up(hnv, RT_BLOCK * RT_ITEMS)), dim3(RT_BLOCK), 0, al.s, nvDev, thr, lev, list,
               ctl + 12);
    launch_pdl(k_rb_thread, dim3(div_up(listCap, RT_BLOCK)), dim3(RT_BLOCK), 0, al.s, list, ctl + 12, listCap, thr,
               boxes, ids, lev, forced, ctl + 11);
  }
  uint2 *pending = nullptr;
  if ((s = tmp.get(&pending, 2ull * div_up(hnv, AGG_CHUNK))) != BQ_OK) return fail(s);
  // ---- leaf threshold 1: the full tree is the result unless the thread
  // phase made leaves of several prims ----
  if (thr == 1) {
    if ((s = al.get(&nodes, 2ull * hnv)) != BQ_OK) return fail(s);
    {
      AggArgsT<uint16_t> ag{lev, slot, ids, boxes, nodes, nullptr, nvDev, nullptr, pending, nullptr, 0};
      if ((s = agglomerate<false>(ag, hnv, al.s, "rebin.agg_local", "rebin.agg_global")) != BQ_OK) return fail(s);
    }
    uint32_t hf[12];
    if ((ce = cudaMemcpyAsync(hf, ctl, sizeof(hf), cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
      return fail(cuda_error(ce, "rebin sync"));
    if (hf[1]) return fail(set_error(BQ_ERR_CUDA, "device-side check failed in the rebin build"));
    if (hf[11] == 0) {
      bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
      bvh->numNodes = 2 * hnv;
      bvh->primIDs = ids;
      bvh->numPrims = hnv;
      return BQ_OK;
    }
    al.free_bytes(nodes);  // rare: multi-prim leaves, go through the collapse below
    nodes = nullptr;
  }
  // ---- full tree, then collapse ----
  Node *full = nullptr;
  uint2 *ranges = nullptr;
  uint32_t *kept = nullptr, *rank = nullptr;
  if ((s = tmp.get(&full, 2ull * hnv)) != BQ_OK) return fail(s);
  if ((s = tmp.get(&ranges, hnv)) != BQ_OK) return fail(s);
  if ((s = tmp.get(&kept, hnv)) != BQ_OK) return fail(s);
  if ((s = tmp.get(&rank, hnv)) != BQ_OK) return fail(s);
  {
    AggArgsT<uint16_t> ag{lev, slot, ids, boxes, full, nullptr, nvDev, ranges, pending, nullptr, 0};
    if ((s = agglomerate<false>(ag, hnv, al.s, "rebin.agg_local", "rebin.agg_global")) != BQ_OK) return fail(s);
  }
  if ((ce = cudaMemsetAsync(kept, 0, sizeof(uint32_t) * hnv, al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "memset"));
  {
    ProfScope ps("rebin.collapse", al.s, 4);
    launch_pdl(k_rb_kept, dim3(div_up(hnv, 256)), dim3(256), 0, al.s, ranges, forced, nvDev, thr, kept);
    if ((s = exclusive_scan_u32(kept, rank, hnv > 1 ? hnv - 1 : 1, nullptr, ctl + 9, al)) != BQ_OK) return fail(s);
  }
  uint32_t hk[2];
  if ((ce = cudaMemcpyAsync(hk, ctl + 8, 8, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess ||
      (ce = cudaStreamSynchronize(al.s)) != cudaSuccess)
    return fail(cuda_error(ce, "rebin sync"));
  // the root is internal unless it is a leaf by size or a thread-phase leaf
  // (then no split is kept); otherwise every kept split owns a node pair
  const uint64_t numNodes = 2ull + 2ull * hk[1];
  if ((s = al.get(&nodes, numNodes)) != BQ_OK) return fail(s);
  launch_pdl(k_rb_collapse, dim3(div_up(hnv, 256)), dim3(256), 0, al.s, full, ranges, kept, rank, forced, nvDev, thr,
             nodes);
  if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_error(ce, "k_rb_collapse"));
  bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
  bvh->numNodes = (uint32_t)numNodes;
  bvh->primIDs = ids;
  bvh->numPrims = hnv;
  return BQ_OK;
}

} // namespace bq
