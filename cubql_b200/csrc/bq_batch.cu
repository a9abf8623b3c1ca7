// bq_batch.cu -- many point clouds built and queried in one pass.
//
// A batch is numSegs clouds of uneven size stored back to back; segment s
// owns boxes[off[s] .. off[s+1]).  The reference has no batched entry
// point: a user loops cuda::radixBuilder + a findKNN kernel per cloud
// (cuBQL/builder/cuda/radix.h:591-771, cuBQL/queries/points/knn.h:75-116).
// Here the whole batch goes through one fixed sequence of launches with no
// host synchronisation (so it can be captured in a CUDA graph):
//
//   k_seg_bounds_init / k_seg_bounds / k_seg_quant
//                    per-cloud centroid bounds and quantizer (the same
//                    formulas as the single build, per cloud)
//   k_seg_keygen     63-bit Morton key of every prim in its cloud's frame
//   onesweep x 8     stable sort by Morton key over the whole batch
//   k_seg_ids + onesweep x ceil(segBits/8)
//                    stable sort by cloud id: the result is ordered by
//                    (cloud, key) -- the 72-bit composite key sorted as
//                    Morton passes followed by cloud passes
//   k_seg_gather     keys and prim ids in final order
//   k_seg_delta / k_seg_agglomerate
//                    the bottom-up builder of bq_morton.cu with every climb
//                    stopped at its cloud's boundaries
//   (leaf threshold > 1: k_kept-style collapse with per-cloud ranks)
//   k_seg_desc       one BinaryBVH descriptor per cloud
// Every per-cloud tree equals bq_build_morton63_f3 on that cloud alone
// (node layout relative to the cloud's node block; primIDs local to the
// cloud).  Clouds with empty boxes are not supported in batches.
//
// Batched kNN: queries are also stored cloud by cloud; they are sorted by
// (cloud, 30-bit Morton code in the cloud's root box) and answered by a
// persistent work-stealing kernel (one CTA per SM slot; warps grab chunks
// of `queriesPerWarp` queries from a global counter until the batch is
// exhausted), which keeps all SMs busy despite very uneven clouds.
#include <algorithm>
#include <climits>
#include <cfloat>

#include "bq_agglom.cuh"
#include "bq_traverse.cuh"

namespace bq {
int query_config(const bq_query_config *q, bq_query_config &out);

namespace {

__device__ __forceinline__ uint32_t seg_of(const uint32_t *__restrict__ off, uint32_t numSegs, uint32_t i)
{
  // largest s with off[s] <= i
  uint32_t lo = 0, hi = numSegs;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (__ldg(off + m) <= i) lo = m; else hi = m;
  }
  return lo;
}

// box center (lower + upper) / 2, as a multiply by 0.5: the same float
__device__ __forceinline__ float ctr(float lo, float hi) { return __fmul_rn(__fadd_rn(lo, hi), 0.5f); }

struct SegQuant {
  float bias[3];
  float scale;
};

__global__ void k_seg_bounds_init(int32_t *segLoHi, uint32_t numSegs)
{
  griddep_wait();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= numSegs) return;
  for (int d = 0; d < 3; d++) {
    segLoHi[6 * s + d] = INT_MAX;
    segLoHi[6 * s + 3 + d] = INT_MIN;
  }
}

// per-block pre-reduction of runs of equal segments, then one atomic per
// (block, segment, component)
__global__ void __launch_bounds__(256) k_seg_bounds(const bq_box3f *__restrict__ boxes, uint32_t n,
                                                    const uint32_t *__restrict__ off, uint32_t numSegs,
                                                    int32_t *segLoHi)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  uint32_t s = valid ? seg_of(off, numSegs, i) : 0xffffffffu;
  int32_t v[6];
  if (valid) {
    const bq_box3f b = boxes[i];
    for (int d = 0; d < 3; d++) {
      v[d] = enc_f(ctr(b.lower[d], b.upper[d]));
      v[3 + d] = v[d];
    }
  }
  // warp-level: lanes sharing the warp's first segment reduce together
  const uint32_t s0 = __shfl_sync(0xffffffffu, s, 0);
  const bool same = valid && s == s0;
  const uint32_t m = __ballot_sync(0xffffffffu, same);
  for (int d = 0; d < 6; d++) {
    int32_t x = same ? v[d] : (d < 3 ? INT_MAX : INT_MIN);
    x = d < 3 ? __reduce_min_sync(0xffffffffu, x) : __reduce_max_sync(0xffffffffu, x);
    if (same && (threadIdx.x & 31) == (uint32_t)(__ffs(m) - 1)) {
      if (d < 3) atomicMin(&segLoHi[6 * s0 + d], x);
      else atomicMax(&segLoHi[6 * s0 + d], x);
    }
  }
  if (valid && !same) {
    for (int d = 0; d < 3; d++) {
      atomicMin(&segLoHi[6 * s + d], v[d]);
      atomicMax(&segLoHi[6 * s + 3 + d], v[3 + d]);
    }
  }
}

__global__ void k_seg_quant(const int32_t *__restrict__ segLoHi, uint32_t numSegs, SegQuant *__restrict__ q)
{
  griddep_wait();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= numSegs) return;
  float lo[3], sz[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = dec_f(segLoHi[6 * s + d]);
    sz[d] = __fsub_rn(dec_f(segLoHi[6 * s + 3 + d]), lo[d]);
  }
  const float ext = fmaxf(fmaxf(sz[0], sz[1]), sz[2]);
  const float rc = __fdiv_rn(1.0f, fmaxf(ext, 1e-20f));
  SegQuant r;
  for (int d = 0; d < 3; d++) r.bias[d] = lo[d];
  r.scale = __fmul_rn(2097152.0f, rc);
  q[s] = r;
}

__global__ void __launch_bounds__(256) k_seg_keygen(const bq_box3f *__restrict__ boxes, uint32_t n,
                                                    const uint32_t *__restrict__ off, uint32_t numSegs,
                                                    const SegQuant *__restrict__ quant, uint64_t *__restrict__ keys,
                                                    uint32_t *__restrict__ ids, uint32_t *__restrict__ hist)
{
  griddep_wait();
  __shared__ uint32_t sh[8 * 256];
  for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) sh[j] = 0;
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint32_t s = seg_of(off, numSegs, i);
    const SegQuant q = quant[s];
    const bq_box3f b = boxes[i];
    const uint64_t key = spread21(quant_cell(ctr(b.lower[0], b.upper[0]), q.bias[0], q.scale, 2097151u)) |
                         (spread21(quant_cell(ctr(b.lower[1], b.upper[1]), q.bias[1], q.scale, 2097151u)) << 1) |
                         (spread21(quant_cell(ctr(b.lower[2], b.upper[2]), q.bias[2], q.scale, 2097151u)) << 2);
    keys[i] = key;
    ids[i] = i;
    for (int p = 0; p < 8; p++) atomicAdd(&sh[p * 256 + ((key >> (8 * p)) & 0xff)], 1u);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x)
    if (sh[j]) atomicAdd(&hist[j], sh[j]);
}

// cloud id of every Morton-sorted element; value = its sorted position
__global__ void k_seg_ids(const uint32_t *__restrict__ idsSorted, uint32_t n, const uint32_t *__restrict__ off,
                          uint32_t numSegs, uint32_t *__restrict__ segKey, uint32_t *__restrict__ pos)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  segKey[i] = seg_of(off, numSegs, idsSorted[i]);
  pos[i] = i;
}

__global__ void k_seg_gather(const uint32_t *__restrict__ pos, const uint64_t *__restrict__ keysMorton,
                             const uint32_t *__restrict__ idsMorton, uint32_t n, uint64_t *__restrict__ keys,
                             uint32_t *__restrict__ ids)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = pos[i];
  keys[i] = keysMorton[p];
  ids[i] = idsMorton[p];
}

// split level of the boundary between sorted positions i and i+1 inside
// the cloud [b0, e0) (same encoding as bq_morton.cu)
__device__ __forceinline__ uint8_t seg_split_level(const uint64_t *__restrict__ keys, uint32_t b0, uint32_t e0,
                                                   uint32_t i)
{
  const uint64_t a = keys[i], b = keys[i + 1];
  if (a != b) return (uint8_t)(64 + (63 - __clzll(a ^ b)));
  const uint32_t r0 = run_begin(keys, b0, i, a);
  const uint32_t r1 = run_end(keys, i + 1, e0, a);
  // the reference splits the run [r0,r1) at (b+e)/2 with cloud-local b,e
  const uint64_t s = (uint64_t)i + 1 - b0;
  uint64_t bb = r0 - b0, ee = r1 - b0;
  int depth = 0;
  while (true) {
    const uint64_t m = (bb + ee) / 2;
    if (s == m) break;
    if (s < m) ee = m; else bb = m;
    depth++;
  }
  return (uint8_t)(63 - depth);
}

__global__ void k_seg_delta(const uint64_t *__restrict__ keys, uint32_t n, const uint32_t *__restrict__ off,
                            uint32_t numSegs, uint8_t *__restrict__ delta)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = seg_of(off, numSegs, i);
  const uint32_t b0 = __ldg(off + s), e0 = __ldg(off + s + 1);
  if (i + 1 < e0) delta[i] = seg_split_level(keys, b0, e0, i);
}

// leaf threshold > 1: kept inner nodes (split positions inside clouds)
__global__ void k_seg_kept(const uint2 *__restrict__ ranges, uint32_t n, const uint32_t *__restrict__ off,
                           uint32_t numSegs, int thr, uint32_t *__restrict__ kept)
{
  griddep_wait();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t k = 0;
  if (s > 0) {
    const uint32_t sg = seg_of(off, numSegs, s);
    if (s != __ldg(off + sg)) {  // s is a split position inside cloud sg
      const uint2 rg = ranges[s];
      k = (rg.y - rg.x + 1 > (uint32_t)thr) ? 1u : 0u;
    }
  }
  kept[s] = k;
}

__global__ void k_seg_collapse(const Node *__restrict__ full, const uint2 *__restrict__ ranges,
                               const uint32_t *__restrict__ kept, const uint32_t *__restrict__ rank, uint32_t n,
                               const uint32_t *__restrict__ off, uint32_t numSegs, int thr, Node *__restrict__ out)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t sg = seg_of(off, numSegs, t);
  const uint32_t b0 = __ldg(off + sg), e0 = __ldg(off + sg + 1);
  const uint64_t base = 2ull * b0;
  const uint32_t rank0 = rank[b0];  // kept[b0] == 0: exclusive rank at the cloud's start
  const uint32_t nv = e0 - b0;
  if (t == b0) {  // root of the cloud
    const Node root = full[base];
    uint64_t a;
    if (nv > (uint32_t)thr) {
      const uint32_t s0 = (uint32_t)((admin_offset(node_admin(root)) + base) >> 1);
      a = make_admin(2ull + 2ull * (rank[s0] - rank0), 0);
    } else {
      a = make_admin(0, nv);
    }
    out[base] = make_node(root.a.x, root.a.y, root.a.z, root.a.w, root.b.x, root.b.y, a);
    out[base + 1] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0);
    return;
  }
  if (!kept[t]) return;
  const uint32_t s = t;
  const uint2 rg = ranges[s];
  const uint64_t pair = base + 2ull + 2ull * (rank[s] - rank0);
#pragma unroll
  for (int side = 0; side < 2; side++) {
    const Node c = full[2ull * s + side];
    const uint32_t cl = side ? s : rg.x, cr = side ? rg.y : s - 1;
    const uint32_t sz = cr - cl + 1;
    uint64_t a;
    if (sz > (uint32_t)thr) {
      const uint32_t cs = (uint32_t)((admin_offset(node_admin(c)) + base) >> 1);
      a = make_admin(2ull + 2ull * (rank[cs] - rank0), 0);
    } else {
      a = make_admin(cl - b0, sz);
    }
    out[pair + side] = make_node(c.a.x, c.a.y, c.a.z, c.a.w, c.b.x, c.b.y, a);
  }
}

__global__ void k_seg_desc(const uint32_t *__restrict__ off, uint32_t numSegs, uint32_t n, int thr,
                           const uint32_t *__restrict__ rank, bq_node3f *nodes, uint32_t *primIDs,
                           bq_bvh3f *__restrict__ bvhs)
{
  griddep_wait();
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= numSegs) return;
  const uint32_t b0 = off[s], e0 = off[s + 1], nv = e0 - b0;
  bq_bvh3f d;
  d.nodes = nv ? nodes + 2ull * b0 : nullptr;
  d.primIDs = nv ? primIDs + b0 : nullptr;
  d.numPrims = nv;
  if (nv == 0) d.numNodes = 0;
  else if (thr <= 1) d.numNodes = 2 * nv;
  else {
    // kept splits of this cloud: rank over positions [b0, e0)
    const uint32_t endRank = (e0 < n) ? rank[e0] : rank[n - 1] + 0;  // see host: rank has n+1 entries
    d.numNodes = nv > (uint32_t)thr ? 2 + 2 * (endRank - rank[b0]) : 2;
  }
  bvhs[s] = d;
}

// ------------------------------------------------------------------
// batched kNN
// ------------------------------------------------------------------
__global__ void k_seg_query_keys(const bq_bvh3f *__restrict__ bvhs, const float *__restrict__ queries, uint32_t nq,
                                 const uint32_t *__restrict__ qoff, uint32_t numSegs, uint64_t *__restrict__ keys,
                                 uint32_t *__restrict__ idx)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t s = seg_of(qoff, numSegs, t);
  uint32_t code = 0;
  const bq_bvh3f d = bvhs[s];
  if (d.numNodes) {
    const Node root = ldg_node((const Node *)d.nodes);
    const float ext = fmaxf(fmaxf(root.a.w - root.a.x, root.b.x - root.a.y), root.b.y - root.a.z);
    const float sc = 1024.0f / fmaxf(ext, 1e-20f);
    const float *q = queries + 3ull * t;
    const uint32_t cx = min(__float2uint_rz((q[0] - root.a.x) * sc), 1023u);
    const uint32_t cy = min(__float2uint_rz((q[1] - root.a.y) * sc), 1023u);
    const uint32_t cz = min(__float2uint_rz((q[2] - root.a.z) * sc), 1023u);
    code = spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
  }
  keys[t] = ((uint64_t)s << 32) | code;
  idx[t] = t;
}

template <int K, int TIE>
struct BKnnLeaf {
  const uint32_t *__restrict__ primIDs;
  const float *__restrict__ points;
  float qx, qy, qz;
  float maxSqr;
  KnnList<K, TIE> list;
  __device__ __forceinline__ float operator()(uint64_t o, uint32_t cnt)
  {
    for (uint32_t j = 0; j < cnt; j++) {
      const uint32_t pid = __ldg(primIDs + o + j);
      const float *p = points + 3ull * pid;
      const float d = sqr_pp(__ldg(p), __ldg(p + 1), __ldg(p + 2), qx, qy, qz);
      if (TIE == TIE_LOWEST && !(d < maxSqr)) continue;
      list.offer(d, (int32_t)pid);
    }
    return fminf(maxSqr, list.worst());
  }
};

template <int K, int TIE, int STACK>
__global__ void __launch_bounds__(128) k_seg_knn(const bq_bvh3f *__restrict__ bvhs,
                                                 const uint32_t *__restrict__ poff, const float *__restrict__ points,
                                                 const float *__restrict__ queries,
                                                 const uint64_t *__restrict__ sortedKeys,
                                                 const uint32_t *__restrict__ order, uint32_t nq, int k,
                                                 float maxSqr, int chunk, uint32_t *workCtr,
                                                 int32_t *__restrict__ outIds, float *__restrict__ outD,
                                                 int32_t *__restrict__ numFound, uint32_t *__restrict__ ovfList,
                                                 uint32_t *ovfCount)
{
  griddep_wait();
  const int lane = threadIdx.x & 31;
  while (true) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(workCtr, (uint32_t)chunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= nq) return;
    const uint32_t end = min(nq, base + (uint32_t)chunk);
    for (uint32_t t = base + lane; t < end; t += 32) {
      const uint32_t qi = order ? __ldg(order + t) : t;
      const uint32_t s = (uint32_t)(__ldg(sortedKeys + t) >> 32);
      const bq_bvh3f d = bvhs[s];
      int32_t *oi = outIds + (size_t)qi * k;
      float *od = outD + (size_t)qi * k;
      if (d.numNodes == 0) {
        for (int j = 0; j < k; j++) { oi[j] = -1; od[j] = INFINITY; }
        if (numFound) numFound[qi] = 0;
        continue;
      }
      const float *q = queries + 3ull * qi;
      BKnnLeaf<K, TIE> leaf;
      leaf.primIDs = d.primIDs;
      leaf.points = points + 3ull * __ldg(poff + s);
      leaf.qx = __ldg(q); leaf.qy = __ldg(q + 1); leaf.qz = __ldg(q + 2);
      leaf.maxSqr = maxSqr;
      leaf.list.init(k);
      LocalStack<STACK> st;
      if (!traverse<TIE>((const Node *)d.nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) {
        ovfList[atomicAdd(ovfCount, 1u)] = t;
        continue;
      }
      int found = 0;
#pragma unroll
      for (int j = 0; j < K; j++) {
        if (j >= K - k) {
          const bool real = leaf.list.real(j);
          oi[j - (K - k)] = real ? leaf.list.id(j) : -1;
          od[j - (K - k)] = real ? leaf.list.dist(j) : INFINITY;
          found += real ? 1 : 0;
        }
      }
      if (numFound) numFound[qi] = found;
    }
  }
}

template <int K, int TIE>
__global__ void k_seg_knn_deep(const bq_bvh3f *__restrict__ bvhs, const uint32_t *__restrict__ poff,
                               const float *__restrict__ points, const float *__restrict__ queries,
                               const uint64_t *__restrict__ sortedKeys, const uint32_t *__restrict__ order, int k,
                               float maxSqr, int32_t *__restrict__ outIds, float *__restrict__ outD,
                               int32_t *__restrict__ numFound, const uint32_t *ovfList, const uint32_t *ovfCount,
                               StackEntry *stacks, int cap, uint32_t *err)
{
  griddep_wait();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t t = ovfList[w];
    const uint32_t qi = order ? order[t] : t;
    const uint32_t s = (uint32_t)(sortedKeys[t] >> 32);
    const bq_bvh3f d = bvhs[s];
    const float *q = queries + 3ull * qi;
    BKnnLeaf<K, TIE> leaf;
    leaf.primIDs = d.primIDs;
    leaf.points = points + 3ull * poff[s];
    leaf.qx = q[0]; leaf.qy = q[1]; leaf.qz = q[2];
    leaf.maxSqr = maxSqr;
    leaf.list.init(k);
    GlobalStack st{stacks + (size_t)tid * cap, cap, 0};
    int32_t *oi = outIds + (size_t)qi * k;
    float *od = outD + (size_t)qi * k;
    if (!traverse<TIE>((const Node *)d.nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) {
      for (int j = 0; j < k; j++) { oi[j] = -1; od[j] = INFINITY; }
      if (numFound) numFound[qi] = 0;
      atomicOr(err, DEV_ERR_STACK);
      continue;
    }
    int found = 0;
    for (int j = K - k; j < K; j++) {
      const bool real = leaf.list.real(j);
      oi[j - (K - k)] = real ? leaf.list.id(j) : -1;
      od[j - (K - k)] = real ? leaf.list.dist(j) : INFINITY;
      found += real ? 1 : 0;
    }
    if (numFound) numFound[qi] = found;
  }
}

constexpr int DEEP_THREADS = 2048;
constexpr int DEEP_STACK = 1024;

template <int K, int TIE, int STACK>
int launch_seg_knn(const bq_bvh3f *bvhs, const uint32_t *poff, const float *points, const float *queries,
                   const uint64_t *skeys, const uint32_t *order, uint32_t nq, int k, float maxSqr, int block,
                   int chunk, uint32_t *workCtr, int32_t *ids, float *d, int32_t *nf, uint32_t *ovfList,
                   uint32_t *ovfCount, StackEntry *deep, uint32_t *err, cudaStream_t s)
{
  int perSm = 0;
  BQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_seg_knn<K, TIE, STACK>, block, 0));
  const int grid = std::max(1, std::min(num_sms() * std::max(perSm, 1), div_up(nq, block)));
  {
    ProfScope ps("batch.knn", s);
    launch_pdl(k_seg_knn<K, TIE, STACK>, dim3(grid), dim3(block), 0, s, bvhs, poff, points, queries, skeys, order, nq,
               k, maxSqr, chunk, workCtr, ids, d, nf, ovfList, ovfCount);
  }
  ProfScope ps("batch.deep", s);
  launch_pdl(k_seg_knn_deep<K, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, bvhs, poff, points, queries, skeys,
             order, k, maxSqr, ids, d, nf, ovfList, ovfCount, deep, DEEP_STACK, err);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

template <int K, int TIE>
int stack_dispatch(int stack, const bq_bvh3f *bvhs, const uint32_t *poff, const float *points, const float *queries,
                   const uint64_t *skeys, const uint32_t *order, uint32_t nq, int k, float maxSqr, int block,
                   int chunk, uint32_t *workCtr, int32_t *ids, float *d, int32_t *nf, uint32_t *ovfList,
                   uint32_t *ovfCount, StackEntry *deep, uint32_t *err, cudaStream_t s)
{
  if (stack <= 32)
    return launch_seg_knn<K, TIE, 32>(bvhs, poff, points, queries, skeys, order, nq, k, maxSqr, block, chunk, workCtr,
                                      ids, d, nf, ovfList, ovfCount, deep, err, s);
  if (stack <= 64)
    return launch_seg_knn<K, TIE, 64>(bvhs, poff, points, queries, skeys, order, nq, k, maxSqr, block, chunk, workCtr,
                                      ids, d, nf, ovfList, ovfCount, deep, err, s);
  return launch_seg_knn<K, TIE, 128>(bvhs, poff, points, queries, skeys, order, nq, k, maxSqr, block, chunk, workCtr,
                                     ids, d, nf, ovfList, ovfCount, deep, err, s);
}

} // namespace

int batched_build_morton63(const bq_box3f *boxes, const uint32_t *off, uint32_t numSegs, uint32_t n,
                           const bq_build_config *cfg, bq_node3f *nodesOut, uint32_t *primIDs, bq_bvh3f *bvhs,
                           uint32_t *errOut, Alloc &al)
{
  const int maxLeaf = cfg ? cfg->maxAllowedLeafSize : (1 << 15);
  const int mlt = cfg ? cfg->makeLeafThreshold : 0;
  const int thr = mlt > 0 ? std::min(mlt, maxLeaf) : 1;
  if (thr < 1 || thr > 65535) return set_error(BQ_ERR_INVALID_ARGUMENT, "leaf threshold must be in [1, 65535]");
  if (numSegs == 0) return BQ_OK;
  TempSet tmp(al);
  int32_t *segLoHi = nullptr;
  SegQuant *quant = nullptr;
  uint32_t *hist = nullptr, *ids[2], *segKey[2], *pos[2], *slot = nullptr, *err = nullptr;
  uint64_t *keys[2], *fkeys = nullptr;
  uint32_t *fids = nullptr;
  uint8_t *delta = nullptr;
  uint32_t *rank = nullptr, *kept = nullptr;
  uint2 *ranges = nullptr;
  Node *full = nullptr;
  BQ_TRY(tmp.get(&segLoHi, 6ull * numSegs));
  BQ_TRY(tmp.get(&quant, numSegs));
  BQ_TRY(tmp.get(&hist, 8 * 256));
  BQ_TRY(tmp.get(&err, 1));
  if (n == 0) {
    launch_pdl(k_seg_desc, dim3(div_up(numSegs, 128)), dim3(128), 0, al.s, off, numSegs, n, thr, nullptr, nodesOut,
               primIDs, bvhs);
    BQ_CUDA(cudaGetLastError());
    return BQ_OK;
  }
  BQ_TRY(tmp.get(&keys[0], n));
  BQ_TRY(tmp.get(&keys[1], n));
  BQ_TRY(tmp.get(&ids[0], n));
  BQ_TRY(tmp.get(&ids[1], n));
  BQ_TRY(tmp.get(&segKey[0], n));
  BQ_TRY(tmp.get(&segKey[1], n));
  BQ_TRY(tmp.get(&pos[0], n));
  BQ_TRY(tmp.get(&pos[1], n));
  BQ_TRY(tmp.get(&fkeys, n));
  BQ_TRY(tmp.get(&fids, n));
  BQ_TRY(tmp.get(&delta, n));
  BQ_TRY(tmp.get(&slot, n));
  uint32_t *dErr = errOut ? errOut : err;
  if (!errOut) BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  BQ_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 8 * 256, al.s));
  {
    ProfScope ps("batch.bounds", al.s, 3);
    launch_pdl(k_seg_bounds_init, dim3(div_up(numSegs, 128)), dim3(128), 0, al.s, segLoHi, numSegs);
    launch_pdl(k_seg_bounds, dim3(div_up(n, 256)), dim3(256), 0, al.s, boxes, n, off, numSegs, segLoHi);
    launch_pdl(k_seg_quant, dim3(div_up(numSegs, 128)), dim3(128), 0, al.s, segLoHi, numSegs, quant);
  }
  {
    ProfScope ps("batch.keygen", al.s);
    launch_pdl(k_seg_keygen, dim3(div_up(n, 256)), dim3(256), 0, al.s, boxes, n, off, numSegs, quant, keys[0], ids[0],
               hist);
  }
  BQ_CUDA(cudaGetLastError());
  int sel = 0;
  BQ_TRY(onesweep_sort_u64(keys, ids, n, nullptr, 0, 63, hist, &sel, dErr, al));
  uint64_t *mk = keys[sel];
  uint32_t *mi = ids[sel];
  int segBits = 1;
  while (segBits < 32 && (1ull << segBits) < numSegs) segBits++;
  {
    ProfScope ps("batch.segkeys", al.s);
    launch_pdl(k_seg_ids, dim3(div_up(n, 256)), dim3(256), 0, al.s, mi, n, off, numSegs, segKey[0], pos[0]);
  }
  int sel2 = 0;
  BQ_TRY(onesweep_sort_u32(segKey, pos, n, nullptr, 0, segBits, nullptr, &sel2, dErr, al));
  {
    ProfScope ps("batch.gather", al.s);
    launch_pdl(k_seg_gather, dim3(div_up(n, 256)), dim3(256), 0, al.s, pos[sel2], mk, mi, n, fkeys, fids);
  }
  {
    ProfScope ps("batch.delta", al.s);
    launch_pdl(k_seg_delta, dim3(div_up(n, 256)), dim3(256), 0, al.s, fkeys, n, off, numSegs, delta);
  }
  uint2 *pending = nullptr;
  BQ_TRY(tmp.get(&pending, 2ull * div_up(n, AGG_CHUNK)));
  // the prim count on the device is the last cloud offset (no host copy,
  // so the sequence stays capturable)
  AggArgs ag{delta, slot, fids, boxes, (Node *)nodesOut, primIDs, off + numSegs, nullptr, pending, off, numSegs};
  if (thr == 1) {
    BQ_TRY(agglomerate<true>(ag, n, al.s, "batch.agg_local", "batch.agg_global"));
  } else {
    BQ_TRY(tmp.get(&full, 2ull * n));
    BQ_TRY(tmp.get(&ranges, n));
    BQ_TRY(tmp.get(&kept, n + 1ull));
    BQ_TRY(tmp.get(&rank, n + 1ull));
    ag.nodes = full;
    ag.ranges = ranges;
    BQ_TRY(agglomerate<true>(ag, n, al.s, "batch.agg_local", "batch.agg_global"));
    ProfScope ps("batch.collapse", al.s, 6);  // kept, memset, scan (3), collapse
    launch_pdl(k_seg_kept, dim3(div_up(n, 256)), dim3(256), 0, al.s, ranges, n, off, numSegs, thr, kept);
    BQ_CUDA(cudaMemsetAsync(kept + n, 0, 4, al.s));
    BQ_TRY(exclusive_scan_u32(kept, rank, n + 1, nullptr, nullptr, al));
    launch_pdl(k_seg_collapse, dim3(div_up(n, 256)), dim3(256), 0, al.s, full, ranges, kept, rank, n, off, numSegs,
               thr, (Node *)nodesOut);
  }
  launch_pdl(k_seg_desc, dim3(div_up(numSegs, 128)), dim3(128), 0, al.s, off, numSegs, n, thr, rank, nodesOut,
             primIDs, bvhs);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

int batched_knn(const bq_bvh3f *bvhs, const uint32_t *poff, const float *points, const float *queries,
                const uint32_t *qoff, uint32_t numSegs, uint32_t nq, int k, float maxSqr, const bq_query_config *qcfg,
                int32_t *ids, float *d, int32_t *nf, uint32_t *errOut, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  const int chunk = c.queriesPerWarp;
  if (k < 1 || k > 64) return set_error(BQ_ERR_INVALID_ARGUMENT, "k must be in [1, 64]");
  if (nq == 0 || numSegs == 0) return BQ_OK;
  TempSet tmp(al);
  uint64_t *keys[2];
  uint32_t *idx[2], *ovfList = nullptr, *ctl = nullptr;
  StackEntry *deep = nullptr;
  BQ_TRY(tmp.get(&keys[0], nq));
  BQ_TRY(tmp.get(&keys[1], nq));
  BQ_TRY(tmp.get(&idx[0], nq));
  BQ_TRY(tmp.get(&idx[1], nq));
  BQ_TRY(tmp.get(&ovfList, nq));
  BQ_TRY(tmp.get(&ctl, 4));  // [0] work counter [1] overflow count [2] error
  BQ_TRY(tmp.get(&deep, (size_t)DEEP_THREADS * DEEP_STACK));
  BQ_CUDA(cudaMemsetAsync(ctl, 0, 16, al.s));
  uint32_t *dErr = errOut ? errOut : ctl + 2;
  {
    ProfScope ps("batch.query_keys", al.s);
    launch_pdl(k_seg_query_keys, dim3(div_up(nq, 256)), dim3(256), 0, al.s, bvhs, queries, nq, qoff, numSegs, keys[0],
               idx[0]);
  }
  int segBits = 1;
  while (segBits < 32 && (1ull << segBits) < numSegs) segBits++;
  int sel = 0;
  const uint32_t *order = nullptr;
  const uint64_t *skeys = keys[0];
  if (c.reorder) {
    BQ_TRY(onesweep_sort_u64(keys, idx, nq, nullptr, 6, 32 + segBits, nullptr, &sel, dErr, al));  // order only
    order = idx[sel];
    skeys = keys[sel];
  }
  const int tie = c.tieMode, st = c.stackDepth, b = c.blockSize;
#define BQ_SEG_KNN(KK)                                                                                             \
  (tie == BQ_TIES_REFERENCE                                                                                        \
       ? stack_dispatch<KK, TIE_REFERENCE>(st, bvhs, poff, points, queries, skeys, order, nq, k, maxSqr, b, chunk, \
                                           ctl, ids, d, nf, ovfList, ctl + 1, deep, dErr, al.s)                    \
       : stack_dispatch<KK, TIE_LOWEST>(st, bvhs, poff, points, queries, skeys, order, nq, k, maxSqr, b, chunk,    \
                                        ctl, ids, d, nf, ovfList, ctl + 1, deep, dErr, al.s))
  int s;
  if (k <= 4) s = BQ_SEG_KNN(4);
  else if (k <= 8) s = BQ_SEG_KNN(8);
  else if (k <= 16) s = BQ_SEG_KNN(16);
  else if (k <= 32) s = BQ_SEG_KNN(32);
  else s = BQ_SEG_KNN(64);
#undef BQ_SEG_KNN
  return s;
}

// ------------------------------------------------------------------
// autotuner: time every knob combination on the caller's inputs
// ------------------------------------------------------------------
int autotune_batched_knn(const bq_box3f *boxes, const float *points, const uint32_t *off, uint32_t numSegs,
                         uint32_t n, const float *queries, const uint32_t *qoff, uint32_t nq, int k, bq_tuning *best,
                         Alloc &al)
{
  if (!best) return set_error(BQ_ERR_INVALID_ARGUMENT, "best is NULL");
  TempSet tmp(al);
  bq_node3f *nodes = nullptr;
  uint32_t *prims = nullptr;
  bq_bvh3f *bvhs = nullptr;
  int32_t *ids = nullptr;
  float *d = nullptr;
  BQ_TRY(tmp.get(&nodes, 2ull * n + 2));
  BQ_TRY(tmp.get(&prims, n + 1ull));
  BQ_TRY(tmp.get(&bvhs, numSegs));
  BQ_TRY(tmp.get(&ids, (size_t)nq * k));
  BQ_TRY(tmp.get(&d, (size_t)nq * k));
  cudaEvent_t e[3];
  for (auto &x : e) BQ_CUDA(cudaEventCreate(&x));
  const int leaves[] = {1, 2, 4, 8}, stacks[] = {32, 64}, blocks[] = {64, 128}, grabs[] = {32, 128};
  float bestMs = INFINITY;
  int status = BQ_OK;
  for (int lf : leaves) {
    bq_build_config bc{1 << 15, lf, BQ_SPATIAL_MEDIAN};
    for (int st : stacks)
      for (int bl : blocks)
        for (int gr : grabs) {
          bq_query_config qc{BQ_TIES_LOWEST_ID, st, bl, 1, gr};
          float tb = 0.f, tq = 0.f;
          for (int rep = 0; rep < 2 && status == BQ_OK; rep++) {  // rep 0 warms up
            cudaEventRecord(e[0], al.s);
            status = batched_build_morton63(boxes, off, numSegs, n, &bc, nodes, prims, bvhs, nullptr, al);
            cudaEventRecord(e[1], al.s);
            if (status == BQ_OK)
              status = batched_knn(bvhs, off, points, queries, qoff, numSegs, nq, k, INFINITY, &qc, ids, d, nullptr,
                                   nullptr, al);
            cudaEventRecord(e[2], al.s);
            cudaEventSynchronize(e[2]);
            cudaEventElapsedTime(&tb, e[0], e[1]);
            cudaEventElapsedTime(&tq, e[1], e[2]);
          }
          if (status != BQ_OK) break;
          if (tb + tq < bestMs) {
            bestMs = tb + tq;
            *best = bq_tuning{lf, st, bl, gr, tb, tq};
          }
        }
  }
  for (auto &x : e) cudaEventDestroy(x);
  return status;
}

} // namespace bq
