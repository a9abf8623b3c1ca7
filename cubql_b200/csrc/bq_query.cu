// bq_query.cu -- batched closest-point and kNN queries over point BVHs.
//
// The reference exposes these as per-thread device functions
// (cuBQL/queries/points/findClosest.h:181-226 findClosest_withBlackList,
// cuBQL/queries/points/knn.h:75-116 findKNN) that user kernels call one
// thread per query in input order.  Here one call answers a whole batch:
//
//   k_query_keys   30-bit Morton code of every query inside the root box
//   onesweep sort  queries reordered along the curve (top 24 key bits),
//                  so neighbouring threads walk nearly the same nodes
//                  (L1/L2 reuse, less divergence)
//   k_closest / k_knn
//                  one thread per query, shrinking-radius traversal with a
//                  local-memory stack (bq_traverse.cuh); kNN keeps its
//                  sorted top-k in registers
//   *_deep         queries whose stack overflowed are re-run with a deep
//                  stack in global memory instead of returning a wrong
//                  answer (the reference returns early, :475-478)
#include <algorithm>

#include "bq_query.cuh"

namespace bq {
namespace {

// stack entries a closest-point thread keeps in shared memory (the top of
// its traversal stack); the rest of the stack is in local memory.  8 took
// 10M closest-point queries from 4.17 to 3.69 ms (4: 3.92, 12: 3.83, 16:
// 3.99).  The kNN kernel, at 62 registers and fewer threads per SM, gained
// nothing from it (29.7 ms with none, 29.8-30.3 with 4..16), so its stack
// stays in local memory.
constexpr int SMEM_STACK = 8;
constexpr int KNN_SMEM_STACK = 0;

// rootBox: lower xyz, upper xyz (the first 24 bytes of a binary root node)
__global__ void k_query_keys(const float *__restrict__ rootBox, const float *__restrict__ queries, uint32_t nq,
                             uint32_t *__restrict__ keys, uint32_t *__restrict__ idx)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const float lx = __ldg(rootBox), ly = __ldg(rootBox + 1), lz = __ldg(rootBox + 2);
  const float ext = fmaxf(fmaxf(__ldg(rootBox + 3) - lx, __ldg(rootBox + 4) - ly), __ldg(rootBox + 5) - lz);
  const float sc = 1024.0f / fmaxf(ext, 1e-20f);
  const float *q = queries + 3ull * t;
  const uint32_t cx = min(__float2uint_rz((q[0] - lx) * sc), 1023u);
  const uint32_t cy = min(__float2uint_rz((q[1] - ly) * sc), 1023u);
  const uint32_t cz = min(__float2uint_rz((q[2] - lz) * sc), 1023u);
  keys[t] = spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
  idx[t] = t;
}

template <int TIE, typename Stack>
__device__ __forceinline__ bool run_cp(const Node *nodes, const uint32_t *primIDs, const float *points,
                                       const float *queries, uint32_t qi, float maxSqr, Stack &st, int32_t *outIds,
                                       float *outD, CpExclude ex)
{
  const float *q = queries + 3ull * qi;
  CPLeaf<TIE> leaf{primIDs, points, __ldg(q), __ldg(q + 1), __ldg(q + 2), maxSqr, -1,
                   ex.ids ? __ldg(ex.ids + qi) : -1, ex.self};
  if (!traverse<TIE>(nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) return false;
  outIds[qi] = leaf.id;
  outD[qi] = leaf.id >= 0 ? leaf.best : INFINITY;
  return true;
}

template <int TIE, int STACK>
__global__ void __launch_bounds__(128) k_closest(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                 const float *__restrict__ points, const float *__restrict__ queries,
                                                 const uint32_t *__restrict__ order, uint32_t nq, float maxSqr,
                                                 int32_t *__restrict__ outIds, float *__restrict__ outD,
                                                 uint32_t *__restrict__ ovfList, uint32_t *ovfCount, CpExclude ex)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t qi = order ? __ldg(order + t) : t;
  extern __shared__ StackEntry sStack[];
  HybridStack<SMEM_STACK, STACK> st(sStack);
  if (!run_cp<TIE>(nodes, primIDs, points, queries, qi, maxSqr, st, outIds, outD, ex))
    ovfList[atomicAdd(ovfCount, 1u)] = qi;
}

template <int TIE>
__global__ void k_closest_deep(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                               const float *__restrict__ points, const float *__restrict__ queries, float maxSqr,
                               int32_t *__restrict__ outIds, float *__restrict__ outD, const uint32_t *ovfList,
                               const uint32_t *ovfCount, StackEntry *stacks, uint32_t *err, CpExclude ex)
{
  griddep_wait();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t qi = ovfList[w];
    GlobalStack st{stacks + (size_t)tid * DEEP_STACK, DEEP_STACK, 0};
    if (!run_cp<TIE>(nodes, primIDs, points, queries, qi, maxSqr, st, outIds, outD, ex)) {
      outIds[qi] = -1;
      outD[qi] = INFINITY;
      atomicOr(err, DEV_ERR_STACK);
    }
  }
}

// ------------------------------------------------------------------
// kNN
// ------------------------------------------------------------------
template <int K, int TIE>
struct KnnLeaf {
  const uint32_t *__restrict__ primIDs;
  const float *__restrict__ points;
  float qx, qy, qz;
  float maxSqr;
  KnnList<K, TIE> list;
  __device__ __forceinline__ float operator()(uint64_t off, uint32_t cnt)
  {
    for (uint32_t j = 0; j < cnt; j++) {
      const uint32_t pid = __ldg(primIDs + off + j);
      const float *p = points + 3ull * pid;
      const float d = sqr_pp(__ldg(p), __ldg(p + 1), __ldg(p + 2), qx, qy, qz);
      if (TIE == TIE_LOWEST && !(d < maxSqr)) continue;
      list.offer(d, (int32_t)pid);
    }
    // knn::Result.sqrDistMax: the radius until k are found, then the k-th
    return fminf(maxSqr, list.worst());
  }
};

template <int K, int TIE, typename Stack>
__device__ __forceinline__ bool run_knn(const Node *nodes, const uint32_t *primIDs, const float *points,
                                        const float *queries, uint32_t qi, int k, float maxSqr, Stack &st,
                                        int32_t *outIds, float *outD, int32_t *numFound)
{
  const float *q = queries + 3ull * qi;
  KnnLeaf<K, TIE> leaf;
  leaf.primIDs = primIDs;
  leaf.points = points;
  leaf.qx = __ldg(q);
  leaf.qy = __ldg(q + 1);
  leaf.qz = __ldg(q + 2);
  leaf.maxSqr = maxSqr;
  leaf.list.init(k);
  if (!traverse<TIE>(nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) return false;
  int found = 0;
  int32_t *oi = outIds + (size_t)qi * k;
  float *od = outD + (size_t)qi * k;
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
  return true;
}

template <int K, int TIE, int STACK>
__global__ void __launch_bounds__(128) k_knn(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                             const float *__restrict__ points, const float *__restrict__ queries,
                                             const uint32_t *__restrict__ order, uint32_t nq, int k, float maxSqr,
                                             int32_t *__restrict__ outIds, float *__restrict__ outD,
                                             int32_t *__restrict__ numFound, uint32_t *__restrict__ ovfList,
                                             uint32_t *ovfCount)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t qi = order ? __ldg(order + t) : t;
  extern __shared__ StackEntry sStack[];
  HybridStack<KNN_SMEM_STACK, STACK> st(sStack);
  if (!run_knn<K, TIE>(nodes, primIDs, points, queries, qi, k, maxSqr, st, outIds, outD, numFound))
    ovfList[atomicAdd(ovfCount, 1u)] = qi;
}

template <int K, int TIE>
__global__ void k_knn_deep(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                           const float *__restrict__ points, const float *__restrict__ queries, int k, float maxSqr,
                           int32_t *__restrict__ outIds, float *__restrict__ outD, int32_t *__restrict__ numFound,
                           const uint32_t *ovfList, const uint32_t *ovfCount, StackEntry *stacks, uint32_t *err)
{
  griddep_wait();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t qi = ovfList[w];
    GlobalStack st{stacks + (size_t)tid * DEEP_STACK, DEEP_STACK, 0};
    if (!run_knn<K, TIE>(nodes, primIDs, points, queries, qi, k, maxSqr, st, outIds, outD, numFound)) {
      for (int j = 0; j < k; j++) {
        outIds[(size_t)qi * k + j] = -1;
        outD[(size_t)qi * k + j] = INFINITY;
      }
      if (numFound) numFound[qi] = 0;
      atomicOr(err, DEV_ERR_STACK);
    }
  }
}

// ------------------------------------------------------------------
// kNN with G lanes per query: the group walks the tree together (every
// lane runs the same traversal on the same query, so the group never
// diverges and node loads are broadcast) and holds the sorted top-k list
// one candidate per lane (lane j: the j-th best).  A leaf's prims are
// tested G at a time, one per lane; each candidate that beats the k-th best
// is placed with one ballot (how many entries it follows) and moved in with
// one __shfl_up_sync.  k <= G.
// ------------------------------------------------------------------
template <int G, int TIE>
struct GroupKnnLeaf {
  const uint32_t *__restrict__ primIDs;
  const float *__restrict__ points;
  float qx, qy, qz;
  float maxSqr;
  int k;
  uint32_t lane;   // lane in the group
  uint32_t gmask;  // the group's lanes in the warp
  float D;         // this lane's list entry
  int32_t I;
  __device__ __forceinline__ bool before(float d, int32_t id, float D2, int32_t I2) const
  {
    return cand_before<TIE>(d, id, D2, I2);
  }
  __device__ __forceinline__ float worst() const { return __shfl_sync(gmask, D, k - 1, G); }
  // place candidate (d, id), already known to beat the k-th best
  __device__ __forceinline__ void insert(float d, int32_t id)
  {
    // entries the candidate stays behind: all lanes below its position
    const uint32_t behind = __ballot_sync(gmask, lane < (uint32_t)k && !before(d, id, D, I)) & gmask;
    const uint32_t pos = __popc(behind);
    const float upD = __shfl_up_sync(gmask, D, 1, G);
    const int32_t upI = __shfl_up_sync(gmask, I, 1, G);
    if (lane == pos) {
      D = d;
      I = id;
    } else if (lane > pos) {
      D = upD;
      I = upI;
    }
  }
  __device__ __forceinline__ float operator()(uint64_t off, uint32_t cnt)
  {
    // every shuffle below runs on all lanes of the group (never inside a
    // condition that only some lanes take)
    float w = worst();
    int32_t wi = __shfl_sync(gmask, I, k - 1, G);
    for (uint32_t base = 0; base < cnt; base += G) {
      float d = INFINITY;
      int32_t pid = 0x7fffffff;
      const bool mine = base + lane < cnt;
      if (mine) {
        pid = (int32_t)__ldg(primIDs + off + base + lane);
        const float *p = points + 3ull * pid;
        d = sqr_pp(__ldg(p), __ldg(p + 1), __ldg(p + 2), qx, qy, qz);
      }
      const bool ok = mine && (TIE == TIE_REFERENCE || d < maxSqr);
      // candidates of this round that beat the k-th best, handled in prim order
      uint32_t m = __ballot_sync(gmask, ok && before(d, pid, w, wi)) & gmask;
      while (m) {
        const int src = __ffs(m) - 1;
        const float cd = __shfl_sync(gmask, d, src & (G - 1), G);
        const int32_t ci = __shfl_sync(gmask, pid, src & (G - 1), G);
        insert(cd, ci);
        w = worst();
        wi = __shfl_sync(gmask, I, k - 1, G);
        m &= ~(1u << src);
        m &= __ballot_sync(gmask, ok && before(d, pid, w, wi)) & gmask;
      }
    }
    return fminf(maxSqr, w);
  }
};

template <int G, int TIE, int STACK>
__global__ void __launch_bounds__(128) k_knn_group(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                   const float *__restrict__ points, const float *__restrict__ queries,
                                                   const uint32_t *__restrict__ order, uint32_t nq, int k,
                                                   float maxSqr, int32_t *__restrict__ outIds,
                                                   float *__restrict__ outD, int32_t *__restrict__ numFound,
                                                   uint32_t *__restrict__ ovfList, uint32_t *ovfCount)
{
  griddep_wait();
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t t = gt / G;  // the group's query slot (whole groups leave together)
  if (t >= nq) return;
  const uint32_t lane = threadIdx.x & (G - 1);
  const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1) << ((threadIdx.x & 31) & ~(G - 1)));
  const uint32_t qi = order ? __ldg(order + t) : t;
  const float *q = queries + 3ull * qi;
  GroupKnnLeaf<G, TIE> leaf;
  leaf.primIDs = primIDs;
  leaf.points = points;
  leaf.qx = __ldg(q);
  leaf.qy = __ldg(q + 1);
  leaf.qz = __ldg(q + 2);
  leaf.maxSqr = maxSqr;
  leaf.k = k;
  leaf.lane = lane;
  leaf.gmask = gmask;
  // lanes past k hold a sentinel that every candidate stays behind
  leaf.D = lane < (uint32_t)k ? INFINITY : -1.0f;
  leaf.I = lane < (uint32_t)k ? 0x7fffffff : -1;
  LocalStack<STACK> st;
  if (!traverse<TIE>(nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) {
    if (lane == 0) ovfList[atomicAdd(ovfCount, 1u)] = qi;
    return;
  }
  const bool real = leaf.I != 0x7fffffff && leaf.D != INFINITY;
  if (lane < (uint32_t)k) {
    outIds[(size_t)qi * k + lane] = real ? leaf.I : -1;
    outD[(size_t)qi * k + lane] = real ? leaf.D : INFINITY;
  }
  const uint32_t found = __popc(__ballot_sync(gmask, lane < (uint32_t)k && real) & gmask);
  if (numFound && lane == 0) numFound[qi] = (int32_t)found;
}

template <int G, int TIE, int STACK>
void launch_knn_group(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k,
                      float maxSqr, int block, int32_t *ids, float *d, int32_t *nf, QueryScratch &qs, cudaStream_t s)
{
  const Node *nodes = (const Node *)bvh->nodes;
  {
    ProfScope ps("query.knn_group", s);
    launch_pdl(k_knn_group<G, TIE, STACK>, dim3(div_up((uint64_t)nq * G, block)), dim3(block), 0, s, nodes,
               bvh->primIDs, points, queries, qs.order, nq, k, maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount);
  }
  // overflowing queries: the per-thread deep-stack kernel (same answers)
  ProfScope ps("query.deep", s);
  if (k <= 4)
    launch_pdl(k_knn_deep<4, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries, k,
               maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount, qs.deep, qs.err);
  else if (k <= 8)
    launch_pdl(k_knn_deep<8, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries, k,
               maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount, qs.deep, qs.err);
  else if (k <= 16)
    launch_pdl(k_knn_deep<16, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries,
               k, maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount, qs.deep, qs.err);
  else
    launch_pdl(k_knn_deep<32, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries,
               k, maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount, qs.deep, qs.err);
}

template <int TIE>
void dispatch_knn_group(int G, int stack, const bq_bvh3f *bvh, const float *points, const float *queries,
                        uint32_t nq, int k, float maxSqr, int block, int32_t *ids, float *d, int32_t *nf,
                        QueryScratch &qs, cudaStream_t s)
{
#define BQ_KG(GG)                                                                                              \
  do {                                                                                                         \
    if (stack <= 32) launch_knn_group<GG, TIE, 32>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);  \
    else if (stack <= 64) launch_knn_group<GG, TIE, 64>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s); \
    else launch_knn_group<GG, TIE, 128>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);          \
  } while (0)
  if (G == 4) BQ_KG(4);
  else if (G == 8) BQ_KG(8);
  else if (G == 16) BQ_KG(16);
  else BQ_KG(32);
#undef BQ_KG
}

template <int TIE, int STACK>
void launch_cp(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, float maxSqr,
               int block, int32_t *ids, float *d, QueryScratch &qs, cudaStream_t s, CpExclude ex)
{
  const Node *nodes = (const Node *)bvh->nodes;
  {
    ProfScope ps("query.closest", s);
    launch_pdl(k_closest<TIE, STACK>, dim3(div_up(nq, block)), dim3(block), SMEM_STACK * sizeof(StackEntry) * block,
               s, nodes, bvh->primIDs, points, queries, qs.order, nq, maxSqr, ids, d, qs.ovfList, qs.ovfCount, ex);
  }
  ProfScope ps("query.deep", s);
  launch_pdl(k_closest_deep<TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries,
             maxSqr, ids, d, qs.ovfList, qs.ovfCount, qs.deep, qs.err, ex);
}

template <int K, int TIE, int STACK>
void launch_knn(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k, float maxSqr,
                int block, int32_t *ids, float *d, int32_t *nf, QueryScratch &qs, cudaStream_t s)
{
  const Node *nodes = (const Node *)bvh->nodes;
  {
    ProfScope ps("query.knn", s);
    launch_pdl(k_knn<K, TIE, STACK>, dim3(div_up(nq, block)), dim3(block),
               KNN_SMEM_STACK * sizeof(StackEntry) * block, s, nodes, bvh->primIDs, points, queries, qs.order, nq, k,
               maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount);
  }
  ProfScope ps("query.deep", s);
  launch_pdl(k_knn_deep<K, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, nodes, bvh->primIDs, points, queries, k,
             maxSqr, ids, d, nf, qs.ovfList, qs.ovfCount, qs.deep, qs.err);
}

template <int K, int TIE>
void dispatch_knn_stack(int stack, const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq,
                        int k, float maxSqr, int block, int32_t *ids, float *d, int32_t *nf, QueryScratch &qs,
                        cudaStream_t s)
{
  if (stack <= 32) launch_knn<K, TIE, 32>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);
  else if (stack <= 64) launch_knn<K, TIE, 64>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);
  else launch_knn<K, TIE, 128>(bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);
}

template <int K>
void dispatch_knn_tie(int tie, int stack, const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq,
                      int k, float maxSqr, int block, int32_t *ids, float *d, int32_t *nf, QueryScratch &qs,
                      cudaStream_t s)
{
  if (tie == BQ_TIES_REFERENCE)
    dispatch_knn_stack<K, TIE_REFERENCE>(stack, bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);
  else
    dispatch_knn_stack<K, TIE_LOWEST>(stack, bvh, points, queries, nq, k, maxSqr, block, ids, d, nf, qs, s);
}

// ------------------------------------------------------------------
// visit counts (the measurement pass of the query rooflines): the same
// traversal per query, in input order, counting node pairs loaded, admin
// loads and prims tested.  A query whose 128-entry stack overflows
// contributes what it visited until then.
// ------------------------------------------------------------------
template <int TIE, int K>
__global__ void __launch_bounds__(128) k_visit_count(const Node *__restrict__ nodes,
                                                     const uint32_t *__restrict__ primIDs,
                                                     const float *__restrict__ points,
                                                     const float *__restrict__ queries, uint32_t nq, int k,
                                                     float maxSqr, unsigned long long *out)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  VisitCount vc;
  uint32_t prims = 0;
  if (t < nq) {  // no early return: every lane takes part in the warp sum below
    const float *q = queries + 3ull * t;
    LocalStack<128> st;
    if constexpr (K == 0) {
      CPLeaf<TIE> leaf{primIDs, points, __ldg(q), __ldg(q + 1), __ldg(q + 2), maxSqr, -1, -1, 0};
      CountingLeaf<CPLeaf<TIE>> cl{leaf};
      traverse_counted<TIE>(nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, cl, vc);
      prims = cl.prims;
    } else {
      KnnLeaf<K, TIE> leaf;
      leaf.primIDs = primIDs;
      leaf.points = points;
      leaf.qx = __ldg(q);
      leaf.qy = __ldg(q + 1);
      leaf.qz = __ldg(q + 2);
      leaf.maxSqr = maxSqr;
      leaf.list.init(k);
      CountingLeaf<KnnLeaf<K, TIE>> cl{leaf};
      traverse_counted<TIE>(nodes, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, cl, vc);
      prims = cl.prims;
    }
  }
  add_visit_counts(vc.pairs, vc.admins, prims, out);
}

template <int TIE>
void launch_visit_count(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k,
                        float maxSqr, unsigned long long *out, cudaStream_t s)
{
  const Node *nodes = (const Node *)bvh->nodes;
  const int g = div_up(nq, 128);
#define BQ_VC(KK) k_visit_count<TIE, KK><<<g, 128, 0, s>>>(nodes, bvh->primIDs, points, queries, nq, k, maxSqr, out)
  if (k == 0) BQ_VC(0);
  else if (k <= 4) BQ_VC(4);
  else if (k <= 8) BQ_VC(8);
  else if (k <= 16) BQ_VC(16);
  else if (k <= 32) BQ_VC(32);
  else BQ_VC(64);
#undef BQ_VC
}

} // namespace

__global__ void k_fill_empty(uint32_t nq, int k, int32_t *ids, float *d, int32_t *numFound)
{
  griddep_wait();
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (uint64_t)nq * k) return;
  ids[t] = -1;
  d[t] = INFINITY;
  if (numFound && t < nq) numFound[t] = 0;
}

int prepare_queries(const float *rootBox, const float *queries, uint32_t nq, bool reorder, TempSet &tmp, Alloc &al,
                    QueryScratch &qs)
{
  BQ_TRY(tmp.get(&qs.ovfList, nq));
  BQ_TRY(tmp.get(&qs.ovfCount, 2));
  qs.err = qs.ovfCount + 1;
  BQ_TRY(tmp.get(&qs.deep, (size_t)DEEP_THREADS * DEEP_STACK));
  BQ_CUDA(cudaMemsetAsync(qs.ovfCount, 0, 8, al.s));
  if (reorder && nq > 1) {
    uint32_t *keys[2], *idx[2];
    BQ_TRY(tmp.get(&keys[0], nq));
    BQ_TRY(tmp.get(&keys[1], nq));
    BQ_TRY(tmp.get(&idx[0], nq));
    BQ_TRY(tmp.get(&idx[1], nq));
    {
      ProfScope ps("query.keys", al.s);
      launch_pdl(k_query_keys, dim3(div_up(nq, 256)), dim3(256), 0, al.s, rootBox, queries, nq, keys[0], idx[0]);
    }
    BQ_CUDA(cudaGetLastError());
    int sel = 0;
    // the order only steers performance: the top 24 key bits (3 passes)
    // suffice; up to 2M queries the top 16 (2 passes) do as well
    const int loBit = nq <= (1u << 21) ? 14 : 6;
    BQ_TRY(onesweep_sort_u32(keys, idx, nq, nullptr, loBit, 30, nullptr, &sel, qs.err, al));
    qs.order = idx[sel];
  }
  return BQ_OK;
}

int finish_queries(QueryScratch &qs, Alloc &al)
{
  // the only host synchronisation: read the device error word
  uint32_t err = 0;
  BQ_CUDA(cudaMemcpyAsync(&err, qs.err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (err & DEV_ERR_STACK) return set_error(BQ_ERR_STACK_OVERFLOW, "query exceeded the deep fallback stack");
  if (err & DEV_ERR_TIMEOUT) return set_error(BQ_ERR_TIMEOUT, "query reordering sort timed out");
  return BQ_OK;
}

int query_config(const bq_query_config *q, bq_query_config &out)
{
  out.tieMode = q ? q->tieMode : BQ_TIES_LOWEST_ID;
  out.stackDepth = (q && q->stackDepth) ? q->stackDepth : 64;
  out.blockSize = (q && q->blockSize) ? q->blockSize : 128;
  out.reorder = q ? q->reorder : 1;
  out.queriesPerWarp = (q && q->queriesPerWarp) ? q->queriesPerWarp : 32;
  out.lanesPerQuery = (q && q->lanesPerQuery) ? q->lanesPerQuery : 1;
  if (out.lanesPerQuery != 1 && out.lanesPerQuery != 4 && out.lanesPerQuery != 8 && out.lanesPerQuery != 16 &&
      out.lanesPerQuery != 32)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "lanesPerQuery must be 1, 4, 8, 16 or 32");
  if (out.tieMode != BQ_TIES_LOWEST_ID && out.tieMode != BQ_TIES_REFERENCE)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "tieMode must be BQ_TIES_LOWEST_ID or BQ_TIES_REFERENCE");
  if (out.stackDepth != 32 && out.stackDepth != 64 && out.stackDepth != 128)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "stackDepth must be 32, 64 or 128");
  if (out.blockSize != 64 && out.blockSize != 128)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "blockSize must be 64 or 128");
  if (out.queriesPerWarp < 32 || out.queriesPerWarp > 1024 || out.queriesPerWarp % 32)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "queriesPerWarp must be a multiple of 32 up to 1024");
  return BQ_OK;
}

int closest_point(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, float maxSqr,
                  const bq_query_config *qcfg, int32_t *ids, float *d, Alloc &al, const int32_t *excludeIds,
                  int excludeSelf)
{
  const CpExclude ex{excludeIds, excludeSelf};
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    launch_pdl(k_fill_empty, dim3(div_up(nq, 256)), dim3(256), 0, al.s, nq, 1, ids, d, nullptr);
    BQ_CUDA(cudaGetLastError());
    return BQ_OK;
  }
  TempSet tmp(al);
  QueryScratch qs;
  BQ_TRY(prepare_queries((const float *)bvh->nodes, queries, nq, c.reorder != 0, tmp, al, qs));
  const int tie = c.tieMode, st = c.stackDepth, b = c.blockSize;
  if (tie == BQ_TIES_REFERENCE) {
    if (st == 32) launch_cp<TIE_REFERENCE, 32>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
    else if (st == 64) launch_cp<TIE_REFERENCE, 64>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
    else launch_cp<TIE_REFERENCE, 128>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
  } else {
    if (st == 32) launch_cp<TIE_LOWEST, 32>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
    else if (st == 64) launch_cp<TIE_LOWEST, 64>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
    else launch_cp<TIE_LOWEST, 128>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, al.s, ex);
  }
  BQ_CUDA(cudaGetLastError());
  return finish_queries(qs, al);
}

int knn(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k, float maxSqr,
        const bq_query_config *qcfg, int32_t *ids, float *d, int32_t *numFound, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (k < 1 || k > 64) return set_error(BQ_ERR_INVALID_ARGUMENT, "k must be in [1, 64]");
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    launch_pdl(k_fill_empty, dim3(div_up((uint64_t)nq * k, 256)), dim3(256), 0, al.s, nq, k, ids, d, numFound);
    BQ_CUDA(cudaGetLastError());
    return BQ_OK;
  }
  TempSet tmp(al);
  QueryScratch qs;
  BQ_TRY(prepare_queries((const float *)bvh->nodes, queries, nq, c.reorder != 0, tmp, al, qs));
  const int tie = c.tieMode, st = c.stackDepth, b = c.blockSize;
  if (c.lanesPerQuery > 1) {
    if (k > c.lanesPerQuery) return set_error(BQ_ERR_INVALID_ARGUMENT, "lanesPerQuery must be at least k");
    if (tie == BQ_TIES_REFERENCE)
      dispatch_knn_group<TIE_REFERENCE>(c.lanesPerQuery, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound,
                                        qs, al.s);
    else
      dispatch_knn_group<TIE_LOWEST>(c.lanesPerQuery, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound,
                                     qs, al.s);
    BQ_CUDA(cudaGetLastError());
    return finish_queries(qs, al);
  }
  if (k <= 4) dispatch_knn_tie<4>(tie, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound, qs, al.s);
  else if (k <= 8) dispatch_knn_tie<8>(tie, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound, qs, al.s);
  else if (k <= 16) dispatch_knn_tie<16>(tie, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound, qs, al.s);
  else if (k <= 32) dispatch_knn_tie<32>(tie, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound, qs, al.s);
  else dispatch_knn_tie<64>(tie, st, bvh, points, queries, nq, k, maxSqr, b, ids, d, numFound, qs, al.s);
  BQ_CUDA(cudaGetLastError());
  return finish_queries(qs, al);
}

int query_visit_counts(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k,
                       float maxSqr, const bq_query_config *qcfg, uint64_t *hostCounts, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (k < 0 || k > 64) return set_error(BQ_ERR_INVALID_ARGUMENT, "k must be 0 (closest point) or in [1, 64]");
  hostCounts[0] = hostCounts[1] = hostCounts[2] = 0;
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  TempSet tmp(al);
  unsigned long long *out = nullptr;
  BQ_TRY(tmp.get(&out, 3));
  BQ_CUDA(cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), al.s));
  if (c.tieMode == BQ_TIES_REFERENCE) launch_visit_count<TIE_REFERENCE>(bvh, points, queries, nq, k, maxSqr, out, al.s);
  else launch_visit_count<TIE_LOWEST>(bvh, points, queries, nq, k, maxSqr, out, al.s);
  BQ_CUDA(cudaGetLastError());
  unsigned long long h[3];
  BQ_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  for (int i = 0; i < 3; i++) hostCounts[i] = h[i];
  return BQ_OK;
}

} // namespace bq
