// bq_traverse.cuh -- shrinking-radius stack traversal over a BinaryBVH.
//
// Same visiting order as cuBQL::shrinkingRadiusQuery::forEachLeaf
// (cuBQL/traversal/shrinkingRadiusQuery.h:409-508): both children of an
// inner node are loaded (2 x 32 B, each as two 16-byte vector loads), the
// nearer one is descended (ties to child 1), the farther one is pushed when
// it is inside the cull radius, leaves report a new radius, and popped
// entries are skipped once the radius has shrunk below them.
//
// TIE selects the comparison rules:
//   TIE_REFERENCE: exactly the reference's (cull at >=, push at <, pop at <=),
//     so results match its kernels bit for bit, ties included;
//   TIE_LOWEST:    nodes at exactly the cull distance are kept, so a leaf
//     functor can prefer the lowest primID among equal distances.
#pragma once

#include "bq_internal.cuh"

namespace bq {

enum { TIE_LOWEST = 0, TIE_REFERENCE = 1 };

struct StackEntry {
  uint32_t idx;
  float dist;
};

// fixed-size stack in local memory
template <int N>
struct LocalStack {
  StackEntry e[N];
  int sp = 0;
  __device__ __forceinline__ bool push(uint32_t i, float d)
  {
    if (sp >= N) return false;
    e[sp].idx = i;
    e[sp].dist = d;
    sp++;
    return true;
  }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ StackEntry pop() { return e[--sp]; }
};

// S entries in shared memory (this thread's column of a [S][blockDim]
// array, so a warp's accesses to the same depth hit 32 different banks
// pairs), the rest of N in local memory.  Shallow traversals never touch
// local memory.
template <int S, int N>
struct HybridStack {
  static_assert(S < N, "the shared part is the top of a deeper stack");
  StackEntry *sh;  // &shared[0][threadIdx.x]
  uint32_t stride; // blockDim.x
  StackEntry e[N - S];
  int sp = 0;
  __device__ __forceinline__ HybridStack(StackEntry *base) : sh(base + threadIdx.x), stride(blockDim.x) {}
  __device__ __forceinline__ bool push(uint32_t i, float d)
  {
    if (sp >= N) return false;
    const StackEntry x{i, d};
    if (sp < S) sh[(uint32_t)sp * stride] = x;
    else e[sp - S] = x;
    sp++;
    return true;
  }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ StackEntry pop()
  {
    --sp;
    return sp < S ? sh[(uint32_t)sp * stride] : e[sp - S];
  }
};

// deep stack in a caller-provided global-memory slice
struct GlobalStack {
  StackEntry *e;
  int cap;
  int sp = 0;
  __device__ __forceinline__ bool push(uint32_t i, float d)
  {
    if (sp >= cap) return false;
    e[sp].idx = i;
    e[sp].dist = d;
    sp++;
    return true;
  }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ StackEntry pop() { return e[--sp]; }
};

__device__ __forceinline__ uint64_t ldg_admin(const Node *p)
{
  const float4 b = __ldg(&p->b);
  return ((uint64_t)__float_as_uint(b.w) << 32) | __float_as_uint(b.z);
}

// In TIE_LOWEST mode node distances are compared against the cull radius
// widened by 2^-20 relative: a node box distance and the distance to a
// point inside it are rounded differently (each carries a few ulp of
// error), so without the slack a node holding an equally close point with
// a lower id could be culled by one ulp.  The slack only adds visits; the
// answer is decided by the exact per-prim comparisons.
__device__ __forceinline__ float lowest_slack(float c) { return __fmaf_rn(c, 0x1p-20f, c); }

// Node-visit counters of the traversal (the measurement pass of the query
// rooflines counts with VisitCount; the query kernels use NoVisitCount,
// which compiles to nothing).  pair(): both children of an inner node
// loaded (2 x 32 B); admin(): the admin half of one node loaded (16 B: the
// root, and every popped entry that is descended).
struct NoVisitCount {
  __device__ __forceinline__ void pair() {}
  __device__ __forceinline__ void admin() {}
};
struct VisitCount {
  uint32_t pairs = 0, admins = 0;
  __device__ __forceinline__ void pair() { pairs++; }
  __device__ __forceinline__ void admin() { admins++; }
};

// Leaf functor contract: float operator()(uint64_t offset, uint32_t count)
// processes primIDs[offset .. offset+count) and returns the new cull
// radius proposal.  Returns false if the stack overflowed (the query then
// has to be re-run with a deeper stack; its partial state is discarded).
template <int TIE, typename Stack, typename Leaf, typename Count>
__device__ __forceinline__ bool traverse_counted(const Node *__restrict__ nodes, float qx, float qy, float qz,
                                                 float cull, Stack &stack, Leaf &leaf, Count &count)
{
  uint64_t admin = ldg_admin(nodes);
  count.admin();
  while (true) {
    bool dead = false;
    while (admin_count(admin) == 0) {
      const uint64_t off = admin_offset(admin);
      const Node n0 = ldg_node(nodes + off);
      const Node n1 = ldg_node(nodes + off + 1);
      count.pair();
      const float d0 = sqr_pbox(qx, qy, qz, n0.a.x, n0.a.y, n0.a.z, n0.a.w, n0.b.x, n0.b.y);
      const float d1 = sqr_pbox(qx, qy, qz, n1.a.x, n1.a.y, n1.a.z, n1.a.w, n1.b.x, n1.b.y);
      const float dmin = fminf(d0, d1), dmax = fmaxf(d0, d1);
      const float cs = TIE == TIE_REFERENCE ? cull : lowest_slack(cull);
      if (TIE == TIE_REFERENCE ? (dmin >= cull) : (dmin > cs)) {
        dead = true;
        break;
      }
      uint32_t farID;
      if (d0 < d1) {
        admin = node_admin(n0);
        farID = (uint32_t)off + 1;
      } else {
        admin = node_admin(n1);
        farID = (uint32_t)off;
      }
      if (TIE == TIE_REFERENCE ? (dmax < cull) : (dmax <= cs)) {
        if (!stack.push(farID, dmax)) return false;
      }
    }
    if (!dead) cull = fminf(cull, leaf(admin_offset(admin), admin_count(admin)));
    while (true) {
      if (stack.empty()) return true;
      const StackEntry e = stack.pop();
      if (e.dist <= (TIE == TIE_REFERENCE ? cull : lowest_slack(cull))) {
        admin = ldg_admin(nodes + e.idx);
        count.admin();
        break;
      }
    }
  }
}

template <int TIE, typename Stack, typename Leaf>
__device__ __forceinline__ bool traverse(const Node *__restrict__ nodes, float qx, float qy, float qz, float cull,
                                         Stack &stack, Leaf &leaf)
{
  NoVisitCount none;
  return traverse_counted<TIE>(nodes, qx, qy, qz, cull, stack, leaf, none);
}

// a leaf functor that also counts the prims it is handed
template <typename Leaf>
struct CountingLeaf {
  Leaf &inner;
  uint32_t prims = 0;
  __device__ __forceinline__ float operator()(uint64_t off, uint32_t cnt)
  {
    prims += cnt;
    return inner(off, cnt);
  }
};

// adds one thread's counts to out[0..2] (node pairs, admin loads, prims),
// one atomic per warp and counter
__device__ __forceinline__ void add_visit_counts(uint32_t pairs, uint32_t admins, uint32_t prims,
                                                 unsigned long long *out)
{
  unsigned long long a = pairs, b = admins, c = prims;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
    c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, a);
    atomicAdd(out + 1, b);
    atomicAdd(out + 2, c);
  }
}

// ------------------------------------------------------------------
// candidate lists kept in registers
// ------------------------------------------------------------------
template <int TIE>
__device__ __forceinline__ bool cand_before(float d, int32_t id, float D, int32_t I)
{
  if (TIE == TIE_REFERENCE) return d < D;  // insert after equal distances (common/knn.h:67-71)
  return d < D || (d == D && id < I);
}

// sorted list of K (distance, id) pairs; slots [0, K-k) hold sentinels
// below every candidate so the k-th best always sits at index K-1
template <int K, int TIE>
struct KnnList {
  float D[K];
  int32_t I[K];
  __device__ __forceinline__ void init(int k)
  {
#pragma unroll
    for (int j = 0; j < K; j++) {
      const bool sentinel = j < K - k;
      D[j] = sentinel ? -1.0f : INFINITY;
      I[j] = sentinel ? -1 : 0x7fffffff;
    }
  }
  __device__ __forceinline__ float worst() const { return D[K - 1]; }
  __device__ __forceinline__ float dist(int j) const { return D[j]; }
  __device__ __forceinline__ int32_t id(int j) const { return I[j]; }
  __device__ __forceinline__ bool real(int j) const { return I[j] != 0x7fffffff && D[j] != INFINITY; }
  // insert if it belongs to the list
  __device__ __forceinline__ void offer(float d, int32_t id)
  {
    if (!cand_before<TIE>(d, id, D[K - 1], I[K - 1])) return;
#pragma unroll
    for (int j = K - 1; j >= 0; j--) {
      const bool fromPrev = (j > 0) && cand_before<TIE>(d, id, D[j > 0 ? j - 1 : 0], I[j > 0 ? j - 1 : 0]);
      const bool here = cand_before<TIE>(d, id, D[j], I[j]);
      const float nd = fromPrev ? D[j > 0 ? j - 1 : 0] : (here ? d : D[j]);
      const int32_t ni = fromPrev ? I[j > 0 ? j - 1 : 0] : (here ? id : I[j]);
      D[j] = nd;
      I[j] = ni;
    }
  }
};

// Lowest-id ties: a candidate is the 64-bit key (distance bits << 32 | id).
// Distances are >= +0, so key order is (distance, id) order and one 64-bit
// compare replaces the float compare, the equality test and the id compare.
constexpr uint64_t KNN_KEY_EMPTY = (0x7f800000ull << 32) | 0xffffffffull;  // (+inf, above every id)
template <int K>
struct KnnList<K, TIE_LOWEST> {
  uint64_t L[K];
  __device__ __forceinline__ void init(int k)
  {
#pragma unroll
    for (int j = 0; j < K; j++) L[j] = j < K - k ? 0ull : KNN_KEY_EMPTY;  // 0: below every candidate
  }
  __device__ __forceinline__ float worst() const { return __uint_as_float((uint32_t)(L[K - 1] >> 32)); }
  __device__ __forceinline__ float dist(int j) const { return __uint_as_float((uint32_t)(L[j] >> 32)); }
  __device__ __forceinline__ int32_t id(int j) const { return (int32_t)(uint32_t)L[j]; }
  __device__ __forceinline__ bool real(int j) const { return L[j] != KNN_KEY_EMPTY; }
  __device__ __forceinline__ void offer(float d, int32_t id)
  {
    const uint64_t key = ((uint64_t)__float_as_uint(d) << 32) | (uint32_t)id;
    if (!(key < L[K - 1])) return;
#pragma unroll
    for (int j = K - 1; j >= 0; j--) {
      const bool fromPrev = (j > 0) && key < L[j > 0 ? j - 1 : 0];
      const bool here = key < L[j];
      L[j] = fromPrev ? L[j > 0 ? j - 1 : 0] : (here ? key : L[j]);
    }
  }
};

} // namespace bq
