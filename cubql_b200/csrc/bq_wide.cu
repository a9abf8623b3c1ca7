// bq_wide.cu -- WideBVH<float,3,W>: collapse of a binary tree into a
// W-wide tree, and closest-point queries over it.
//
// Collapse (the reference: cuBQL/builder/cuda/wide_gpu_builder.h:40-213).
// A binary inner node whose depth is a multiple of log2(W) roots a wide
// node; the wide node's slots are the frontier of the binary treelet below
// it (leaves, and inner nodes one wide level down), taken in the order the
// reference's collapseExecute pops them from its stack (:131-149): the
// second child's subtree before the first's.  Four steps, all O(nodes):
//   k_wc_parent   parent of every binary node
//   k_wc_flag     depth by walking up the parents (the parent array of a
//                 10M-node tree is 40 MB and stays in L2), flag = wide root
//   scan          wide node id = number of wide roots with a lower binary
//                 index: deterministic, unlike the reference's atomicAdd
//                 numbering (:101-104), which varies from run to run
//   k_wc_emit     one thread per wide root writes its W slots
// The root is always wide node 0; a root that is a leaf gives one wide
// node with a single leaf slot (the reference only handles that case for
// a one-node tree, :93-95).
//
// Closest point (cuBQL/queries/points/findClosest.h:228-270 over
// cuBQL/traversal/shrinkingRadiusQuery.h:553-636): one thread per query,
// a wide node's valid slots within the cull radius become 64-bit keys
// (distance bits << 32 | payload), sorted ascending by the same exchange
// network as the reference's sort(ChildOrder) (:525-538); the nearest is
// entered, the others pushed farthest first.  Popped entries farther than
// the (shrunk) radius are dropped.  BQ_TIES_REFERENCE keeps exactly these
// rules; BQ_TIES_LOWEST_ID keeps nodes at the radius (with the 2^-20
// slack of the binary traversal) so the lowest id among equal distances
// wins.  A stack overflow re-runs the query from a deep global stack.
#include "bq_query.cuh"
#include "bq_wide.cuh"

namespace bq {

int build_spatial_median(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);

namespace {

constexpr uint32_t WC_NONE = 0xFFFFFFFFu;
constexpr uint32_t WC_MAX_DEPTH = 1u << 16;

__global__ void k_wc_parent(const Node *__restrict__ nodes, uint32_t numNodes, uint32_t *__restrict__ parent,
                            uint32_t *err)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || i == 1) return;  // node 1 is unused
  const uint64_t admin = node_admin(ldg_node(nodes + i));
  if (admin_count(admin) != 0) return;
  const uint64_t off = admin_offset(admin);
  if (off < 2 || off + 1 >= numNodes) {
    atomicOr(err, DEV_ERR_RANGE);
    return;
  }
  parent[off] = i;
  parent[off + 1] = i;
}

// flag[i] = 1 if binary node i roots a wide node
__global__ void k_wc_flag(const Node *__restrict__ nodes, uint32_t numNodes, const uint32_t *__restrict__ parent,
                          int logW, uint32_t *__restrict__ flag, uint32_t *err)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes) return;
  uint32_t f = 0;
  if (i == 0) {
    f = 1;
  } else if (i != 1 && admin_count(node_admin(ldg_node(nodes + i))) == 0) {
    uint32_t depth = 0, n = i;
    while (n != 0) {
      n = __ldg(parent + n);
      depth++;
      if (n >= numNodes || depth > WC_MAX_DEPTH) {  // unreachable node or a cycle
        depth = 1;
        if (n != WC_NONE) atomicOr(err, DEV_ERR_RANGE);
        break;
      }
    }
    f = (n == 0 && depth % logW == 0) ? 1u : 0u;
  }
  flag[i] = f;
}

template <int W>
__global__ void k_wc_emit(const Node *__restrict__ nodes, uint32_t numNodes, const uint32_t *__restrict__ flag,
                          const uint32_t *__restrict__ wideId, Node *__restrict__ wide, uint32_t numWide,
                          uint32_t *err)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || !__ldg(flag + i)) return;
  const uint32_t w = __ldg(wideId + i);
  if (w >= numWide) {
    atomicOr(err, DEV_ERR_RANGE);
    return;
  }
  Node *out = wide + (size_t)w * W;
  uint32_t stack[WideLog<W>::value + 2];
  int sp = 0, written = 0;
  stack[sp++] = i;
  while (sp > 0) {
    const uint32_t n = stack[--sp];
    const Node nd = ldg_node(nodes + n);
    const uint64_t admin = node_admin(nd);
    const uint32_t cnt = admin_count(admin);
    if (cnt > 0 || (n != i && __ldg(flag + n))) {
      if (written >= W) {
        atomicOr(err, DEV_ERR_RANGE);
        return;
      }
      const uint64_t word = cnt ? make_wslot(admin_offset(admin), cnt) : make_wslot(__ldg(wideId + n), 0);
      out[written++] = make_node(nd.a.x, nd.a.y, nd.a.z, nd.a.w, nd.b.x, nd.b.y, word);
    } else {
      const uint64_t off = admin_offset(admin);
      if (off + 1 >= numNodes || sp + 2 > WideLog<W>::value + 2) {
        atomicOr(err, DEV_ERR_RANGE);
        return;
      }
      stack[sp++] = (uint32_t)off;
      stack[sp++] = (uint32_t)off + 1;
    }
  }
  for (; written < W; written++)
    out[written] = make_node(INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, WSLOT_UNUSED);
}

// ------------------------------------------------------------------
// closest point over a wide tree
// ------------------------------------------------------------------
// the top WIDE_SMEM_STACK entries in shared memory (one column per thread,
// so a warp's pushes and pops are conflict-free), the rest in local memory:
// most wide traversals never go deeper than the shared part
constexpr int WIDE_SMEM_STACK = 8;
template <int S, int N>
struct WHybridStack {
  static_assert(S < N, "the shared part is the top of a deeper stack");
  uint64_t *sh;     // &shared[0][threadIdx.x]
  uint32_t stride;  // blockDim.x
  uint64_t e[N - S];
  int sp = 0;
  __device__ __forceinline__ explicit WHybridStack(uint64_t *base) : sh(base + threadIdx.x), stride(blockDim.x) {}
  __device__ __forceinline__ bool push(uint64_t v)
  {
    if (sp >= N) return false;
    if (sp < S) sh[(uint32_t)sp * stride] = v;
    else e[sp - S] = v;
    sp++;
    return true;
  }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ uint64_t pop()
  {
    --sp;
    return sp < S ? sh[(uint32_t)sp * stride] : e[sp - S];
  }
};

struct WGlobalStack {
  uint64_t *e;
  int cap;
  int sp = 0;
  __device__ __forceinline__ bool push(uint64_t v)
  {
    if (sp >= cap) return false;
    e[sp++] = v;
    return true;
  }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ uint64_t pop() { return e[--sp]; }
};

constexpr uint64_t WKEY_NONE = ~0ull;
constexpr uint32_t WNODE_NONE = 0xFFFFFFFFu;
constexpr uint32_t WLEAF_BIT = 0x80000000u;

__device__ __forceinline__ void cex(uint64_t &a, uint64_t &b)
{
  const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
  a = lo;
  b = hi;
}

// ascending sort of W unique keys: 1, 5 and 19 compare-exchanges (Batcher's
// odd-even merge for 8)
template <int W>
__device__ __forceinline__ void sort_keys(uint64_t v[W])
{
  if constexpr (W == 2) {
    cex(v[0], v[1]);
  } else if constexpr (W == 4) {
    cex(v[0], v[1]); cex(v[2], v[3]);
    cex(v[0], v[2]); cex(v[1], v[3]);
    cex(v[1], v[2]);
  } else {
    static_assert(W == 8, "width 2, 4 or 8");
    cex(v[0], v[1]); cex(v[2], v[3]); cex(v[4], v[5]); cex(v[6], v[7]);
    cex(v[0], v[2]); cex(v[1], v[3]); cex(v[4], v[6]); cex(v[5], v[7]);
    cex(v[1], v[2]); cex(v[5], v[6]);
    cex(v[0], v[4]); cex(v[1], v[5]); cex(v[2], v[6]); cex(v[3], v[7]);
    cex(v[2], v[4]); cex(v[3], v[5]);
    cex(v[1], v[2]); cex(v[3], v[4]); cex(v[5], v[6]);
  }
}

// Closest-point traversal of a WideBVH for the lowest-id tie rule, whose
// answer does not depend on the visiting order: leaf slots inside the
// (slack-widened) cull radius are processed as they are met, the nearest
// inner child is descended and the other inner children are pushed
// unsorted; popped entries beyond the shrunken radius are skipped.  Stack
// entries are (distance bits << 32 | wide node).  Returns false on stack
// overflow.
template <int W, typename Stack, typename Leaf>
__device__ __forceinline__ bool wide_traverse_lowest(const Node *__restrict__ slots, float qx, float qy, float qz,
                                                     float cull, Stack &st, Leaf &leaf)
{
  uint32_t nodeID = 0;
  while (true) {
    const Node *nd = slots + (size_t)nodeID * W;
    float cs = lowest_slack(cull);
    float nearD = INFINITY;
    uint32_t nearN = WNODE_NONE;
#pragma unroll
    for (int c = 0; c < W; c++) {
      const Node sl = ldg_node(nd + c);
      const uint64_t word = node_admin(sl);
      if (!wslot_valid(word)) continue;
      const float d = sqr_pbox(qx, qy, qz, sl.a.x, sl.a.y, sl.a.z, sl.a.w, sl.b.x, sl.b.y);
      if (d > cs) continue;
      if (wslot_count(word)) {  // a leaf: at once, so the radius shrinks before the next slots
        cull = fminf(cull, leaf(wslot_offset(word), wslot_count(word)));
        cs = lowest_slack(cull);
        continue;
      }
      const uint32_t child = (uint32_t)wslot_offset(word);
      if (d < nearD) {
        if (nearN != WNODE_NONE && !st.push(((uint64_t)__float_as_uint(nearD) << 32) | nearN)) return false;
        nearD = d;
        nearN = child;
      } else if (!st.push(((uint64_t)__float_as_uint(d) << 32) | child)) {
        return false;
      }
    }
    if (nearN != WNODE_NONE && !(nearD > lowest_slack(cull))) {
      nodeID = nearN;
      continue;
    }
    while (true) {
      if (st.empty()) return true;
      const uint64_t tos = st.pop();
      if (__uint_as_float((uint32_t)(tos >> 32)) <= lowest_slack(cull)) {
        nodeID = (uint32_t)tos;
        break;
      }
    }
  }
}

// shrinkingRadiusQuery::forEachLeaf over a WideBVH (:553-636).  Leaf
// functor as in bq_traverse.cuh.  Returns false on stack overflow.
template <int W, int TIE, typename Stack, typename Leaf>
__device__ __forceinline__ bool wide_traverse(const Node *__restrict__ slots, float qx, float qy, float qz, float cull,
                                              Stack &st, Leaf &leaf)
{
  constexpr int LOGW = WideLog<W>::value;
  uint32_t nodeID = 0;
  while (true) {
    while (true) {
      while (nodeID == WNODE_NONE) {
        if (st.empty()) return true;
        const uint64_t tos = st.pop();
        const float d = __uint_as_float((uint32_t)(tos >> 32));
        if (d > (TIE == TIE_REFERENCE ? cull : lowest_slack(cull))) continue;
        nodeID = (uint32_t)tos;
      }
      if (nodeID & WLEAF_BIT) break;
      const float cs = TIE == TIE_REFERENCE ? cull : lowest_slack(cull);
      uint64_t v[W];
#pragma unroll
      for (int c = 0; c < W; c++) {
        const Node sl = ldg_node(slots + (size_t)nodeID * W + c);
        const uint64_t word = node_admin(sl);
        v[c] = WKEY_NONE;
        if (wslot_valid(word)) {
          const float d = sqr_pbox(qx, qy, qz, sl.a.x, sl.a.y, sl.a.z, sl.a.w, sl.b.x, sl.b.y);
          if (!(d > cs)) {
            const uint32_t payload =
                wslot_count(word) ? (WLEAF_BIT | (nodeID << LOGW) | (uint32_t)c) : (uint32_t)wslot_offset(word);
            v[c] = ((uint64_t)__float_as_uint(d) << 32) | payload;
          }
        }
      }
      // sort(ChildOrder<W>) (:525-538).  The keys are unique (the payload
      // differs per slot), so any sorting network gives the reference's
      // exchange-network order; these are the shortest ones.
      sort_keys<W>(v);
#pragma unroll
      for (int c = W - 1; c > 0; --c)
        if (v[c] != WKEY_NONE && !st.push(v[c])) return false;
      nodeID = v[0] == WKEY_NONE ? WNODE_NONE : (uint32_t)v[0];
    }
    const uint32_t c = nodeID & (W - 1);
    const uint32_t n = (nodeID & ~WLEAF_BIT) >> LOGW;
    const uint64_t word = node_admin(ldg_node(slots + (size_t)n * W + c));
    cull = fminf(cull, leaf(wslot_offset(word), wslot_count(word)));
    nodeID = WNODE_NONE;
  }
}

template <int W, int TIE, typename Stack>
__device__ __forceinline__ bool run_wide_cp(const Node *slots, const uint32_t *primIDs, const float *points,
                                            const float *queries, uint32_t qi, float maxSqr, Stack &st,
                                            int32_t *outIds, float *outD)
{
  const float *q = queries + 3ull * qi;
  CPLeaf<TIE> leaf{primIDs, points, __ldg(q), __ldg(q + 1), __ldg(q + 2), maxSqr, -1, -1, 0};
  if constexpr (TIE == TIE_LOWEST) {
    if (!wide_traverse_lowest<W>(slots, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) return false;
  } else {
    if (!wide_traverse<W, TIE>(slots, leaf.qx, leaf.qy, leaf.qz, maxSqr, st, leaf)) return false;
  }
  outIds[qi] = leaf.id;
  outD[qi] = leaf.id >= 0 ? leaf.best : INFINITY;
  return true;
}

template <int W, int TIE, int STACK>
__global__ void __launch_bounds__(128) k_wide_closest(const Node *__restrict__ slots,
                                                      const uint32_t *__restrict__ primIDs,
                                                      const float *__restrict__ points,
                                                      const float *__restrict__ queries,
                                                      const uint32_t *__restrict__ order, uint32_t nq, float maxSqr,
                                                      int32_t *__restrict__ outIds, float *__restrict__ outD,
                                                      uint32_t *__restrict__ ovfList, uint32_t *ovfCount)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t qi = order ? __ldg(order + t) : t;
  extern __shared__ uint64_t sWideStack[];
  WHybridStack<WIDE_SMEM_STACK, STACK> st(sWideStack);
  if (!run_wide_cp<W, TIE>(slots, primIDs, points, queries, qi, maxSqr, st, outIds, outD))
    ovfList[atomicAdd(ovfCount, 1u)] = qi;
}

template <int W, int TIE>
__global__ void k_wide_closest_deep(const Node *__restrict__ slots, const uint32_t *__restrict__ primIDs,
                                    const float *__restrict__ points, const float *__restrict__ queries, float maxSqr,
                                    int32_t *__restrict__ outIds, float *__restrict__ outD, const uint32_t *ovfList,
                                    const uint32_t *ovfCount, uint64_t *stacks, uint32_t *err)
{
  griddep_wait();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t qi = ovfList[w];
    WGlobalStack st{stacks + (size_t)tid * DEEP_STACK, DEEP_STACK, 0};
    if (!run_wide_cp<W, TIE>(slots, primIDs, points, queries, qi, maxSqr, st, outIds, outD)) {
      outIds[qi] = -1;
      outD[qi] = INFINITY;
      atomicOr(err, DEV_ERR_STACK);
    }
  }
}

template <int W, int TIE, int STACK>
void launch_wide_cp(const bq_wide_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, float maxSqr,
                    int block, int32_t *ids, float *d, QueryScratch &qs, cudaStream_t s)
{
  const Node *slots = (const Node *)bvh->nodes;
  {
    ProfScope ps("wide.closest", s);
    launch_pdl(k_wide_closest<W, TIE, STACK>, dim3(div_up(nq, block)), dim3(block),
               WIDE_SMEM_STACK * sizeof(uint64_t) * block, s, slots, bvh->primIDs, points, queries, qs.order, nq,
               maxSqr, ids, d, qs.ovfList, qs.ovfCount);
  }
  ProfScope ps("wide.deep", s);
  launch_pdl(k_wide_closest_deep<W, TIE>, dim3(DEEP_THREADS / 128), dim3(128), 0, s, slots, bvh->primIDs, points,
             queries, maxSqr, ids, d, qs.ovfList, qs.ovfCount, (uint64_t *)qs.deep, qs.err);
}

template <int W>
void dispatch_wide_cp(int tie, int st, const bq_wide_bvh3f *bvh, const float *points, const float *queries,
                      uint32_t nq, float maxSqr, int b, int32_t *ids, float *d, QueryScratch &qs, cudaStream_t s)
{
  if (tie == BQ_TIES_REFERENCE) {
    if (st == 32) launch_wide_cp<W, TIE_REFERENCE, 32>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
    else if (st == 64) launch_wide_cp<W, TIE_REFERENCE, 64>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
    else launch_wide_cp<W, TIE_REFERENCE, 128>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
  } else {
    if (st == 32) launch_wide_cp<W, TIE_LOWEST, 32>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
    else if (st == 64) launch_wide_cp<W, TIE_LOWEST, 64>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
    else launch_wide_cp<W, TIE_LOWEST, 128>(bvh, points, queries, nq, maxSqr, b, ids, d, qs, s);
  }
}

} // namespace

int query_config(const bq_query_config *q, bq_query_config &out);

int wide_closest_point(const bq_wide_bvh3f *bvh, int W, const float *points, const float *queries, uint32_t nq,
                       float maxSqr, const bq_query_config *qcfg, int32_t *ids, float *d, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    launch_pdl(k_fill_empty, dim3(div_up(nq, 256)), dim3(256), 0, al.s, nq, 1, ids, d, nullptr);
    BQ_CUDA(cudaGetLastError());
    return BQ_OK;
  }
  TempSet tmp(al);
  float *rootBox = nullptr;
  BQ_TRY(tmp.get(&rootBox, 6));
  const Node *slots = (const Node *)bvh->nodes;
  if (W == 2) launch_pdl(k_wide_root_box<2>, dim3(1), dim3(32), 0, al.s, slots, rootBox);
  else if (W == 4) launch_pdl(k_wide_root_box<4>, dim3(1), dim3(32), 0, al.s, slots, rootBox);
  else launch_pdl(k_wide_root_box<8>, dim3(1), dim3(32), 0, al.s, slots, rootBox);
  BQ_CUDA(cudaGetLastError());
  QueryScratch qs;
  BQ_TRY(prepare_queries(rootBox, queries, nq, c.reorder != 0, tmp, al, qs));
  if (W == 2) dispatch_wide_cp<2>(c.tieMode, c.stackDepth, bvh, points, queries, nq, maxSqr, c.blockSize, ids, d, qs, al.s);
  else if (W == 4) dispatch_wide_cp<4>(c.tieMode, c.stackDepth, bvh, points, queries, nq, maxSqr, c.blockSize, ids, d, qs, al.s);
  else dispatch_wide_cp<8>(c.tieMode, c.stackDepth, bvh, points, queries, nq, maxSqr, c.blockSize, ids, d, qs, al.s);
  BQ_CUDA(cudaGetLastError());
  return finish_queries(qs, al);
}

// Collapses `bin` into `out` (W = 2, 4 or 8).  The primIDs are moved
// (copyPrims false: out takes bin's array) or copied.
int collapse_wide(const bq_bvh3f *bin, int W, bq_wide_bvh3f *out, bool copyPrims, Alloc &al)
{
  out->nodes = nullptr;
  out->numNodes = 0;
  out->primIDs = nullptr;
  out->numPrims = 0;
  const uint32_t nn = bin->numNodes;
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nn == 0) return BQ_OK;
  const int logW = W == 2 ? 1 : (W == 4 ? 2 : 3);
  const Node *nodes = (const Node *)bin->nodes;
  TempSet tmp(al);
  uint32_t *parent = nullptr, *flag = nullptr, *wid = nullptr, *ctl = nullptr;
  BQ_TRY(tmp.get(&parent, nn));
  BQ_TRY(tmp.get(&flag, nn));
  BQ_TRY(tmp.get(&wid, nn));
  BQ_TRY(tmp.get(&ctl, 2));  // [0] wide node count [1] device error bits
  BQ_CUDA(cudaMemsetAsync(parent, 0xFF, sizeof(uint32_t) * nn, al.s));
  BQ_CUDA(cudaMemsetAsync(ctl, 0, 8, al.s));
  {
    ProfScope ps("wide.flags", al.s, 2);
    launch_pdl(k_wc_parent, dim3(div_up(nn, 256)), dim3(256), 0, al.s, nodes, nn, parent, ctl + 1);
    launch_pdl(k_wc_flag, dim3(div_up(nn, 256)), dim3(256), 0, al.s, nodes, nn, parent, logW, flag, ctl + 1);
  }
  BQ_CUDA(cudaGetLastError());
  {
    ProfScope ps("wide.scan", al.s, 3);
    BQ_TRY(exclusive_scan_u32(flag, wid, nn, nullptr, ctl, al));
  }
  uint32_t h[2];
  BQ_CUDA(cudaMemcpyAsync(h, ctl, 8, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (h[1]) return set_error(BQ_ERR_INVALID_ARGUMENT, "binary tree has a child offset out of range or a cycle");
  const uint32_t numWide = h[0];
  Node *wide = nullptr;
  BQ_TRY(al.get(&wide, (size_t)numWide * W));
  uint32_t *prims = bin->primIDs;
  if (copyPrims) {
    if (al.get(&prims, bin->numPrims) != BQ_OK) {
      al.free_bytes(wide);
      return BQ_ERR_ALLOC;
    }
    cudaError_t ce = cudaMemcpyAsync(prims, bin->primIDs, sizeof(uint32_t) * bin->numPrims,
                                     cudaMemcpyDeviceToDevice, al.s);
    if (ce != cudaSuccess) {
      al.free_bytes(prims);
      al.free_bytes(wide);
      return cuda_error(ce, "collapse primIDs copy");
    }
  }
  {
    ProfScope ps("wide.emit", al.s);
    if (W == 2) launch_pdl(k_wc_emit<2>, dim3(div_up(nn, 256)), dim3(256), 0, al.s, nodes, nn, flag, wid, wide,
                           numWide, ctl + 1);
    else if (W == 4) launch_pdl(k_wc_emit<4>, dim3(div_up(nn, 256)), dim3(256), 0, al.s, nodes, nn, flag, wid, wide,
                                numWide, ctl + 1);
    else launch_pdl(k_wc_emit<8>, dim3(div_up(nn, 256)), dim3(256), 0, al.s, nodes, nn, flag, wid, wide, numWide,
                    ctl + 1);
  }
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h[1], ctl + 1, 4, cudaMemcpyDeviceToHost, al.s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(al.s);
  if (ce != cudaSuccess || h[1]) {
    if (copyPrims) al.free_bytes(prims);
    al.free_bytes(wide);
    if (ce != cudaSuccess) return cuda_error(ce, "collapse");
    return set_error(BQ_ERR_INVALID_ARGUMENT, "binary tree is not a valid BinaryBVH (treelet wider than W)");
  }
  out->nodes = reinterpret_cast<bq_wide_child3f *>(wide);
  out->numNodes = numWide;
  out->primIDs = prims;
  out->numPrims = bin->numPrims;
  return BQ_OK;
}

int build_wide(bq_wide_bvh3f *out, int W, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al)
{
  out->nodes = nullptr;
  out->numNodes = 0;
  out->primIDs = nullptr;
  out->numPrims = 0;
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  bq_bvh3f bin;
  BQ_TRY(build_spatial_median(&bin, boxes, n, cfg, al));
  const int s = collapse_wide(&bin, W, out, false, al);
  al.free_bytes(bin.nodes);
  if (s != BQ_OK) al.free_bytes(bin.primIDs);
  return s;
}

} // namespace bq
