// bq_sm.cu -- spatial-median BVH builder (the cuBQL::gpuBuilder method).
//
// Same splitting rule as gpuBuilder_impl (cuBQL/builder/cuda/sm_builder.h:
// 147-426): a node with more than makeLeafThreshold prims is split at the
// middle of its prims' centroid bounds along the widest axis (prims with
// centre >= pos go right); a node whose centroid bounds are flat or too thin
// to split (dim == -1) deals its prims to the two sides alternately.
//
// Different mechanics, B200-first: the reference re-reads every prim at
// every level and grows child counts and centroid boxes with global
// atomics (shared-memory ones for the first 512 new nodes).  Here each
// level works on a compacted array holding only the prims of still-open
// nodes, stored as float4 (centre xyz, primID):
//   k_sm_select    per open node: leaf (prims copied to their final slots)
//                  or split plane
//   scans          child numbering (BFS order, like a level-synchronous
//                  allocator) and the next level's compacted layout
//   k_sm_flags     per prim: side; one scan of the right-side flags gives
//                  every prim its stable position inside its child
//   k_sm_children  per split node: child ranges, child node ids
//   k_sm_scatter   per prim: move to the next level's array
//   k_sm_bounds    per tile: centroid bounds of the children, reduced in
//                  shared memory; one atomicMin/Max per (tile, node) merges
//                  tiles (min/max is order-independent: deterministic)
// Degenerate nodes send their k-th prim (primID order) to side
// (t0 + k) & 1, where t0 is the encoded centroid lower-z: that is the
// start value of the reference's tie-break counter, which aliases that
// field (sm_builder.h:82-103, 362-364), so child sizes match it exactly.
// Leaves list their prims in ascending primID order, like the
// reference's final (nodeID, primID) sort (sm_builder.h:565-605).
// One small device-to-host read per level decides when to stop.
#include <algorithm>
#include <climits>
#include <cfloat>

#include "bq_internal.cuh"

namespace bq {
int refit(const bq_bvh3f *bvh, const bq_box3f *boxes, Alloc &al);

namespace {

struct SmNode {
  uint32_t cbegin, count, fbegin, nodeID;
  int32_t lo[3], hi[3];
};

constexpr int SB_TILE = 1024;

__device__ __forceinline__ float ctr2(float lo, float hi) { return __fdiv_rn(__fadd_rn(lo, hi), 2.0f); }

__global__ void k_sm_valid(const bq_box3f *__restrict__ boxes, uint32_t n, uint32_t *__restrict__ valid)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 a = *reinterpret_cast<const float2 *>(boxes + i);
  const float2 b = *(reinterpret_cast<const float2 *>(boxes + i) + 1);
  valid[i] = (a.x <= b.y) ? 1u : 0u;  // initPrims: lower.x <= upper.x (sm_builder.h:134)
}

__global__ void k_sm_init(const bq_box3f *__restrict__ boxes, uint32_t n, const uint32_t *__restrict__ vpos,
                          const uint32_t *nvPtr, float4 *__restrict__ pc, uint32_t *__restrict__ pn,
                          uint32_t *__restrict__ primIDs, SmNode *root)
{
  const uint32_t nv = *nvPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    root->cbegin = 0; root->count = nv; root->fbegin = 0; root->nodeID = 0;
    for (int d = 0; d < 3; d++) { root->lo[d] = INT_MAX; root->hi[d] = INT_MIN; }
  }
  if (i >= n) return;
  const bq_box3f b = boxes[i];
  const uint32_t p = vpos[i];
  if (b.lower[0] <= b.upper[0]) {
    pc[p] = make_float4(ctr2(b.lower[0], b.upper[0]), ctr2(b.lower[1], b.upper[1]), ctr2(b.lower[2], b.upper[2]),
                        __uint_as_float(i));
    pn[p] = 0;
  } else {
    primIDs[nv + (i - p)] = i;  // invalid prims after all valid ones, ascending
  }
}

__global__ void k_sm_select(const SmNode *__restrict__ list, uint32_t K, int thr, const float4 *__restrict__ pc,
                            uint32_t *__restrict__ isSplit, uint32_t *__restrict__ splitCount, int *__restrict__ dimArr,
                            float *__restrict__ posArr, uint32_t *__restrict__ tbArr, Node *__restrict__ out,
                            uint32_t *__restrict__ primIDs)
{
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const SmNode nd = list[k];
  if ((int64_t)nd.count <= thr) {  // selectSplits: leaf (sm_builder.h:183-191)
    out[nd.nodeID] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(nd.fbegin, nd.count));
    for (uint32_t j = 0; j < nd.count; j++) primIDs[nd.fbegin + j] = __float_as_uint(pc[nd.cbegin + j].w);
    isSplit[k] = 0;
    splitCount[k] = 0;
    return;
  }
  float widestWidth = 0.f, wLo = 0.f, wHi = 0.f, wCtr = 0.f;
  int widestDim = -1;
#pragma unroll
  for (int d = 0; d < 3; d++) {  // sm_builder.h:192-219
    const float lo = dec_f(nd.lo[d]), hi = dec_f(nd.hi[d]);
    const float width = __fsub_rn(hi, lo);
    if (width <= widestWidth) continue;
    const float ctr = __fmul_rn(0.5f, __fadd_rn(hi, lo));
    widestWidth = width; widestDim = d; wLo = lo; wHi = hi; wCtr = ctr;
  }
  dimArr[k] = (widestDim < 0 || wCtr == wLo || wCtr == wHi) ? -1 : widestDim;
  posArr[k] = wCtr;
  tbArr[k] = (uint32_t)nd.lo[2];
  isSplit[k] = 1;
  splitCount[k] = nd.count;
}

__device__ __forceinline__ int sm_side(const float4 c, uint32_t rankInNode, int dim, float pos, uint32_t tb)
{
  if (dim < 0) return (int)((tb + rankInNode) & 1u);
  const float v = dim == 0 ? c.x : (dim == 1 ? c.y : c.z);
  return v >= pos ? 1 : 0;
}

__global__ void k_sm_flags(const float4 *__restrict__ pc, const uint32_t *__restrict__ pn, uint32_t A,
                           const SmNode *__restrict__ list, const uint32_t *__restrict__ isSplit,
                           const int *__restrict__ dimArr, const float *__restrict__ posArr,
                           const uint32_t *__restrict__ tbArr, uint32_t *__restrict__ right)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) right[A] = 0;
  if (i >= A) return;
  const uint32_t k = pn[i];
  uint32_t r = 0;
  if (isSplit[k]) r = (uint32_t)sm_side(pc[i], i - list[k].cbegin, dimArr[k], posArr[k], tbArr[k]);
  right[i] = r;
}

__global__ void k_sm_children(const SmNode *__restrict__ list, uint32_t K, const uint32_t *__restrict__ isSplit,
                              const uint32_t *__restrict__ rank, const uint32_t *__restrict__ nextBegin,
                              const uint32_t *__restrict__ Rx, uint32_t nodeBase, SmNode *__restrict__ next,
                              Node *__restrict__ out)
{
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K || !isSplit[k]) return;
  const SmNode nd = list[k];
  const uint32_t nR = Rx[nd.cbegin + nd.count] - Rx[nd.cbegin];
  const uint32_t nL = nd.count - nR;
  const uint32_t r = rank[k];
  const uint32_t child = nodeBase + 2 * r;
  out[nd.nodeID] = make_node(0.f, 0.f, 0.f, 0.f, 0.f, 0.f, make_admin(child, 0));
  SmNode c0, c1;
  c0.cbegin = nextBegin[k]; c0.count = nL; c0.fbegin = nd.fbegin; c0.nodeID = child;
  c1.cbegin = nextBegin[k] + nL; c1.count = nR; c1.fbegin = nd.fbegin + nL; c1.nodeID = child + 1;
  for (int d = 0; d < 3; d++) { c0.lo[d] = c1.lo[d] = INT_MAX; c0.hi[d] = c1.hi[d] = INT_MIN; }
  next[2 * r] = c0;
  next[2 * r + 1] = c1;
}

__global__ void k_sm_scatter(const float4 *__restrict__ pc, const uint32_t *__restrict__ pn, uint32_t A,
                             const SmNode *__restrict__ list, const uint32_t *__restrict__ isSplit,
                             const int *__restrict__ dimArr, const float *__restrict__ posArr,
                             const uint32_t *__restrict__ tbArr, const uint32_t *__restrict__ rank,
                             const uint32_t *__restrict__ nextBegin, const uint32_t *__restrict__ Rx,
                             float4 *__restrict__ pcNext, uint32_t *__restrict__ pnNext)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A) return;
  const uint32_t k = pn[i];
  if (!isSplit[k]) return;
  const SmNode nd = list[k];
  const float4 c = pc[i];
  const int side = sm_side(c, i - nd.cbegin, dimArr[k], posArr[k], tbArr[k]);
  const uint32_t rb = Rx[nd.cbegin];
  const uint32_t rBefore = Rx[i] - rb;
  const uint32_t nL = nd.count - (Rx[nd.cbegin + nd.count] - rb);
  const uint32_t dest = side ? nextBegin[k] + nL + rBefore : nextBegin[k] + (i - nd.cbegin) - rBefore;
  pcNext[dest] = c;
  pnNext[dest] = 2 * rank[k] + side;
}

__global__ void __launch_bounds__(256) k_sm_bounds(const float4 *__restrict__ pc, const uint32_t *__restrict__ pn,
                                                   uint32_t A, SmNode *__restrict__ list)
{
  __shared__ int32_t sLo[3][SB_TILE], sHi[3][SB_TILE];
  const uint32_t t0 = blockIdx.x * SB_TILE;
  const uint32_t t1 = min(A, t0 + SB_TILE);
  const uint32_t first = pn[t0];
  const uint32_t nLocal = pn[t1 - 1] - first + 1;  // pn is non-decreasing
  for (uint32_t j = threadIdx.x; j < nLocal; j += blockDim.x)
    for (int d = 0; d < 3; d++) { sLo[d][j] = INT_MAX; sHi[d][j] = INT_MIN; }
  __syncthreads();
  for (uint32_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
    const float4 c = pc[i];
    const uint32_t j = pn[i] - first;
    const int32_t e0 = enc_f(c.x), e1 = enc_f(c.y), e2 = enc_f(c.z);
    atomicMin(&sLo[0][j], e0); atomicMin(&sLo[1][j], e1); atomicMin(&sLo[2][j], e2);
    atomicMax(&sHi[0][j], e0); atomicMax(&sHi[1][j], e1); atomicMax(&sHi[2][j], e2);
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < nLocal; j += blockDim.x) {
    if (sLo[0][j] == INT_MAX && sHi[0][j] == INT_MIN) continue;
    SmNode *nd = list + first + j;
    for (int d = 0; d < 3; d++) {
      atomicMin(&nd->lo[d], sLo[d][j]);
      atomicMax(&nd->hi[d], sHi[d][j]);
    }
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
  uint32_t *valid = nullptr, *vpos = nullptr, *counts = nullptr, *pnA = nullptr, *pnB = nullptr, *right = nullptr;
  float4 *pcA = nullptr, *pcB = nullptr;
  SmNode *listA = nullptr, *listB = nullptr;
  uint32_t *isSplit = nullptr, *splitCount = nullptr, *rank = nullptr, *nextBegin = nullptr, *tb = nullptr;
  int *dim = nullptr;
  float *pos = nullptr;
  Node *tnodes = nullptr;
  BQ_TRY(tmp.get(&valid, n));
  BQ_TRY(tmp.get(&vpos, n));
  BQ_TRY(tmp.get(&counts, 4));  // [0] valid count, [1] #splits, [2] next active count
  BQ_TRY(tmp.get(&pcA, n));
  BQ_TRY(tmp.get(&pcB, n));
  BQ_TRY(tmp.get(&pnA, n));
  BQ_TRY(tmp.get(&pnB, n));
  BQ_TRY(tmp.get(&right, n + 1ull));
  BQ_TRY(tmp.get(&listA, n));
  BQ_TRY(tmp.get(&listB, n));
  BQ_TRY(tmp.get(&isSplit, n));
  BQ_TRY(tmp.get(&splitCount, n));
  BQ_TRY(tmp.get(&rank, n));
  BQ_TRY(tmp.get(&nextBegin, n));
  BQ_TRY(tmp.get(&tb, n));
  BQ_TRY(tmp.get(&dim, n));
  BQ_TRY(tmp.get(&pos, n));
  BQ_TRY(tmp.get(&tnodes, 2ull * n + 2));
  uint32_t *primIDs = nullptr;
  BQ_TRY(al.get(&primIDs, n));
  auto fail = [&](int code) {
    al.free_bytes(primIDs);
    return code;
  };
  cudaError_t ce;
  int s;
  k_sm_valid<<<div_up(n, 256), 256, 0, al.s>>>(boxes, n, valid);
  if ((s = exclusive_scan_u32(valid, vpos, n, nullptr, counts, al)) != BQ_OK) return fail(s);
  k_sm_init<<<div_up(n, 256), 256, 0, al.s>>>(boxes, n, vpos, counts, pcA, pnA, primIDs, listA);
  uint32_t hc[4] = {0, 0, 0, 0};
  if ((ce = cudaMemcpyAsync(hc, counts, 4, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess) return fail(cuda_error(ce, "copy"));
  if ((ce = cudaStreamSynchronize(al.s)) != cudaSuccess) return fail(cuda_error(ce, "sync"));
  const uint32_t nv = hc[0];
  if (nv == 0) {  // nothing to build over
    al.free_bytes(primIDs);
    return BQ_OK;
  }
  uint32_t A = nv, K = 1, nodeBase = 2;
  k_sm_bounds<<<div_up(A, SB_TILE), 256, 0, al.s>>>(pcA, pnA, A, listA);
  float4 *pcCur = pcA, *pcNext = pcB;
  uint32_t *pnCur = pnA, *pnNext = pnB;
  SmNode *listCur = listA, *listNext = listB;
  while (K > 0) {
    {
      ProfScope ps("sm.nodes", al.s, 7);
      k_sm_select<<<div_up(K, 128), 128, 0, al.s>>>(listCur, K, thr, pcCur, isSplit, splitCount, dim, pos, tb, tnodes,
                                                    primIDs);
      if ((s = exclusive_scan_u32(isSplit, rank, K, nullptr, counts + 1, al)) != BQ_OK) return fail(s);
      if ((s = exclusive_scan_u32(splitCount, nextBegin, K, nullptr, counts + 2, al)) != BQ_OK) return fail(s);
    }
    {
      ProfScope ps("sm.partition", al.s, 6);
      k_sm_flags<<<div_up(A, 256), 256, 0, al.s>>>(pcCur, pnCur, A, listCur, isSplit, dim, pos, tb, right);
      if ((s = exclusive_scan_u32(right, right, A + 1, nullptr, nullptr, al)) != BQ_OK) return fail(s);
      k_sm_children<<<div_up(K, 128), 128, 0, al.s>>>(listCur, K, isSplit, rank, nextBegin, right, nodeBase,
                                                      listNext, tnodes);
      k_sm_scatter<<<div_up(A, 256), 256, 0, al.s>>>(pcCur, pnCur, A, listCur, isSplit, dim, pos, tb, rank,
                                                     nextBegin, right, pcNext, pnNext);
    }
    {
      ProfScope ps("sm.sync", al.s, 0);
      if ((ce = cudaMemcpyAsync(hc + 1, counts + 1, 8, cudaMemcpyDeviceToHost, al.s)) != cudaSuccess)
        return fail(cuda_error(ce, "copy"));
      if ((ce = cudaStreamSynchronize(al.s)) != cudaSuccess) return fail(cuda_error(ce, "sync"));
    }
    const uint32_t S = hc[1], An = hc[2];
    if (S > 0) {
      ProfScope ps("sm.bounds", al.s);
      k_sm_bounds<<<div_up(An, SB_TILE), 256, 0, al.s>>>(pcNext, pnNext, An, listNext);
    }
    if ((ce = cudaGetLastError()) != cudaSuccess) return fail(cuda_error(ce, "spatial median level"));
    nodeBase += 2 * S;
    K = 2 * S;
    A = An;
    std::swap(pcCur, pcNext);
    std::swap(pnCur, pnNext);
    std::swap(listCur, listNext);
  }
  const uint32_t numNodes = nodeBase;
  Node *nodes = nullptr;
  if ((s = al.get(&nodes, numNodes)) != BQ_OK) return fail(s);
  if ((ce = cudaMemcpyAsync(nodes, tnodes, sizeof(Node) * numNodes, cudaMemcpyDeviceToDevice, al.s)) != cudaSuccess) {
    al.free_bytes(nodes);
    return fail(cuda_error(ce, "copy nodes"));
  }
  if ((ce = cudaMemsetAsync(nodes + 1, 0, sizeof(Node), al.s)) != cudaSuccess) {
    al.free_bytes(nodes);
    return fail(cuda_error(ce, "memset"));
  }
  bvh->nodes = reinterpret_cast<bq_node3f *>(nodes);
  bvh->numNodes = numNodes;
  bvh->primIDs = primIDs;
  bvh->numPrims = n;  // sm_builder.h:584: invalid prims stay listed after the valid ones
  if ((s = refit(bvh, boxes, al)) != BQ_OK) {
    al.free_bytes(nodes);
    bvh->nodes = nullptr; bvh->numNodes = 0; bvh->primIDs = nullptr; bvh->numPrims = 0;
    return fail(s);
  }
  return BQ_OK;
}

} // namespace bq
