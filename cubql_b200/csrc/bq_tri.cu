// bq_tri.cu -- point-to-triangle closest point (forward) and its adjoint.
//
// Forward: cuBQL::triangles::findClosest (cuBQL/queries/triangles/
// findClosest.h:132-152) over an indexed mesh, batched like the point
// queries (Morton-ordered queries, local stack, deep-stack fallback).  The
// per-triangle arithmetic follows findClosest.h:56-122 expression for
// expression (edge projections with clamped t, the three edge-plane tests,
// the normalised plane distance), so nvcc contracts it as it does the
// reference's.
//
// Adjoint (no counterpart in the reference): for the closest point
// X = sum_k w_k v_k with barycentric weights w on the fixed simplex, the
// envelope theorem gives
//     d sqrDist / d q   =  2 (q - X)
//     d sqrDist / d v_k = -2 w_k (q - X).
// Per query the three vertex contributions become (vertexID, pair index)
// records; a stable radix sort by vertex id groups them and one thread per
// vertex sums its group in sorted order.  No float atomics: the result is
// bitwise reproducible.
#include <algorithm>

#include "bq_traverse.cuh"

namespace bq {
namespace {

constexpr int DEEP_THREADS = 2048;
constexpr int DEEP_STACK = 1024;
// stack entries a triangle-query thread keeps in shared memory (the top of
// its traversal stack); the rest of the stack is in local memory.  Measured
// on the 4M-query, 1.31M-triangle workload: 45.0 ms with none, 46.4 with 8,
// 44.8 with 16 -- the kernel waits on its node and vertex loads, not on the
// stack -- so none.
constexpr int TRI_SMEM_STACK = 0;

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
// dot as the reference's accumulating loop (cuBQL/math/vec.h:459-466)
__device__ __forceinline__ float v3dot(V3 a, V3 b)
{
  float r = 0.f;
  r += a.x * b.x;
  r += a.y * b.y;
  r += a.z * b.z;
  return r;
}
// cuBQL/math/vec.h:232-237
__device__ __forceinline__ V3 v3cross(V3 a, V3 b)
{
  return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ V3 ldv(const float *verts, int32_t i)
{
  const float *p = verts + 3ll * i;
  return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// closest point on one triangle; region: 0 = inside (plane distance),
// 1 = edge ab, 2 = edge bc, 3 = edge ca; t = parameter along that edge
struct TriHit {
  float d;
  V3 P;
  int region;
  float t;
};

// Edge::closestPoint (findClosest.h:74-88)
__device__ __forceinline__ void edge_cp(TriHit &h, V3 a, V3 b, V3 p, int region)
{
  const V3 ba = v3sub(b, a);
  float t = v3dot(v3sub(p, a), ba) / v3dot(ba, ba);
  t = fminf(fmaxf(t, 0.f), 1.f);
  const V3 cp = V3{a.x + t * ba.x, a.y + t * ba.y, a.z + t * ba.z};
  const V3 dv = v3sub(cp, p);
  const float sd = v3dot(dv, dv);
  if (sd >= h.d) return;
  h.d = sd;
  h.P = cp;
  h.region = region;
  h.t = t;
}

// closestPoint(result, triangle, qp) (findClosest.h:93-122), evaluated
// against a running best starting at +inf
__device__ __forceinline__ TriHit tri_cp(V3 a, V3 b, V3 c, V3 qp)
{
  TriHit h;
  h.d = INFINITY;
  h.P = V3{0.f, 0.f, 0.f};
  h.region = -1;
  h.t = 0.f;
  V3 N = v3cross(v3sub(b, a), v3sub(c, a));
  const bool outside = (N.x == 0.f && N.y == 0.f && N.z == 0.f) ||
                       (v3dot(v3sub(qp, a), v3cross(v3sub(b, a), N)) >= 0.f) ||
                       (v3dot(v3sub(qp, b), v3cross(v3sub(c, b), N)) >= 0.f) ||
                       (v3dot(v3sub(qp, c), v3cross(v3sub(a, c), N)) >= 0.f);
  if (outside) {
    edge_cp(h, a, b, qp, 1);
    edge_cp(h, b, c, qp, 2);
    edge_cp(h, c, a, qp, 3);
    return h;
  }
  const float inv = 1.f / sqrtf(v3dot(N, N));
  N = V3{N.x * inv, N.y * inv, N.z * inv};
  const float sd = v3dot(v3sub(qp, a), N);
  h.d = sd * sd;
  h.P = V3{qp.x - sd * N.x, qp.y - sd * N.y, qp.z - sd * N.z};
  h.region = 0;
  return h;
}

template <int TIE>
struct TriLeaf {
  const uint32_t *__restrict__ primIDs;
  const int32_t *__restrict__ tris;
  const float *__restrict__ verts;
  V3 q;
  float best;
  int32_t id;
  V3 P;
  __device__ __forceinline__ float operator()(uint64_t off, uint32_t cnt)
  {
    for (uint32_t j = 0; j < cnt; j++) {
      const uint32_t pid = __ldg(primIDs + off + j);
      const int32_t *t = tris + 3ull * pid;
      const TriHit h = tri_cp(ldv(verts, __ldg(t)), ldv(verts, __ldg(t + 1)), ldv(verts, __ldg(t + 2)), q);
      const bool take = (TIE == TIE_REFERENCE) ? (h.d < best)
                                               : (h.d < best || (h.d == best && id >= 0 && (int32_t)pid < id));
      if (take) {
        best = h.d;
        id = (int32_t)pid;
        P = h.P;
      }
    }
    return best;
  }
};

template <int TIE, typename Stack>
__device__ __forceinline__ bool run_tri(const Node *nodes, const uint32_t *primIDs, const int32_t *tris,
                                        const float *verts, const float *queries, uint32_t qi, float maxSqr,
                                        Stack &st, int32_t *outIds, float *outD, float *outP)
{
  const float *qp = queries + 3ull * qi;
  TriLeaf<TIE> leaf{primIDs, tris, verts, V3{__ldg(qp), __ldg(qp + 1), __ldg(qp + 2)}, maxSqr, -1, V3{0.f, 0.f, 0.f}};
  if (!traverse<TIE>(nodes, leaf.q.x, leaf.q.y, leaf.q.z, maxSqr, st, leaf)) return false;
  outIds[qi] = leaf.id;
  outD[qi] = leaf.id >= 0 ? leaf.best : INFINITY;
  if (outP) {
    outP[3ull * qi + 0] = leaf.P.x;
    outP[3ull * qi + 1] = leaf.P.y;
    outP[3ull * qi + 2] = leaf.P.z;
  }
  return true;
}

template <int TIE, int STACK>
__global__ void __launch_bounds__(128) k_tri(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                             const int32_t *__restrict__ tris, const float *__restrict__ verts,
                                             const float *__restrict__ queries, const uint32_t *__restrict__ order,
                                             uint32_t nq, float maxSqr, int32_t *__restrict__ outIds,
                                             float *__restrict__ outD, float *__restrict__ outP,
                                             uint32_t *__restrict__ ovfList, uint32_t *ovfCount)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t qi = order ? __ldg(order + t) : t;
  extern __shared__ StackEntry sStack[];
  HybridStack<TRI_SMEM_STACK, STACK> st(sStack);
  if (!run_tri<TIE>(nodes, primIDs, tris, verts, queries, qi, maxSqr, st, outIds, outD, outP))
    ovfList[atomicAdd(ovfCount, 1u)] = qi;
}

template <int TIE>
__global__ void k_tri_deep(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                           const int32_t *__restrict__ tris, const float *__restrict__ verts,
                           const float *__restrict__ queries, float maxSqr, int32_t *__restrict__ outIds,
                           float *__restrict__ outD, float *__restrict__ outP, const uint32_t *ovfList,
                           const uint32_t *ovfCount, StackEntry *stacks, uint32_t *err)
{
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t qi = ovfList[w];
    GlobalStack st{stacks + (size_t)tid * DEEP_STACK, DEEP_STACK, 0};
    if (!run_tri<TIE>(nodes, primIDs, tris, verts, queries, qi, maxSqr, st, outIds, outD, outP)) {
      outIds[qi] = -1;
      outD[qi] = INFINITY;
      atomicOr(err, DEV_ERR_STACK);
    }
  }
}

// visit counts of the triangle traversal (measurement pass of the forward's
// roofline): node pairs loaded, admin loads, triangles tested
template <int TIE>
__global__ void __launch_bounds__(128) k_tri_visit_count(const Node *__restrict__ nodes,
                                                         const uint32_t *__restrict__ primIDs,
                                                         const int32_t *__restrict__ tris,
                                                         const float *__restrict__ verts,
                                                         const float *__restrict__ queries, uint32_t nq, float maxSqr,
                                                         unsigned long long *out)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  VisitCount vc;
  uint32_t prims = 0;
  if (t < nq) {  // no early return: every lane takes part in the warp sum below
    const float *qp = queries + 3ull * t;
    TriLeaf<TIE> leaf{primIDs, tris, verts, V3{__ldg(qp), __ldg(qp + 1), __ldg(qp + 2)}, maxSqr, -1,
                      V3{0.f, 0.f, 0.f}};
    CountingLeaf<TriLeaf<TIE>> cl{leaf};
    LocalStack<128> st;
    traverse_counted<TIE>(nodes, leaf.q.x, leaf.q.y, leaf.q.z, maxSqr, st, cl, vc);
    prims = cl.prims;
  }
  add_visit_counts(vc.pairs, vc.admins, prims, out);
}

__global__ void k_tri_keys(const Node *__restrict__ nodes, const float *__restrict__ queries, uint32_t nq,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ idx)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const Node root = ldg_node(nodes);
  const float ext = fmaxf(fmaxf(root.a.w - root.a.x, root.b.x - root.a.y), root.b.y - root.a.z);
  const float sc = 1024.0f / fmaxf(ext, 1e-20f);
  const float *q = queries + 3ull * t;
  const uint32_t cx = min(__float2uint_rz((q[0] - root.a.x) * sc), 1023u);
  const uint32_t cy = min(__float2uint_rz((q[1] - root.a.y) * sc), 1023u);
  const uint32_t cz = min(__float2uint_rz((q[2] - root.a.z) * sc), 1023u);
  keys[t] = spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
  idx[t] = t;
}

__global__ void k_tri_fill_empty(uint32_t nq, int32_t *ids, float *d, float *P)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  ids[t] = -1;
  d[t] = INFINITY;
  if (P) P[3ull * t] = P[3ull * t + 1] = P[3ull * t + 2] = 0.f;
}

// ------------------------------------------------------------------
// adjoint
// ------------------------------------------------------------------
__global__ void k_tri_bwd_pairs(const int32_t *__restrict__ tris, const float *__restrict__ verts,
                                const float *__restrict__ queries, uint32_t nq, const int32_t *__restrict__ ids,
                                const float *__restrict__ gradSqr, float *__restrict__ gradQ,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                float *__restrict__ contrib)
{
  const uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  const int32_t id = ids[qi];
  const float *qp = queries + 3ull * qi;
  const V3 q = V3{qp[0], qp[1], qp[2]};
  float r[3] = {0.f, 0.f, 0.f}, w[3] = {0.f, 0.f, 0.f};
  int32_t vi[3] = {-1, -1, -1};
  if (id >= 0) {
    const int32_t *t = tris + 3ll * id;
    vi[0] = t[0]; vi[1] = t[1]; vi[2] = t[2];
    const V3 a = ldv(verts, vi[0]), b = ldv(verts, vi[1]), c = ldv(verts, vi[2]);
    const TriHit h = tri_cp(a, b, c, q);
    if (h.region == 0) {
      // barycentric weights of the projection of q (the off-plane part of
      // q - a drops out of both triple products)
      const V3 N = v3cross(v3sub(b, a), v3sub(c, a));
      const float nn = v3dot(N, N);
      const V3 qa = v3sub(q, a);
      const float u = v3dot(v3cross(qa, v3sub(c, a)), N) / nn;
      const float v = v3dot(v3cross(v3sub(b, a), qa), N) / nn;
      w[0] = 1.f - u - v; w[1] = u; w[2] = v;
    } else if (h.region == 1) {
      w[0] = 1.f - h.t; w[1] = h.t;
    } else if (h.region == 2) {
      w[1] = 1.f - h.t; w[2] = h.t;
    } else if (h.region == 3) {
      w[2] = 1.f - h.t; w[0] = h.t;
    }
    const float g = 2.f * gradSqr[qi];
    r[0] = (q.x - h.P.x) * g;
    r[1] = (q.y - h.P.y) * g;
    r[2] = (q.z - h.P.z) * g;
  }
  gradQ[3ull * qi + 0] = r[0];
  gradQ[3ull * qi + 1] = r[1];
  gradQ[3ull * qi + 2] = r[2];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint64_t pi = 3ull * qi + k;
    keys[pi] = vi[k] >= 0 ? (uint32_t)vi[k] : 0xffffffffu;
    vals[pi] = (uint32_t)pi;
    contrib[3 * pi + 0] = -w[k] * r[0];
    contrib[3 * pi + 1] = -w[k] * r[1];
    contrib[3 * pi + 2] = -w[k] * r[2];
  }
}

__global__ void k_tri_bwd_reduce(const uint32_t *__restrict__ sortedKeys, const uint32_t *__restrict__ sortedVals,
                                 uint32_t numPairs, const float *__restrict__ contrib, uint32_t numVerts,
                                 float *__restrict__ gradV)
{
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= numVerts) return;
  uint32_t lo = 0, hi = numPairs;  // first pair with key >= v
  while (lo < hi) {
    uint32_t m = lo + ((hi - lo) >> 1);
    if (sortedKeys[m] < v) lo = m + 1; else hi = m;
  }
  float sx = 0.f, sy = 0.f, sz = 0.f;
  for (uint32_t j = lo; j < numPairs && sortedKeys[j] == v; j++) {
    const uint32_t p = sortedVals[j];
    sx += contrib[3ull * p + 0];
    sy += contrib[3ull * p + 1];
    sz += contrib[3ull * p + 2];
  }
  gradV[3ull * v + 0] = sx;
  gradV[3ull * v + 1] = sy;
  gradV[3ull * v + 2] = sz;
}

// Triangle::bounds() (cuBQL/queries/triangles/Triangle.h:40-41)
__global__ void k_tri_boxes(const int32_t *__restrict__ tris, const float *__restrict__ verts, uint32_t nt,
                            bq_box3f *__restrict__ boxes)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int32_t *ix = tris + 3ull * t;
  const V3 a = ldv(verts, ix[0]), b = ldv(verts, ix[1]), c = ldv(verts, ix[2]);
  bq_box3f bx;
  bx.lower[0] = fminf(fminf(fminf(INFINITY, a.x), b.x), c.x);
  bx.lower[1] = fminf(fminf(fminf(INFINITY, a.y), b.y), c.y);
  bx.lower[2] = fminf(fminf(fminf(INFINITY, a.z), b.z), c.z);
  bx.upper[0] = fmaxf(fmaxf(fmaxf(-INFINITY, a.x), b.x), c.x);
  bx.upper[1] = fmaxf(fmaxf(fmaxf(-INFINITY, a.y), b.y), c.y);
  bx.upper[2] = fmaxf(fmaxf(fmaxf(-INFINITY, a.z), b.z), c.z);
  boxes[t] = bx;
}

} // namespace

int query_config(const bq_query_config *q, bq_query_config &out);

int tri_closest(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries, uint32_t nq,
                float maxSqr, const bq_query_config *qcfg, int32_t *ids, float *d, float *P, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    k_tri_fill_empty<<<div_up(nq, 256), 256, 0, al.s>>>(nq, ids, d, P);
    BQ_CUDA(cudaGetLastError());
    return BQ_OK;
  }
  TempSet tmp(al);
  uint32_t *ovfList = nullptr, *ovfCount = nullptr, *order = nullptr;
  StackEntry *deep = nullptr;
  BQ_TRY(tmp.get(&ovfList, nq));
  BQ_TRY(tmp.get(&ovfCount, 2));
  BQ_TRY(tmp.get(&deep, (size_t)DEEP_THREADS * DEEP_STACK));
  BQ_CUDA(cudaMemsetAsync(ovfCount, 0, 8, al.s));
  uint32_t *err = ovfCount + 1;
  const Node *nodes = (const Node *)bvh->nodes;
  if (c.reorder && nq > 1) {
    uint32_t *keys[2], *idx[2];
    BQ_TRY(tmp.get(&keys[0], nq));
    BQ_TRY(tmp.get(&keys[1], nq));
    BQ_TRY(tmp.get(&idx[0], nq));
    BQ_TRY(tmp.get(&idx[1], nq));
    k_tri_keys<<<div_up(nq, 256), 256, 0, al.s>>>(nodes, queries, nq, keys[0], idx[0]);
    int sel = 0;
    BQ_TRY(onesweep_sort_u32(keys, idx, nq, nullptr, 6, 30, nullptr, &sel, err, al));  // order only: top 24 bits
    order = idx[sel];
  }
  const int b = c.blockSize;
#define BQ_TRI_LAUNCH(TIE, ST)                                                                                     \
  ProfScope ps("tri.closest", al.s, 2);                                                                            \
  k_tri<TIE, ST><<<div_up(nq, b), b, TRI_SMEM_STACK * sizeof(StackEntry) * b, al.s>>>(                           \
      nodes, bvh->primIDs, tris, verts, queries, order, nq, maxSqr, ids,                                           \
                                                d, P, ovfList, ovfCount);                                          \
  k_tri_deep<TIE><<<DEEP_THREADS / 128, 128, 0, al.s>>>(nodes, bvh->primIDs, tris, verts, queries, maxSqr, ids, d, \
                                                        P, ovfList, ovfCount, deep, err)
  if (c.tieMode == BQ_TIES_REFERENCE) {
    if (c.stackDepth == 32) { BQ_TRI_LAUNCH(TIE_REFERENCE, 32); }
    else if (c.stackDepth == 64) { BQ_TRI_LAUNCH(TIE_REFERENCE, 64); }
    else { BQ_TRI_LAUNCH(TIE_REFERENCE, 128); }
  } else {
    if (c.stackDepth == 32) { BQ_TRI_LAUNCH(TIE_LOWEST, 32); }
    else if (c.stackDepth == 64) { BQ_TRI_LAUNCH(TIE_LOWEST, 64); }
    else { BQ_TRI_LAUNCH(TIE_LOWEST, 128); }
  }
#undef BQ_TRI_LAUNCH
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr & DEV_ERR_STACK) return set_error(BQ_ERR_STACK_OVERFLOW, "query exceeded the deep fallback stack");
  if (herr & DEV_ERR_TIMEOUT) return set_error(BQ_ERR_TIMEOUT, "query reordering sort timed out");
  return BQ_OK;
}

int tri_distance_bwd(const int32_t *tris, const float *verts, uint32_t numVerts, const float *queries, uint32_t nq,
                     const int32_t *ids, const float *gradSqr, float *gradQ, float *gradV, Alloc &al)
{
  if (numVerts > 0x7fffffffu) return set_error(BQ_ERR_INVALID_ARGUMENT, "too many vertices");
  if (nq == 0) {
    if (numVerts) BQ_CUDA(cudaMemsetAsync(gradV, 0, sizeof(float) * 3ull * numVerts, al.s));
    return BQ_OK;
  }
  if ((uint64_t)nq * 3 >= (1ull << 30)) return set_error(BQ_ERR_INVALID_ARGUMENT, "too many queries for one call");
  const uint32_t np = nq * 3;
  TempSet tmp(al);
  uint32_t *keys[2], *vals[2], *err = nullptr;
  float *contrib = nullptr;
  BQ_TRY(tmp.get(&keys[0], np));
  BQ_TRY(tmp.get(&keys[1], np));
  BQ_TRY(tmp.get(&vals[0], np));
  BQ_TRY(tmp.get(&vals[1], np));
  BQ_TRY(tmp.get(&contrib, 3ull * np));
  BQ_TRY(tmp.get(&err, 1));
  BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  ProfScope ps("tri.backward", al.s, 5);
  k_tri_bwd_pairs<<<div_up(nq, 128), 128, 0, al.s>>>(tris, verts, queries, nq, ids, gradSqr, gradQ, keys[0], vals[0],
                                                     contrib);
  BQ_CUDA(cudaGetLastError());
  // enough key bits that the "no vertex" key 0xffffffff sorts after every id
  int bits = 1;
  while (bits < 32 && (1ull << bits) <= numVerts) bits++;
  int sel = 0;
  BQ_TRY(onesweep_sort_u32(keys, vals, np, nullptr, 0, bits, nullptr, &sel, err, al));
  if (numVerts)
    k_tri_bwd_reduce<<<div_up(numVerts, 256), 256, 0, al.s>>>(keys[sel], vals[sel], np, contrib, numVerts, gradV);
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr & DEV_ERR_TIMEOUT) return set_error(BQ_ERR_TIMEOUT, "vertex-gradient sort timed out");
  return BQ_OK;
}

int tri_boxes(const int32_t *tris, const float *verts, uint32_t nt, bq_box3f *boxes, cudaStream_t s)
{
  if (nt == 0) return BQ_OK;
  k_tri_boxes<<<div_up(nt, 256), 256, 0, s>>>(tris, verts, nt, boxes);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

int tri_visit_counts(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries, uint32_t nq,
                     float maxSqr, const bq_query_config *qcfg, uint64_t *hostCounts, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  hostCounts[0] = hostCounts[1] = hostCounts[2] = 0;
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  TempSet tmp(al);
  unsigned long long *out = nullptr;
  BQ_TRY(tmp.get(&out, 3));
  BQ_CUDA(cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), al.s));
  const Node *nodes = (const Node *)bvh->nodes;
  if (c.tieMode == BQ_TIES_REFERENCE)
    k_tri_visit_count<TIE_REFERENCE><<<div_up(nq, 128), 128, 0, al.s>>>(nodes, bvh->primIDs, tris, verts, queries, nq,
                                                                        maxSqr, out);
  else
    k_tri_visit_count<TIE_LOWEST><<<div_up(nq, 128), 128, 0, al.s>>>(nodes, bvh->primIDs, tris, verts, queries, nq,
                                                                     maxSqr, out);
  BQ_CUDA(cudaGetLastError());
  unsigned long long h[3];
  BQ_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  for (int i = 0; i < 3; i++) hostCounts[i] = h[i];
  return BQ_OK;
}

} // namespace bq
