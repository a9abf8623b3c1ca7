// bq_batch_tri.cu -- batched meshes: refit of every mesh's tree and the
// closest-triangle query of every mesh's queries, each in one launch.
//
// Layout (as produced by bq_batched_build_morton63_f3 over triangle boxes):
// mesh s owns triangles tris[triOff[s] .. triOff[s+1]) (vertex indices into
// one shared vertex array), its tree's nodes sit in the block starting at
// nodes[2*triOff[s]] and its primIDs (mesh-local triangle ids) at
// primIDs[triOff[s]].  This is the per-step work of a differentiable
// fitting loop: move vertices, recompute triangle boxes, refit all trees,
// query, backpropagate (bq_tri_distance_bwd_f3 works on the shared arrays
// directly because the query returns global triangle ids).
#include <algorithm>

#include <cuda/atomic>

#include "bq_traverse.cuh"

namespace bq {
int query_config(const bq_query_config *q, bq_query_config &out);

namespace {

constexpr uint32_t BR_NO_PARENT = 0xffffffffu;
constexpr int DEEP_THREADS = 2048;
constexpr int DEEP_STACK = 1024;

__device__ __forceinline__ uint32_t seg_find(const uint32_t *__restrict__ off, uint32_t numSegs, uint32_t i)
{
  uint32_t lo = 0, hi = numSegs;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    if (__ldg(off + m) <= i) lo = m; else hi = m;
  }
  return lo;
}

// slot j of the node buffer belongs to the mesh whose block contains it;
// returns false for slots past that tree's node count
__device__ __forceinline__ bool node_slot(const bq_bvh3f *__restrict__ bvhs, const uint32_t *__restrict__ off,
                                          uint32_t numSegs, uint32_t j, uint32_t &s, uint32_t &local)
{
  s = seg_find(off, numSegs, j >> 1);
  local = j - 2 * __ldg(off + s);
  return local < bvhs[s].numNodes;
}

__global__ void k_brefit_parents(const Node *__restrict__ nodes, uint32_t numSlots, const bq_bvh3f *__restrict__ bvhs,
                                 const uint32_t *__restrict__ off, uint32_t numSegs, uint32_t *__restrict__ parent,
                                 uint32_t *__restrict__ counter)
{
  griddep_wait();
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= numSlots) return;
  counter[j] = 0;
  uint32_t s, local;
  if (!node_slot(bvhs, off, numSegs, j, s, local)) return;
  const uint32_t base = 2 * off[s];
  if (local == 0) parent[j] = BR_NO_PARENT;
  if (local == 1) return;
  const uint64_t a = node_admin(nodes[j]);
  if (admin_count(a) == 0) {
    const uint64_t c = base + admin_offset(a);
    parent[c] = j;
    parent[c + 1] = j;
  }
}

__global__ void k_brefit_climb(Node *nodes, uint32_t numSlots, const bq_bvh3f *__restrict__ bvhs,
                               const uint32_t *__restrict__ off, uint32_t numSegs, const uint32_t *__restrict__ primIDs,
                               const bq_box3f *__restrict__ boxes, const uint32_t *__restrict__ parent,
                               uint32_t *counter)
{
  griddep_wait();
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= numSlots) return;
  uint32_t s, local;
  if (!node_slot(bvhs, off, numSegs, j, s, local) || local == 1) return;
  const uint64_t a = node_admin(nodes[j]);
  const uint32_t cnt = admin_count(a);
  if (cnt == 0) return;
  const uint32_t pbase = off[s], base = 2 * pbase;
  const uint64_t o = admin_offset(a);
  float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
  for (uint32_t q = 0; q < cnt; q++) {
    const bq_box3f b = boxes[pbase + primIDs[pbase + o + q]];
    lx = fminf(lx, b.lower[0]); ly = fminf(ly, b.lower[1]); lz = fminf(lz, b.lower[2]);
    hx = fmaxf(hx, b.upper[0]); hy = fmaxf(hy, b.upper[1]); hz = fmaxf(hz, b.upper[2]);
  }
  nodes[j] = make_node(lx, ly, lz, hx, hy, hz, a);
  while (true) {
    const uint32_t p = parent[j];
    if (p == BR_NO_PARENT) return;
    // device-scope release of this node's box / acquire of the sibling's
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrived(counter[p]);
    if (arrived.fetch_add(1u, cuda::memory_order_acq_rel) == 0) return;  // the sibling finishes this parent
    const float4 pb = __ldcg(&nodes[p].b);  // from L2: the box half of this word is being written
    const uint64_t pa = ((uint64_t)__float_as_uint(pb.w) << 32) | __float_as_uint(pb.z);
    const uint64_t c0 = base + admin_offset(pa);
    const Node sib = ldcg_node(nodes + (c0 == j ? c0 + 1 : c0));
    if (c0 == j) {  // union in child order (left, right)
      lx = fminf(lx, sib.a.x); ly = fminf(ly, sib.a.y); lz = fminf(lz, sib.a.z);
      hx = fmaxf(hx, sib.a.w); hy = fmaxf(hy, sib.b.x); hz = fmaxf(hz, sib.b.y);
    } else {
      lx = fminf(sib.a.x, lx); ly = fminf(sib.a.y, ly); lz = fminf(sib.a.z, lz);
      hx = fmaxf(sib.a.w, hx); hy = fmaxf(sib.b.x, hy); hz = fmaxf(sib.b.y, hz);
    }
    nodes[p] = make_node(lx, ly, lz, hx, hy, hz, pa);
    j = p;
  }
}

// ------------------------------------------------------------------
// batched closest triangle
// ------------------------------------------------------------------
struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float v3dot(V3 a, V3 b)
{
  float r = 0.f;
  r += a.x * b.x;
  r += a.y * b.y;
  r += a.z * b.z;
  return r;
}
__device__ __forceinline__ V3 v3cross(V3 a, V3 b)
{
  return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ V3 ldv(const float *verts, int32_t i)
{
  const float *p = verts + 3ll * i;
  return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// the per-triangle test of bq_tri.cu (cuBQL/queries/triangles/findClosest.h:74-122)
__device__ __forceinline__ void edge_cp(float &best, V3 &P, V3 a, V3 b, V3 p)
{
  const V3 ba = v3sub(b, a);
  float t = v3dot(v3sub(p, a), ba) / v3dot(ba, ba);
  t = fminf(fmaxf(t, 0.f), 1.f);
  const V3 cp = V3{a.x + t * ba.x, a.y + t * ba.y, a.z + t * ba.z};
  const V3 dv = v3sub(cp, p);
  const float sd = v3dot(dv, dv);
  if (sd >= best) return;
  best = sd;
  P = cp;
}

__device__ __forceinline__ float tri_cp(V3 a, V3 b, V3 c, V3 qp, V3 &P)
{
  float best = INFINITY;
  V3 N = v3cross(v3sub(b, a), v3sub(c, a));
  const bool outside = (N.x == 0.f && N.y == 0.f && N.z == 0.f) ||
                       (v3dot(v3sub(qp, a), v3cross(v3sub(b, a), N)) >= 0.f) ||
                       (v3dot(v3sub(qp, b), v3cross(v3sub(c, b), N)) >= 0.f) ||
                       (v3dot(v3sub(qp, c), v3cross(v3sub(a, c), N)) >= 0.f);
  if (outside) {
    edge_cp(best, P, a, b, qp);
    edge_cp(best, P, b, c, qp);
    edge_cp(best, P, c, a, qp);
    return best;
  }
  const float inv = 1.f / sqrtf(v3dot(N, N));
  N = V3{N.x * inv, N.y * inv, N.z * inv};
  const float sd = v3dot(v3sub(qp, a), N);
  P = V3{qp.x - sd * N.x, qp.y - sd * N.y, qp.z - sd * N.z};
  return sd * sd;
}

template <int TIE>
struct BTriLeaf {
  const uint32_t *__restrict__ primIDs;  // mesh-local triangle ids
  const int32_t *__restrict__ tris;      // this mesh's first triangle
  const float *__restrict__ verts;
  V3 q;
  float best;
  int32_t id;
  V3 P;
  __device__ __forceinline__ float operator()(uint64_t o, uint32_t cnt)
  {
    for (uint32_t j = 0; j < cnt; j++) {
      const uint32_t pid = __ldg(primIDs + o + j);
      const int32_t *t = tris + 3ull * pid;
      V3 p;
      const float d = tri_cp(ldv(verts, __ldg(t)), ldv(verts, __ldg(t + 1)), ldv(verts, __ldg(t + 2)), q, p);
      const bool take = (TIE == TIE_REFERENCE) ? (d < best)
                                               : (d < best || (d == best && id >= 0 && (int32_t)pid < id));
      if (take) {
        best = d;
        id = (int32_t)pid;
        P = p;
      }
    }
    return best;
  }
};

template <int TIE, typename Stack>
__device__ __forceinline__ bool run_btri(const bq_bvh3f &d, const uint32_t triBase, const int32_t *tris,
                                         const float *verts, const float *queries, uint32_t qi, float maxSqr,
                                         Stack &st, int32_t *outIds, float *outD, float *outP)
{
  const float *qp = queries + 3ull * qi;
  BTriLeaf<TIE> leaf{d.primIDs, tris + 3ull * triBase, verts, V3{__ldg(qp), __ldg(qp + 1), __ldg(qp + 2)}, maxSqr,
                     -1, V3{0.f, 0.f, 0.f}};
  if (d.numNodes && !traverse<TIE>((const Node *)d.nodes, leaf.q.x, leaf.q.y, leaf.q.z, maxSqr, st, leaf))
    return false;
  outIds[qi] = leaf.id >= 0 ? (int32_t)(triBase + leaf.id) : -1;
  outD[qi] = leaf.id >= 0 ? leaf.best : INFINITY;
  if (outP) {
    outP[3ull * qi] = leaf.P.x;
    outP[3ull * qi + 1] = leaf.P.y;
    outP[3ull * qi + 2] = leaf.P.z;
  }
  return true;
}

template <int TIE, int STACK>
__global__ void __launch_bounds__(128) k_btri(const bq_bvh3f *__restrict__ bvhs, const uint32_t *__restrict__ triOff,
                                              const uint32_t *__restrict__ qoff, uint32_t numSegs,
                                              const int32_t *__restrict__ tris, const float *__restrict__ verts,
                                              const float *__restrict__ queries, uint32_t nq, float maxSqr,
                                              int32_t *__restrict__ outIds, float *__restrict__ outD,
                                              float *__restrict__ outP, uint32_t *__restrict__ ovfList,
                                              uint32_t *ovfCount)
{
  griddep_wait();
  const uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  const uint32_t s = seg_find(qoff, numSegs, qi);
  const bq_bvh3f d = bvhs[s];
  LocalStack<STACK> st;
  if (!run_btri<TIE>(d, __ldg(triOff + s), tris, verts, queries, qi, maxSqr, st, outIds, outD, outP))
    ovfList[atomicAdd(ovfCount, 1u)] = qi;
}

template <int TIE>
__global__ void k_btri_deep(const bq_bvh3f *__restrict__ bvhs, const uint32_t *__restrict__ triOff,
                            const uint32_t *__restrict__ qoff, uint32_t numSegs, const int32_t *__restrict__ tris,
                            const float *__restrict__ verts, const float *__restrict__ queries, float maxSqr,
                            int32_t *__restrict__ outIds, float *__restrict__ outD, float *__restrict__ outP,
                            const uint32_t *ovfList, const uint32_t *ovfCount, StackEntry *stacks, uint32_t *err)
{
  griddep_wait();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t cnt = *ovfCount;
  for (uint32_t w = tid; w < cnt; w += gridDim.x * blockDim.x) {
    const uint32_t qi = ovfList[w];
    const uint32_t s = seg_find(qoff, numSegs, qi);
    GlobalStack st{stacks + (size_t)tid * DEEP_STACK, DEEP_STACK, 0};
    if (!run_btri<TIE>(bvhs[s], triOff[s], tris, verts, queries, qi, maxSqr, st, outIds, outD, outP)) {
      outIds[qi] = -1;
      outD[qi] = INFINITY;
      atomicOr(err, DEV_ERR_STACK);
    }
  }
}

} // namespace

int batched_refit(const bq_bvh3f *bvhs, const uint32_t *off, uint32_t numSegs, uint32_t numPrims, bq_node3f *nodes,
                  const uint32_t *primIDs, const bq_box3f *boxes, Alloc &al)
{
  if (numPrims == 0 || numSegs == 0) return BQ_OK;
  const uint32_t slots = 2 * numPrims;
  TempSet tmp(al);
  uint32_t *parent = nullptr, *counter = nullptr;
  BQ_TRY(tmp.get(&parent, slots));
  BQ_TRY(tmp.get(&counter, slots));
  ProfScope ps("batch.refit", al.s, 2);
  launch_pdl(k_brefit_parents, dim3(div_up(slots, 256)), dim3(256), 0, al.s, (const Node *)nodes, slots, bvhs, off,
             numSegs, parent, counter);
  launch_pdl(k_brefit_climb, dim3(div_up(slots, 128)), dim3(128), 0, al.s, (Node *)nodes, slots, bvhs, off, numSegs,
             primIDs, boxes, parent, counter);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

int batched_tri_closest(const bq_bvh3f *bvhs, const uint32_t *triOff, const int32_t *tris, const float *verts,
                        const float *queries, const uint32_t *qoff, uint32_t numSegs, uint32_t nq, float maxSqr,
                        const bq_query_config *qcfg, int32_t *ids, float *d, float *P, uint32_t *errOut, Alloc &al)
{
  bq_query_config c;
  BQ_TRY(query_config(qcfg, c));
  if (nq == 0 || numSegs == 0) return BQ_OK;
  TempSet tmp(al);
  uint32_t *ovfList = nullptr, *ctl = nullptr;
  StackEntry *deep = nullptr;
  BQ_TRY(tmp.get(&ovfList, nq));
  BQ_TRY(tmp.get(&ctl, 2));
  BQ_TRY(tmp.get(&deep, (size_t)DEEP_THREADS * DEEP_STACK));
  BQ_CUDA(cudaMemsetAsync(ctl, 0, 8, al.s));
  uint32_t *err = errOut ? errOut : ctl + 1;
  const int b = c.blockSize;
  ProfScope ps("batch.tri", al.s, 2);
#define BQ_BTRI(TIE, ST)                                                                                           \
  k_btri<TIE, ST><<<div_up(nq, b), b, 0, al.s>>>(bvhs, triOff, qoff, numSegs, tris, verts, queries, nq, maxSqr, ids, \
                                                 d, P, ovfList, ctl);                                              \
  k_btri_deep<TIE><<<DEEP_THREADS / 128, 128, 0, al.s>>>(bvhs, triOff, qoff, numSegs, tris, verts, queries, maxSqr,  \
                                                         ids, d, P, ovfList, ctl, deep, err)
  if (c.tieMode == BQ_TIES_REFERENCE) {
    if (c.stackDepth == 32) { BQ_BTRI(TIE_REFERENCE, 32); }
    else if (c.stackDepth == 64) { BQ_BTRI(TIE_REFERENCE, 64); }
    else { BQ_BTRI(TIE_REFERENCE, 128); }
  } else {
    if (c.stackDepth == 32) { BQ_BTRI(TIE_LOWEST, 32); }
    else if (c.stackDepth == 64) { BQ_BTRI(TIE_LOWEST, 64); }
    else { BQ_BTRI(TIE_LOWEST, 128); }
  }
#undef BQ_BTRI
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

} // namespace bq
