// bq_refit.cu -- bottom-up refit of any BinaryBVH<float,3>.
//
// Replaces gpuBuilder_impl::refit (cuBQL/builder/cuda/sm_builder.h:616-693):
// parent links from the admin words, then one thread per leaf computes its
// box from the prim boxes and climbs; at each parent the first arriving
// child stops and the second merges its own box (kept in registers) with
// its sibling's (a per-node counter, one device-scope acquire/release
// fetch_add per arrival).  min/max are exact, so the boxes equal the
// reference's bit for bit regardless of arrival order.  The admin words are
// never modified, so the same tree can be refitted after every vertex
// update of a fitting loop.
#include <cuda/atomic>

#include "bq_internal.cuh"

namespace bq {
namespace {

constexpr uint32_t NO_PARENT = 0xffffffffu;

__global__ void k_refit_parents(const Node *__restrict__ nodes, uint32_t numNodes, uint32_t *__restrict__ parent,
                                uint32_t *__restrict__ counter)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes) return;
  counter[i] = 0;
  if (i == 0) parent[0] = NO_PARENT;
  if (i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  if (admin_count(a) == 0) {
    const uint64_t off = admin_offset(a);
    if (off + 1 < numNodes) {
      parent[off] = i;
      parent[off + 1] = i;
    }
  }
}

__device__ __forceinline__ void store_bounds(Node *n, float lx, float ly, float lz, float hx, float hy, float hz,
                                             uint64_t admin)
{
  *n = make_node(lx, ly, lz, hx, hy, hz, admin);
}

__global__ void k_refit_climb(Node *nodes, uint32_t numNodes, const uint32_t *__restrict__ primIDs,
                              const bq_box3f *__restrict__ boxes, const uint32_t *__restrict__ parent,
                              uint32_t *counter)
{
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  const uint32_t cnt = admin_count(a);
  if (cnt == 0) return;  // inner node: reached by a climbing leaf thread
  const uint64_t off = admin_offset(a);
  float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
  for (uint32_t j = 0; j < cnt; j++) {
    const bq_box3f b = boxes[primIDs[off + j]];
    lx = fminf(lx, b.lower[0]); ly = fminf(ly, b.lower[1]); lz = fminf(lz, b.lower[2]);
    hx = fmaxf(hx, b.upper[0]); hy = fmaxf(hy, b.upper[1]); hz = fmaxf(hz, b.upper[2]);
  }
  store_bounds(nodes + i, lx, ly, lz, hx, hy, hz, a);
  while (true) {
    const uint32_t p = parent[i];
    if (p == NO_PARENT) return;
    // device-scope release of this node's box / acquire of the sibling's
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrived(counter[p]);
    if (arrived.fetch_add(1u, cuda::memory_order_acq_rel) == 0) return;  // sibling still pending: it carries on
    const float4 pb = __ldcg(&nodes[p].b);  // from L2: the box half of this word is being written
    const uint64_t pa = ((uint64_t)__float_as_uint(pb.w) << 32) | __float_as_uint(pb.z);
    const uint64_t c0 = admin_offset(pa);
    const Node s = ldcg_node(nodes + (c0 == i ? c0 + 1 : c0));  // the sibling's box, from L2
    // union in child order (left, right), as the reference's min/max calls
    if (c0 == i) {
      lx = fminf(lx, s.a.x); ly = fminf(ly, s.a.y); lz = fminf(lz, s.a.z);
      hx = fmaxf(hx, s.a.w); hy = fmaxf(hy, s.b.x); hz = fmaxf(hz, s.b.y);
    } else {
      lx = fminf(s.a.x, lx); ly = fminf(s.a.y, ly); lz = fminf(s.a.z, lz);
      hx = fmaxf(s.a.w, hx); hy = fmaxf(s.b.x, hy); hz = fmaxf(s.b.y, hz);
    }
    store_bounds(nodes + p, lx, ly, lz, hx, hy, hz, pa);
    i = p;
  }
}

} // namespace

int refit(const bq_bvh3f *bvh, const bq_box3f *boxes, Alloc &al)
{
  const uint32_t nn = bvh->numNodes;
  if (nn == 0) return BQ_OK;
  TempSet tmp(al);
  uint32_t *parent = nullptr, *counter = nullptr;
  BQ_TRY(tmp.get(&parent, nn));
  BQ_TRY(tmp.get(&counter, nn));
  Node *nodes = (Node *)bvh->nodes;
  ProfScope ps("refit", al.s, 2);
  k_refit_parents<<<div_up(nn, 256), 256, 0, al.s>>>(nodes, nn, parent, counter);
  k_refit_climb<<<div_up(nn, 128), 128, 0, al.s>>>(nodes, nn, bvh->primIDs, boxes, parent, counter);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

} // namespace bq

// ------------------------------------------------------------------
// helpers: point boxes (box3f().including(p), as the reference's tests
// build them, testing/points/closestPoint.cu:22-29)
// ------------------------------------------------------------------
namespace bq {
namespace {
__global__ void k_points_to_boxes(const float *__restrict__ pts, uint32_t n, bq_box3f *__restrict__ boxes)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = pts[3ull * i], y = pts[3ull * i + 1], z = pts[3ull * i + 2];
  bq_box3f b;
  b.lower[0] = fminf(INFINITY, x); b.lower[1] = fminf(INFINITY, y); b.lower[2] = fminf(INFINITY, z);
  b.upper[0] = fmaxf(-INFINITY, x); b.upper[1] = fmaxf(-INFINITY, y); b.upper[2] = fmaxf(-INFINITY, z);
  boxes[i] = b;
}
} // namespace

int points_to_boxes(const float *points, uint32_t n, bq_box3f *boxes, cudaStream_t s)
{
  if (n == 0) return BQ_OK;
  k_points_to_boxes<<<div_up(n, 256), 256, 0, s>>>(points, n, boxes);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}
} // namespace bq
