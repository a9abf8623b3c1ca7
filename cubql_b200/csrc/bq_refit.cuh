// bq_refit.cuh -- bottom-up refit kernels of any BinaryBVH<float,3>, shared
// by bq_refit_f3 (scratch from the allocator) and bq_refit_noalloc_f3
// (scratch in a fixed device array); each .cu that includes this header
// gets its own copy of the kernels.
//
// Replaces gpuBuilder_impl::refit_init / refit_run
// (cuBQL/builder/cuda/sm_builder.h:616-675): parent links from the admin
// words, then one thread per leaf computes its box from the prim boxes and
// climbs; at each parent the first arriving child stops and the second
// merges its own box (kept in registers) with its sibling's (a per-node
// counter, one device-scope acquire/release fetch_add per arrival).
// min/max are exact, so the boxes equal the reference's bit for bit
// regardless of arrival order.  The admin words are never modified.
//
// The tree may come from the caller, so every index taken from it is
// checked before it is used; a malformed tree sets DEV_ERR_RANGE in *err
// and the offending access is skipped:
//   - an inner node whose children (offset, offset+1) are not in
//     [2, numNodes) (node 0 is the root, node 1 is unused);
//   - a leaf whose prims [offset, offset+count) are not in [0, numPrims);
//   - a climb longer than numNodes steps (a cycle of parent links).
// A node no inner node points at keeps NO_PARENT and ends its climb.
#pragma once

#include <cuda/atomic>

#include "bq_internal.cuh"

namespace bq {
namespace {

constexpr uint32_t RF_NO_PARENT = 0xffffffffu;

// parent[i] = none, counter[i] = 0, *err = 0
__global__ void k_refit_init(uint32_t numNodes, uint32_t *__restrict__ parent, uint32_t *__restrict__ counter,
                             uint32_t *__restrict__ err)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *err = 0;
  if (i >= numNodes) return;
  parent[i] = RF_NO_PARENT;
  counter[i] = 0;
}

__global__ void k_refit_parents(const Node *__restrict__ nodes, uint32_t numNodes, uint32_t *__restrict__ parent,
                                uint32_t *__restrict__ err)
{
  griddep_wait();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  if (admin_count(a) != 0) return;
  const uint64_t off = admin_offset(a);
  if (off < 2 || off + 1 >= numNodes) {
    atomicOr(err, DEV_ERR_RANGE);
    return;
  }
  parent[off] = i;
  parent[off + 1] = i;
}

__global__ void k_refit_climb(Node *nodes, uint32_t numNodes, const uint32_t *__restrict__ primIDs, uint32_t numPrims,
                              const bq_box3f *__restrict__ boxes, const uint32_t *__restrict__ parent,
                              uint32_t *counter, uint32_t *__restrict__ err)
{
  griddep_wait();
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  const uint32_t cnt = admin_count(a);
  if (cnt == 0) return;  // inner node: reached by a climbing leaf thread
  const uint64_t off = admin_offset(a);
  if (off + cnt > numPrims) {
    atomicOr(err, DEV_ERR_RANGE);
    return;
  }
  float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
  for (uint32_t j = 0; j < cnt; j++) {
    const bq_box3f b = boxes[primIDs[off + j]];
    lx = fminf(lx, b.lower[0]); ly = fminf(ly, b.lower[1]); lz = fminf(lz, b.lower[2]);
    hx = fmaxf(hx, b.upper[0]); hy = fmaxf(hy, b.upper[1]); hz = fmaxf(hz, b.upper[2]);
  }
  nodes[i] = make_node(lx, ly, lz, hx, hy, hz, a);
  for (uint32_t steps = 0;; steps++) {
    const uint32_t p = parent[i];  // in [0, numNodes) or none: written by k_refit_parents only
    if (p == RF_NO_PARENT) return;
    if (steps >= numNodes) {  // only a cycle of parent links climbs this far
      atomicOr(err, DEV_ERR_RANGE);
      return;
    }
    // device-scope release of this node's box / acquire of the sibling's
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrived(counter[p]);
    if (arrived.fetch_add(1u, cuda::memory_order_acq_rel) == 0) return;  // sibling still pending: it carries on
    const float4 pb = __ldcg(&nodes[p].b);  // from L2: the box half of this word is being written
    const uint64_t pa = ((uint64_t)__float_as_uint(pb.w) << 32) | __float_as_uint(pb.z);
    const uint64_t c0 = admin_offset(pa);  // p's children were range-checked when p was linked
    const Node s = ldcg_node(nodes + (c0 == i ? c0 + 1 : c0));  // the sibling's box, from L2
    // union in child order (left, right), as the reference's min/max calls
    if (c0 == i) {
      lx = fminf(lx, s.a.x); ly = fminf(ly, s.a.y); lz = fminf(lz, s.a.z);
      hx = fmaxf(hx, s.a.w); hy = fmaxf(hy, s.b.x); hz = fmaxf(hz, s.b.y);
    } else {
      lx = fminf(s.a.x, lx); ly = fminf(s.a.y, ly); lz = fminf(s.a.z, lz);
      hx = fmaxf(s.a.w, hx); hy = fmaxf(s.b.x, hy); hz = fmaxf(s.b.y, hz);
    }
    nodes[p] = make_node(lx, ly, lz, hx, hy, hz, pa);
    i = p;
  }
}

// the three launches of one refit; scratch = parent[numNodes], counter[numNodes]
inline void launch_refit(Node *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                         const bq_box3f *boxes, uint32_t *parent, uint32_t *counter, uint32_t *err, cudaStream_t s)
{
  launch_pdl(k_refit_init, dim3(div_up(numNodes, 256)), dim3(256), 0, s, numNodes, parent, counter, err);
  launch_pdl(k_refit_parents, dim3(div_up(numNodes, 256)), dim3(256), 0, s, nodes, numNodes, parent, err);
  launch_pdl(k_refit_climb, dim3(div_up(numNodes, 128)), dim3(128), 0, s, nodes, numNodes, primIDs, numPrims, boxes,
             parent, counter, err);
}

} // namespace
} // namespace bq
