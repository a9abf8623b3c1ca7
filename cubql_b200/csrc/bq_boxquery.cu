// bq_boxquery.cu -- fixed-box queries: for each query box, the prims whose
// box overlaps it.
//
// The traversal is cuBQL::fixedBoxQuery::forEachLeaf / forEachPrim over a
// BinaryBVH (cuBQL/traversal/fixedBoxQuery.h:74-156): depth first, a node's
// children tested against the query box with box_t::overlaps
// (cuBQL/math/box.h:208-212, closed intervals), the first child entered
// when it overlaps (the second pushed if it overlaps too), leaves visited in
// that order.  The per-prim test the reference leaves to the caller's
// lambda is done here against the prim boxes, so a query reports exactly
// the prims whose boxes overlap its box, in the reference's visiting order.
//
// Over a WideBVH (fixedBoxQuery.h:161-277) the walk is depth first over
// the slots of each wide node in order: a valid slot whose box overlaps is
// entered (an inner slot pushes the resume point, node and next slot) or
// its leaf visited.
//
// One thread per query.  Two passes with the same traversal: k_box_count
// (how many prims per query) and k_box_fill (their ids at the caller's
// per-query offsets).  Every stack push is bounded; a query whose traversal
// would need more than BOX_STACK entries is reported with DEV_ERR_STACK
// and its count set to 0 (the reference's fixed 64-entry stack would
// overflow silently).
#include "bq_wide.cuh"

namespace bq {
namespace {

constexpr int BOX_STACK = 128;

__device__ __forceinline__ bool box_overlaps(const float q[6], float lx, float ly, float lz, float hx, float hy,
                                             float hz)
{
  // !(any(q.upper < b.lower) || any(b.upper < q.lower))
  return !(q[3] < lx || q[4] < ly || q[5] < lz || hx < q[0] || hy < q[1] || hz < q[2]);
}

// Visits the prims of every overlapping leaf whose own box overlaps the
// query box, in fixedBoxQuery order; fn(primID) for each.  Returns false
// when the stack would overflow.
template <typename Fn>
__device__ __forceinline__ bool box_traverse(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                             const bq_box3f *__restrict__ boxes, const float q[6], Fn &fn)
{
  uint64_t stack[BOX_STACK];
  int sp = 0;
  uint64_t admin = node_admin(ldg_node(nodes));
  while (true) {
    bool leaf = true;
    while (admin_count(admin) == 0) {
      const uint64_t off = admin_offset(admin);
      const Node n0 = ldg_node(nodes + off), n1 = ldg_node(nodes + off + 1);
      const bool o0 = box_overlaps(q, n0.a.x, n0.a.y, n0.a.z, n0.a.w, n0.b.x, n0.b.y);
      const bool o1 = box_overlaps(q, n1.a.x, n1.a.y, n1.a.z, n1.a.w, n1.b.x, n1.b.y);
      if (o0) {
        if (o1) {
          if (sp >= BOX_STACK) return false;
          stack[sp++] = node_admin(n1);
        }
        admin = node_admin(n0);
      } else if (o1) {
        admin = node_admin(n1);
      } else {
        leaf = false;
        break;
      }
    }
    if (leaf) {
      const uint64_t off = admin_offset(admin);
      const uint32_t cnt = admin_count(admin);
      for (uint32_t j = 0; j < cnt; j++) {
        const uint32_t pid = __ldg(primIDs + off + j);
        const bq_box3f b = boxes[pid];
        if (box_overlaps(q, b.lower[0], b.lower[1], b.lower[2], b.upper[0], b.upper[1], b.upper[2])) fn(pid);
      }
    }
    if (sp == 0) return true;
    admin = stack[--sp];
  }
}

// fixedBoxQuery::forEachLeaf over a WideBVH (:161-230), same contract as
// box_traverse.  A stack entry is (wide node << 8 | slot to resume at).
template <int W, typename Fn>
__device__ __forceinline__ bool wide_box_traverse(const Node *__restrict__ slots, const uint32_t *__restrict__ primIDs,
                                                  const bq_box3f *__restrict__ boxes, const float q[6], Fn &fn)
{
  uint64_t stack[BOX_STACK];
  int sp = 0;
  uint64_t node = 0;
  uint32_t c = 0;
  while (true) {
    const Node sl = ldg_node(slots + node * W + c);
    const uint64_t word = node_admin(sl);
    if (wslot_valid(word) && box_overlaps(q, sl.a.x, sl.a.y, sl.a.z, sl.a.w, sl.b.x, sl.b.y)) {
      const uint32_t cnt = wslot_count(word);
      if (cnt == 0) {
        if (c + 1 < W) {
          if (sp >= BOX_STACK) return false;
          stack[sp++] = (node << 8) | (c + 1);
        }
        node = wslot_offset(word);
        c = 0;
        continue;
      }
      const uint64_t off = wslot_offset(word);
      for (uint32_t j = 0; j < cnt; j++) {
        const uint32_t pid = __ldg(primIDs + off + j);
        const bq_box3f b = boxes[pid];
        if (box_overlaps(q, b.lower[0], b.lower[1], b.lower[2], b.upper[0], b.upper[1], b.upper[2])) fn(pid);
      }
    }
    if (c + 1 < W) {
      c++;
    } else if (sp > 0) {
      const uint64_t e = stack[--sp];
      node = e >> 8;
      c = (uint32_t)(e & 0xFF);
    } else {
      return true;
    }
  }
}

// W == 0: binary tree, else a W-wide tree
template <int W, typename Fn>
__device__ __forceinline__ bool any_box_traverse(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                 const bq_box3f *__restrict__ boxes, const float q[6], Fn &fn)
{
  if constexpr (W == 0) return box_traverse(nodes, primIDs, boxes, q, fn);
  else return wide_box_traverse<W>(nodes, primIDs, boxes, q, fn);
}

__device__ __forceinline__ void load_query(const bq_box3f *__restrict__ qb, uint32_t i, float q[6])
{
  const bq_box3f b = qb[i];
  q[0] = b.lower[0]; q[1] = b.lower[1]; q[2] = b.lower[2];
  q[3] = b.upper[0]; q[4] = b.upper[1]; q[5] = b.upper[2];
}

template <int W>
__global__ void __launch_bounds__(128) k_box_count(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                   const bq_box3f *__restrict__ boxes,
                                                   const bq_box3f *__restrict__ queryBoxes, uint32_t nq,
                                                   uint32_t *__restrict__ counts, uint32_t *err)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  float q[6];
  load_query(queryBoxes, i, q);
  uint32_t c = 0;
  auto fn = [&](uint32_t) { c++; };
  if (!any_box_traverse<W>(nodes, primIDs, boxes, q, fn)) {
    c = 0;
    atomicOr(err, DEV_ERR_STACK);
  }
  counts[i] = c;
}

template <int W>
__global__ void __launch_bounds__(128) k_box_fill(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                  const bq_box3f *__restrict__ boxes,
                                                  const bq_box3f *__restrict__ queryBoxes, uint32_t nq,
                                                  const uint32_t *__restrict__ offsets, uint64_t capacity,
                                                  int32_t *__restrict__ ids, uint32_t *err)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  float q[6];
  load_query(queryBoxes, i, q);
  uint64_t at = offsets[i];
  // this query's slots, never past the end of ids
  const uint64_t end = min(i + 1 < nq ? (uint64_t)offsets[i + 1] : capacity, capacity);
  bool over = false;
  auto fn = [&](uint32_t pid) {
    if (at < end) ids[at++] = (int32_t)pid;
    else over = true;
  };
  if (!any_box_traverse<W>(nodes, primIDs, boxes, q, fn) || over) atomicOr(err, over ? DEV_ERR_RANGE : DEV_ERR_STACK);
}


template <int W>
int count_impl(const Node *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_box3f *queryBoxes,
               uint32_t nq, uint32_t *counts, Alloc &al)
{
  TempSet tmp(al);
  uint32_t *err = nullptr;
  BQ_TRY(tmp.get(&err, 1));
  BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  {
    ProfScope ps("boxquery.count", al.s);
    k_box_count<W><<<div_up(nq, 128), 128, 0, al.s>>>(nodes, primIDs, boxes, queryBoxes, nq, counts, err);
  }
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr) return set_error(BQ_ERR_STACK_OVERFLOW, "a box query needed more than 128 traversal stack entries");
  return BQ_OK;
}

template <int W>
int fill_impl(const Node *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_box3f *queryBoxes,
              uint32_t nq, const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  TempSet tmp(al);
  uint32_t *err = nullptr;
  BQ_TRY(tmp.get(&err, 1));
  BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  {
    ProfScope ps("boxquery.fill", al.s);
    k_box_fill<W><<<div_up(nq, 128), 128, 0, al.s>>>(nodes, primIDs, boxes, queryBoxes, nq, offsets, capacity, ids,
                                                      err);
  }
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr & DEV_ERR_RANGE) return set_error(BQ_ERR_INVALID_ARGUMENT, "box query results exceed the given offsets");
  if (herr) return set_error(BQ_ERR_STACK_OVERFLOW, "a box query needed more than 128 traversal stack entries");
  return BQ_OK;
}

} // namespace

int box_query_count(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                    uint32_t *counts, Alloc &al)
{
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    BQ_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, al.s));
    return BQ_OK;
  }
  return count_impl<0>((const Node *)bvh->nodes, bvh->primIDs, boxes, queryBoxes, nq, counts, al);
}

int box_query_fill(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                   const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  return fill_impl<0>((const Node *)bvh->nodes, bvh->primIDs, boxes, queryBoxes, nq, offsets, capacity, ids, al);
}

int wide_box_query_count(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t nq, uint32_t *counts, Alloc &al)
{
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    BQ_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, al.s));
    return BQ_OK;
  }
  const Node *n = (const Node *)bvh->nodes;
  if (W == 2) return count_impl<2>(n, bvh->primIDs, boxes, queryBoxes, nq, counts, al);
  if (W == 4) return count_impl<4>(n, bvh->primIDs, boxes, queryBoxes, nq, counts, al);
  return count_impl<8>(n, bvh->primIDs, boxes, queryBoxes, nq, counts, al);
}

int wide_box_query_fill(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                        uint32_t nq, const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  const Node *n = (const Node *)bvh->nodes;
  if (W == 2) return fill_impl<2>(n, bvh->primIDs, boxes, queryBoxes, nq, offsets, capacity, ids, al);
  if (W == 4) return fill_impl<4>(n, bvh->primIDs, boxes, queryBoxes, nq, offsets, capacity, ids, al);
  return fill_impl<8>(n, bvh->primIDs, boxes, queryBoxes, nq, offsets, capacity, ids, al);
}

} // namespace bq
