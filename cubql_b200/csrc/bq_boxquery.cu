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
// One thread per query.  Two ways to the compressed (CSR) result:
//   * k_box_count (how many prims per query), then k_box_fill (their ids at
//     the caller's per-query offsets): two traversals;
//   * k_box_slab keeps the first slabCap prims of every query in a slab row
//     during its one traversal (and lists the queries with more), visiting
//     the queries along a Morton curve of their centres (k_box_query_keys +
//     sort; results stay at each query's own index), then
//     k_box_gather copies the rows to the CSR places and traverses only the
//     listed queries again.  Same result, usually one traversal.  Every stack push is bounded; a query whose traversal
// would need more than BOX_STACK entries is reported with DEV_ERR_STACK
// and its count set to 0 (the reference's fixed 64-entry stack would
// overflow silently).
#include <algorithm>

#include "bq_wide.cuh"

namespace bq {
namespace {

constexpr int BOX_STACK = 128;
constexpr uint32_t BOX_ORDER_MIN = 16384;  // fewer queries are traversed in the given order

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
  griddep_wait();
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
  griddep_wait();
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

// 30-bit Morton code of every query box's centre inside rootBox (lower
// xyz, upper xyz): the visiting order of the queries, so that neighbouring
// threads walk nearly the same nodes.  Results stay at the query's own index.
__global__ void k_box_query_keys(const float *__restrict__ rootBox, const bq_box3f *__restrict__ qb, uint32_t nq,
                                 uint32_t *__restrict__ keys, uint32_t *__restrict__ idx)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const float lx = __ldg(rootBox), ly = __ldg(rootBox + 1), lz = __ldg(rootBox + 2);
  const float ext = fmaxf(fmaxf(__ldg(rootBox + 3) - lx, __ldg(rootBox + 4) - ly), __ldg(rootBox + 5) - lz);
  const float sc = 1024.0f / fmaxf(ext, 1e-20f);
  const bq_box3f b = qb[t];
  // centres outside the root box clamp to its faces (NaN converts to 0)
  const float cx = 0.5f * (b.lower[0] + b.upper[0]), cy = 0.5f * (b.lower[1] + b.upper[1]),
              cz = 0.5f * (b.lower[2] + b.upper[2]);
  const uint32_t ix = min(__float2uint_rz(fmaxf(cx - lx, 0.f) * sc), 1023u);
  const uint32_t iy = min(__float2uint_rz(fmaxf(cy - ly, 0.f) * sc), 1023u);
  const uint32_t iz = min(__float2uint_rz(fmaxf(cz - lz, 0.f) * sc), 1023u);
  keys[t] = spread10(ix) | (spread10(iy) << 1) | (spread10(iz) << 2);
  idx[t] = t;
}

// One traversal that keeps the results: the first slabCap prims of query i
// go to slab[i * slabCap ...], its full count to counts[i]; a query with
// more than slabCap prims is appended to ovf[1..] (ovf[0] counts them) and
// traversed again by k_box_gather.
template <int W>
__global__ void __launch_bounds__(128) k_box_slab(const Node *__restrict__ nodes, const uint32_t *__restrict__ primIDs,
                                                  const bq_box3f *__restrict__ boxes,
                                                  const bq_box3f *__restrict__ queryBoxes, uint32_t nq,
                                                  const uint32_t *__restrict__ order, uint32_t slabCap,
                                                  int32_t *__restrict__ slab, uint32_t *__restrict__ counts,
                                                  uint32_t *__restrict__ ovf, uint32_t *err)
{
  griddep_wait();
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nq) return;
  const uint32_t i = order ? __ldg(order + t) : t;
  float q[6];
  load_query(queryBoxes, i, q);
  int32_t *row = slab + (uint64_t)i * slabCap;
  uint32_t c = 0;
  auto fn = [&](uint32_t pid) {
    if (c < slabCap) row[c] = (int32_t)pid;
    c++;
  };
  if (!any_box_traverse<W>(nodes, primIDs, boxes, q, fn)) {
    c = 0;
    atomicOr(err, DEV_ERR_STACK);
  }
  counts[i] = c;
  if (c > slabCap) ovf[1 + atomicAdd(ovf, 1u)] = i;  // at most nq entries
}

// Results to their CSR places: one warp per query copies its slab row
// (queries of at most slabCap prims); then the listed queries with more are
// traversed again straight into ids (blocks past the copy grid).
template <int W>
__global__ void __launch_bounds__(128) k_box_gather(const Node *__restrict__ nodes,
                                                    const uint32_t *__restrict__ primIDs,
                                                    const bq_box3f *__restrict__ boxes,
                                                    const bq_box3f *__restrict__ queryBoxes, uint32_t nq,
                                                    uint32_t slabCap, const int32_t *__restrict__ slab,
                                                    const uint32_t *__restrict__ counts,
                                                    const uint32_t *__restrict__ ovf,
                                                    const uint32_t *__restrict__ offsets, uint64_t capacity,
                                                    int32_t *__restrict__ ids, uint32_t copyBlocks, uint32_t *err)
{
  griddep_wait();
  if (blockIdx.x < copyBlocks) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)copyBlocks * (blockDim.x / 32);
    for (uint64_t i = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < nq; i += warps) {
      const uint32_t c = counts[i];
      if (c > slabCap) continue;
      const uint64_t at = offsets[i];
      if (at + c > capacity) {
        if (lane == 0) atomicOr(err, DEV_ERR_RANGE);
        continue;
      }
      const int32_t *row = slab + i * slabCap;
      for (uint32_t k = lane; k < c; k += 32) ids[at + k] = row[k];
    }
    return;
  }
  const uint32_t t = (blockIdx.x - copyBlocks) * blockDim.x + threadIdx.x;
  if (t >= ovf[0]) return;
  const uint32_t i = ovf[1 + t];
  float q[6];
  load_query(queryBoxes, i, q);
  uint64_t at = offsets[i];
  const uint64_t end = min(at + counts[i], capacity);
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
    launch_pdl(k_box_count<W>, dim3(div_up(nq, 128)), dim3(128), 0, al.s, nodes, primIDs, boxes, queryBoxes, nq,
               counts, err);
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
    launch_pdl(k_box_fill<W>, dim3(div_up(nq, 128)), dim3(128), 0, al.s, nodes, primIDs, boxes, queryBoxes, nq,
               offsets, capacity, ids, err);
  }
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr & DEV_ERR_RANGE) return set_error(BQ_ERR_INVALID_ARGUMENT, "box query results exceed the given offsets");
  if (herr) return set_error(BQ_ERR_STACK_OVERFLOW, "a box query needed more than 128 traversal stack entries");
  return BQ_OK;
}

// visiting order of nq query boxes along a Morton curve of their centres
// (nullptr: the given order, for few queries)
template <int W>
int box_query_order(const Node *nodes, const bq_box3f *queryBoxes, uint32_t nq, uint32_t *err, TempSet &tmp,
                    Alloc &al, const uint32_t **order)
{
  *order = nullptr;
  if (nq < BOX_ORDER_MIN) return BQ_OK;
  const float *rootBox = (const float *)nodes;  // binary: the root node's box
  if (W != 0) {
    float *rb = nullptr;
    BQ_TRY(tmp.get(&rb, 6));
    launch_pdl(k_wide_root_box<W == 0 ? 2 : W>, dim3(1), dim3(32), 0, al.s, nodes, rb);
    rootBox = rb;
  }
  uint32_t *keys[2], *idx[2];
  BQ_TRY(tmp.get(&keys[0], nq));
  BQ_TRY(tmp.get(&keys[1], nq));
  BQ_TRY(tmp.get(&idx[0], nq));
  BQ_TRY(tmp.get(&idx[1], nq));
  {
    ProfScope ps("boxquery.keys", al.s);
    launch_pdl(k_box_query_keys, dim3(div_up(nq, 256)), dim3(256), 0, al.s, rootBox, queryBoxes, nq, keys[0], idx[0]);
  }
  BQ_CUDA(cudaGetLastError());
  int sel = 0;
  // the order only steers performance: the top 24 key bits (3 passes)
  // suffice; up to 2M queries the top 16 (2 passes) do as well
  const int loBit = nq <= (1u << 21) ? 14 : 6;
  BQ_TRY(onesweep_sort_u32(keys, idx, nq, nullptr, loBit, 30, nullptr, &sel, err, al));
  *order = idx[sel];
  return BQ_OK;
}

template <int W>
int slab_impl(const Node *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_box3f *queryBoxes,
              uint32_t nq, uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *ovf, Alloc &al)
{
  TempSet tmp(al);
  uint32_t *err = nullptr;
  BQ_TRY(tmp.get(&err, 1));
  BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  BQ_CUDA(cudaMemsetAsync(ovf, 0, 4, al.s));
  const uint32_t *order = nullptr;
  BQ_TRY(box_query_order<W>(nodes, queryBoxes, nq, err, tmp, al, &order));
  {
    ProfScope ps("boxquery.slab", al.s);
    launch_pdl(k_box_slab<W>, dim3(div_up(nq, 128)), dim3(128), 0, al.s, nodes, primIDs, boxes, queryBoxes, nq, order,
               slabCap, slab, counts, ovf, err);
  }
  BQ_CUDA(cudaGetLastError());
  uint32_t herr = 0;
  BQ_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (herr & DEV_ERR_TIMEOUT) return set_error(BQ_ERR_TIMEOUT, "box query ordering sort timed out");
  if (herr) return set_error(BQ_ERR_STACK_OVERFLOW, "a box query needed more than 128 traversal stack entries");
  return BQ_OK;
}

template <int W>
int gather_impl(const Node *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                uint32_t nq, uint32_t slabCap, const int32_t *slab, const uint32_t *counts, const uint32_t *ovf,
                const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  TempSet tmp(al);
  uint32_t *err = nullptr;
  BQ_TRY(tmp.get(&err, 1));
  BQ_CUDA(cudaMemsetAsync(err, 0, 4, al.s));
  // queries with more than slabCap prims: at most capacity / (slabCap + 1)
  const uint64_t maxOvf = std::min<uint64_t>(nq, capacity / ((uint64_t)slabCap + 1));
  const uint32_t copyBlocks = (uint32_t)std::max(1, std::min(div_up(nq, 4), num_sms() * 16));
  const uint64_t blocks = copyBlocks + (uint64_t)div_up(maxOvf, 128);
  {
    ProfScope ps("boxquery.gather", al.s);
    launch_pdl(k_box_gather<W>, dim3((unsigned)blocks), dim3(128), 0, al.s, nodes, primIDs, boxes, queryBoxes, nq,
               slabCap, slab, counts, ovf, offsets, capacity, ids, copyBlocks, err);
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

int box_query_slab(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                   uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *ovf, Alloc &al)
{
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    BQ_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, al.s));
    BQ_CUDA(cudaMemsetAsync(ovf, 0, 4, al.s));
    return BQ_OK;
  }
  return slab_impl<0>((const Node *)bvh->nodes, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, al);
}

int box_query_gather(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                     uint32_t slabCap, const int32_t *slab, const uint32_t *counts, const uint32_t *ovf,
                     const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  return gather_impl<0>((const Node *)bvh->nodes, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf,
                        offsets, capacity, ids, al);
}

int wide_box_query_slab(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                        uint32_t nq, uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *ovf, Alloc &al)
{
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nq == 0) return BQ_OK;
  if (bvh->numNodes == 0) {
    BQ_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, al.s));
    BQ_CUDA(cudaMemsetAsync(ovf, 0, 4, al.s));
    return BQ_OK;
  }
  const Node *n = (const Node *)bvh->nodes;
  if (W == 2) return slab_impl<2>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, al);
  if (W == 4) return slab_impl<4>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, al);
  return slab_impl<8>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, al);
}

int wide_box_query_gather(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                          uint32_t nq, uint32_t slabCap, const int32_t *slab, const uint32_t *counts,
                          const uint32_t *ovf, const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al)
{
  if (W != 2 && W != 4 && W != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (nq == 0 || bvh->numNodes == 0) return BQ_OK;
  const Node *n = (const Node *)bvh->nodes;
  if (W == 2)
    return gather_impl<2>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, offsets, capacity, ids, al);
  if (W == 4)
    return gather_impl<4>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, offsets, capacity, ids, al);
  return gather_impl<8>(n, bvh->primIDs, boxes, queryBoxes, nq, slabCap, slab, counts, ovf, offsets, capacity, ids, al);
}

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
