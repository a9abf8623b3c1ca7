// bq_capi.cu -- the extern "C" entry points declared in include/bq.h:
// argument checks, stream/allocator plumbing, dispatch to the kernels.
#include <mutex>

#include "bq_internal.cuh"

namespace bq {
int build_morton63(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int build_rebin_morton30(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int build_spatial_median(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int refit(const bq_bvh3f *bvh, const bq_box3f *boxes, Alloc &al, bool check);
int box_query_count(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                    uint32_t *counts, Alloc &al);
int box_query_fill(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                   const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al);
int wide_box_query_count(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t nq, uint32_t *counts, Alloc &al);
int wide_box_query_fill(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                        uint32_t nq, const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al);
int box_query_slab(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                   uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *ovf, Alloc &al);
int box_query_gather(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t nq,
                     uint32_t slabCap, const int32_t *slab, const uint32_t *counts, const uint32_t *ovf,
                     const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al);
int wide_box_query_slab(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                        uint32_t nq, uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *ovf, Alloc &al);
int wide_box_query_gather(const bq_wide_bvh3f *bvh, int W, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                          uint32_t nq, uint32_t slabCap, const int32_t *slab, const uint32_t *counts,
                          const uint32_t *ovf, const uint32_t *offsets, uint64_t capacity, int32_t *ids, Alloc &al);
int collapse_wide(const bq_bvh3f *bin, int W, bq_wide_bvh3f *out, bool copyPrims, Alloc &al);
int build_sah(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int build_elh(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int build_wide(bq_wide_bvh3f *out, int W, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int wide_closest_point(const bq_wide_bvh3f *bvh, int W, const float *points, const float *queries, uint32_t nq,
                       float maxSqr, const bq_query_config *qcfg, int32_t *ids, float *d, Alloc &al);
int closest_point(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, float maxSqr,
                  const bq_query_config *qcfg, int32_t *ids, float *d, Alloc &al,
                  const int32_t *excludeIds = nullptr, int excludeSelf = 0);
int knn(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k, float maxSqr,
        const bq_query_config *qcfg, int32_t *ids, float *d, int32_t *numFound, Alloc &al);
int tri_closest(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries, uint32_t nq,
                float maxSqr, const bq_query_config *qcfg, int32_t *ids, float *d, float *P, Alloc &al);
int query_visit_counts(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k,
                       float maxSqr, const bq_query_config *qcfg, uint64_t *hostCounts, Alloc &al);
int tri_visit_counts(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries, uint32_t nq,
                     float maxSqr, const bq_query_config *qcfg, uint64_t *hostCounts, Alloc &al);
int tri_distance_bwd(const int32_t *tris, const float *verts, uint32_t numVerts, const float *queries, uint32_t nq,
                     const int32_t *ids, const float *gradSqr, float *gradQ, float *gradV, Alloc &al);
int tri_boxes(const int32_t *tris, const float *verts, uint32_t nt, bq_box3f *boxes, cudaStream_t s);
int points_to_boxes(const float *points, uint32_t n, bq_box3f *boxes, cudaStream_t s);
int batched_build_morton63(const bq_box3f *boxes, const uint32_t *off, uint32_t numSegs, uint32_t n,
                           const bq_build_config *cfg, bq_node3f *nodesOut, uint32_t *primIDs, bq_bvh3f *bvhs,
                           uint32_t *errOut, Alloc &al);
int batched_knn(const bq_bvh3f *bvhs, const uint32_t *poff, const float *points, const float *queries,
                const uint32_t *qoff, uint32_t numSegs, uint32_t nq, int k, float maxSqr, const bq_query_config *qcfg,
                int32_t *ids, float *d, int32_t *nf, uint32_t *errOut, Alloc &al);
int batched_refit(const bq_bvh3f *bvhs, const uint32_t *off, uint32_t numSegs, uint32_t numPrims, bq_node3f *nodes,
                  const uint32_t *primIDs, const bq_box3f *boxes, Alloc &al);
int batched_tri_closest(const bq_bvh3f *bvhs, const uint32_t *triOff, const int32_t *tris, const float *verts,
                        const float *queries, const uint32_t *qoff, uint32_t numSegs, uint32_t nq, float maxSqr,
                        const bq_query_config *qcfg, int32_t *ids, float *d, float *P, uint32_t *errOut, Alloc &al);
int autotune_query(const bq_box3f *boxes, const float *points, uint32_t n, const float *queries, uint32_t nq, int k,
                   bq_tuning *best, Alloc &al);
int autotune_batched_knn(const bq_box3f *boxes, const float *points, const uint32_t *off, uint32_t numSegs,
                         uint32_t n, const float *queries, const uint32_t *qoff, uint32_t nq, int k, bq_tuning *best,
                         Alloc &al);

namespace {
// Like the reference's AsyncGpuMemoryResource (cuBQL/builder/cuda.h:52-72):
// keep freed stream-ordered memory in the device's default pool instead
// of returning it to the driver at every synchronisation.
void keep_pool_memory()
{
  static std::mutex m;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> g(m);
  if (done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[dev] = true;
}

Alloc make_alloc(const bq_allocator *a, bq_stream_t s)
{
  if (!a || !a->malloc || a->scratchFromPool) keep_pool_memory();
  Alloc al;
  al.a = (a && a->malloc && a->free) ? a : nullptr;
  al.s = (cudaStream_t)s;
  return al;
}

bool misaligned(const void *p, size_t a) { return ((uintptr_t)p) % a != 0; }

int check_tree(const bq_bvh3f *bvh)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  if (bvh->numNodes && (!bvh->nodes || !bvh->primIDs))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh has nodes but NULL arrays");
  if (bvh->numNodes && misaligned(bvh->nodes, 16))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh->nodes must be 16-byte aligned");
  return BQ_OK;
}

int check_wide(const bq_wide_bvh3f *bvh, int width)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  if (width != 2 && width != 4 && width != 8) return set_error(BQ_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  if (bvh->numNodes && (!bvh->nodes || !bvh->primIDs))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh has nodes but NULL arrays");
  if (bvh->numNodes && misaligned(bvh->nodes, 16))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh->nodes must be 16-byte aligned");
  return BQ_OK;
}

int check_build(const bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  if (n && !boxes) return set_error(BQ_ERR_INVALID_ARGUMENT, "boxes is NULL");
  if (n && misaligned(boxes, 8)) return set_error(BQ_ERR_INVALID_ARGUMENT, "boxes must be 8-byte aligned");
  if (n >= (1u << 30)) return set_error(BQ_ERR_INVALID_ARGUMENT, "at most 2^30-1 primitives per build");
  return BQ_OK;
}
} // namespace
} // namespace bq

using namespace bq;

extern "C" {

int bq_build_morton63_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                         const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_build(bvh, boxes, numPrims));
  Alloc al = make_alloc(alloc, stream);
  return build_morton63(bvh, boxes, numPrims, cfg, al);
}

int bq_build_rebin_morton30_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                               const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_build(bvh, boxes, numPrims));
  Alloc al = make_alloc(alloc, stream);
  return build_rebin_morton30(bvh, boxes, numPrims, cfg, al);
}

int bq_build_spatial_median_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                               const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_build(bvh, boxes, numPrims));
  if (cfg && cfg->buildMethod != BQ_SPATIAL_MEDIAN && cfg->buildMethod != BQ_SAH && cfg->buildMethod != BQ_ELH)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "buildMethod must be BQ_SPATIAL_MEDIAN, BQ_SAH or BQ_ELH");
  Alloc al = make_alloc(alloc, stream);
  if (cfg && cfg->buildMethod == BQ_SAH) return build_sah(bvh, boxes, numPrims, cfg, al);  // gpu_builder.h:41-53
  if (cfg && cfg->buildMethod == BQ_ELH) return build_elh(bvh, boxes, numPrims, cfg, al);  // gpu_builder.h:54-59
  return build_spatial_median(bvh, boxes, numPrims, cfg, al);
}

int bq_build_sah_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                    const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_build(bvh, boxes, numPrims));
  Alloc al = make_alloc(alloc, stream);
  return build_sah(bvh, boxes, numPrims, cfg, al);
}

int bq_refit_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (bvh->numNodes && !boxes) return set_error(BQ_ERR_INVALID_ARGUMENT, "boxes is NULL");
  Alloc al = make_alloc(alloc, stream);
  return refit(bvh, boxes, al, true);
}

int bq_free_f3(bq_bvh3f *bvh, const bq_allocator *alloc, bq_stream_t stream)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  Alloc al = make_alloc(alloc, stream);
  int s1 = al.free_bytes(bvh->primIDs);
  int s2 = al.free_bytes(bvh->nodes);
  bvh->primIDs = nullptr;
  bvh->nodes = nullptr;
  bvh->numNodes = 0;
  bvh->numPrims = 0;
  return s1 != BQ_OK ? s1 : s2;
}

int bq_build_wide_f3(bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes, uint32_t numPrims,
                     const bq_build_config *cfg, const bq_allocator *alloc, bq_stream_t stream)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  bq_bvh3f probe{};
  BQ_TRY(check_build(&probe, boxes, numPrims));
  if (cfg && cfg->buildMethod != BQ_SPATIAL_MEDIAN)
    return set_error(BQ_ERR_UNSUPPORTED, "wide trees are built by the spatial-median method (collapse others)");
  Alloc al = make_alloc(alloc, stream);
  return build_wide(bvh, width, boxes, numPrims, cfg, al);
}

int bq_collapse_wide_f3(bq_wide_bvh3f *wide, int width, const bq_bvh3f *binary, const bq_allocator *alloc,
                        bq_stream_t stream)
{
  if (!wide) return set_error(BQ_ERR_INVALID_ARGUMENT, "wide is NULL");
  BQ_TRY(check_tree(binary));
  Alloc al = make_alloc(alloc, stream);
  return collapse_wide(binary, width, wide, true, al);
}

int bq_wide_free_f3(bq_wide_bvh3f *bvh, const bq_allocator *alloc, bq_stream_t stream)
{
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  Alloc al = make_alloc(alloc, stream);
  int s1 = al.free_bytes(bvh->primIDs);
  int s2 = al.free_bytes(bvh->nodes);
  bvh->primIDs = nullptr;
  bvh->nodes = nullptr;
  bvh->numNodes = 0;
  bvh->numPrims = 0;
  return s1 != BQ_OK ? s1 : s2;
}

int bq_wide_closest_point_f3(const bq_wide_bvh3f *bvh, int width, const float *points, const float *queries,
                             uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                             float *sqrDist, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_wide(bvh, width));
  if (numQueries && (!queries || !ids || !sqrDist || (bvh->numNodes && !points)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return wide_closest_point(bvh, width, points, queries, numQueries, maxSqrDist, qcfg, ids, sqrDist, al);
}

int bq_wide_box_query_count_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                               const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t *counts,
                               const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_wide(bvh, width));
  if (numQueries && (!queryBoxes || !counts || (bvh->numNodes && !boxes)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return wide_box_query_count(bvh, width, boxes, queryBoxes, numQueries, counts, al);
}

int bq_wide_box_query_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t numQueries, const uint32_t *offsets, uint64_t capacity, int32_t *ids,
                         const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_wide(bvh, width));
  if (numQueries && (!queryBoxes || !offsets || (bvh->numNodes && !boxes) || (capacity && !ids)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return wide_box_query_fill(bvh, width, boxes, queryBoxes, numQueries, offsets, capacity, ids, al);
}

int bq_wide_box_query_slab_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                              const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t slabCap, int32_t *slab,
                              uint32_t *counts, uint32_t *overflow, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_wide(bvh, width));
  if (numQueries && (!queryBoxes || !counts || !overflow || (slabCap && !slab) || (bvh->numNodes && !boxes)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return wide_box_query_slab(bvh, width, boxes, queryBoxes, numQueries, slabCap, slab, counts, overflow, al);
}

int bq_wide_box_query_gather_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                                const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t slabCap,
                                const int32_t *slab, const uint32_t *counts, const uint32_t *overflow,
                                const uint32_t *offsets, uint64_t capacity, int32_t *ids, const bq_allocator *alloc,
                                bq_stream_t stream)
{
  BQ_TRY(check_wide(bvh, width));
  if (numQueries && (!queryBoxes || !counts || !overflow || !offsets || (slabCap && !slab) ||
                     (bvh->numNodes && !boxes) || (capacity && !ids)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return wide_box_query_gather(bvh, width, boxes, queryBoxes, numQueries, slabCap, slab, counts, overflow, offsets,
                               capacity, ids, al);
}

int bq_closest_point_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                        float maxSqrDist, const bq_query_config *qcfg, int32_t *ids, float *sqrDist,
                        const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queries || !ids || !sqrDist || (bvh->numNodes && !points)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return closest_point(bvh, points, queries, numQueries, maxSqrDist, qcfg, ids, sqrDist, al);
}

int bq_closest_point_exclude_id_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                                   const int32_t *excludeIds, float maxSqrDist, const bq_query_config *qcfg,
                                   int32_t *ids, float *sqrDist, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queries || !ids || !sqrDist || !excludeIds || (bvh->numNodes && !points)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return closest_point(bvh, points, queries, numQueries, maxSqrDist, qcfg, ids, sqrDist, al, excludeIds, 0);
}

int bq_closest_point_exclude_self_f3(const bq_bvh3f *bvh, const float *points, const float *queries,
                                     uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                                     float *sqrDist, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queries || !ids || !sqrDist || (bvh->numNodes && !points)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return closest_point(bvh, points, queries, numQueries, maxSqrDist, qcfg, ids, sqrDist, al, nullptr, 1);
}

int bq_box_query_count_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t numQueries,
                          uint32_t *counts, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queryBoxes || !counts || (bvh->numNodes && !boxes)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return box_query_count(bvh, boxes, queryBoxes, numQueries, counts, al);
}

int bq_box_query_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t numQueries,
                    const uint32_t *offsets, uint64_t capacity, int32_t *ids, const bq_allocator *alloc,
                    bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queryBoxes || !offsets || (bvh->numNodes && !boxes) || (capacity && !ids)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return box_query_fill(bvh, boxes, queryBoxes, numQueries, offsets, capacity, ids, al);
}

int bq_box_query_slab_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t numQueries, uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *overflow,
                         const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queryBoxes || !counts || !overflow || (slabCap && !slab) || (bvh->numNodes && !boxes)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return box_query_slab(bvh, boxes, queryBoxes, numQueries, slabCap, slab, counts, overflow, al);
}

int bq_box_query_gather_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                           uint32_t numQueries, uint32_t slabCap, const int32_t *slab, const uint32_t *counts,
                           const uint32_t *overflow, const uint32_t *offsets, uint64_t capacity, int32_t *ids,
                           const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queryBoxes || !counts || !overflow || !offsets || (slabCap && !slab) ||
                     (bvh->numNodes && !boxes) || (capacity && !ids)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return box_query_gather(bvh, boxes, queryBoxes, numQueries, slabCap, slab, counts, overflow, offsets, capacity, ids,
                          al);
}

int bq_knn_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries, int k,
              float maxSqrDist, const bq_query_config *qcfg, int32_t *ids, float *sqrDist, int32_t *numFound,
              const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queries || !ids || !sqrDist || (bvh->numNodes && !points)))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return knn(bvh, points, queries, numQueries, k, maxSqrDist, qcfg, ids, sqrDist, numFound, al);
}

int bq_tri_closest_f3(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries,
                      uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                      float *sqrDist, float *P, const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (numQueries && (!queries || !ids || !sqrDist || (bvh->numNodes && (!tris || !verts))))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return tri_closest(bvh, tris, verts, queries, numQueries, maxSqrDist, qcfg, ids, sqrDist, P, al);
}

int bq_query_visit_counts_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                             int k, float maxSqrDist, const bq_query_config *qcfg, uint64_t *counts,
                             const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (!counts) return set_error(BQ_ERR_INVALID_ARGUMENT, "counts is NULL");
  if (numQueries && (!queries || (bvh->numNodes && !points))) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return query_visit_counts(bvh, points, queries, numQueries, k, maxSqrDist, qcfg, counts, al);
}

int bq_tri_visit_counts_f3(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries,
                           uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, uint64_t *counts,
                           const bq_allocator *alloc, bq_stream_t stream)
{
  BQ_TRY(check_tree(bvh));
  if (!counts) return set_error(BQ_ERR_INVALID_ARGUMENT, "counts is NULL");
  if (numQueries && (!queries || (bvh->numNodes && (!tris || !verts))))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return tri_visit_counts(bvh, tris, verts, queries, numQueries, maxSqrDist, qcfg, counts, al);
}

int bq_tri_distance_bwd_f3(const int32_t *tris, const float *verts, uint32_t numVerts, const float *queries,
                           uint32_t numQueries, const int32_t *ids, const float *gradSqr, float *gradQueries,
                           float *gradVerts, const bq_allocator *alloc, bq_stream_t stream)
{
  if (numQueries && (!tris || !verts || !queries || !ids || !gradSqr || !gradQueries))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (numVerts && !gradVerts) return set_error(BQ_ERR_INVALID_ARGUMENT, "gradVerts is NULL");
  Alloc al = make_alloc(alloc, stream);
  return tri_distance_bwd(tris, verts, numVerts, queries, numQueries, ids, gradSqr, gradQueries, gradVerts, al);
}

int bq_batched_build_morton63_f3(const bq_box3f *boxes, const uint32_t *segOffsets, uint32_t numSegs,
                                 uint32_t numPrims, const bq_build_config *cfg, bq_node3f *nodes, uint32_t *primIDs,
                                 bq_bvh3f *bvhs, uint32_t *deviceErr, const bq_allocator *alloc, bq_stream_t stream)
{
  if (numSegs && (!segOffsets || !bvhs)) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (numPrims && (!boxes || !nodes || !primIDs)) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (numPrims && misaligned(boxes, 8)) return set_error(BQ_ERR_INVALID_ARGUMENT, "boxes must be 8-byte aligned");
  if (numPrims && misaligned(nodes, 16)) return set_error(BQ_ERR_INVALID_ARGUMENT, "nodes must be 16-byte aligned");
  if (numPrims >= (1u << 30)) return set_error(BQ_ERR_INVALID_ARGUMENT, "at most 2^30-1 primitives per batch");
  Alloc al = make_alloc(alloc, stream);
  return batched_build_morton63(boxes, segOffsets, numSegs, numPrims, cfg, nodes, primIDs, bvhs, deviceErr, al);
}

int bq_batched_knn_f3(const bq_bvh3f *bvhs, const uint32_t *pointOffsets, const float *points, const float *queries,
                      const uint32_t *queryOffsets, uint32_t numSegs, uint32_t numQueries, int k, float maxSqrDist,
                      const bq_query_config *qcfg, int32_t *ids, float *sqrDist, int32_t *numFound,
                      uint32_t *deviceErr, const bq_allocator *alloc, bq_stream_t stream)
{
  if (numQueries && (!bvhs || !pointOffsets || !points || !queries || !queryOffsets || !ids || !sqrDist))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (numQueries >= (1u << 30)) return set_error(BQ_ERR_INVALID_ARGUMENT, "at most 2^30-1 queries per batch");
  Alloc al = make_alloc(alloc, stream);
  return batched_knn(bvhs, pointOffsets, points, queries, queryOffsets, numSegs, numQueries, k, maxSqrDist, qcfg, ids,
                     sqrDist, numFound, deviceErr, al);
}

int bq_batched_refit_f3(const bq_bvh3f *bvhs, const uint32_t *segOffsets, uint32_t numSegs, uint32_t numPrims,
                        bq_node3f *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_allocator *alloc,
                        bq_stream_t stream)
{
  if (numPrims && (!bvhs || !segOffsets || !nodes || !primIDs || !boxes))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  if (numPrims >= (1u << 30)) return set_error(BQ_ERR_INVALID_ARGUMENT, "at most 2^30-1 primitives per batch");
  Alloc al = make_alloc(alloc, stream);
  return batched_refit(bvhs, segOffsets, numSegs, numPrims, nodes, primIDs, boxes, al);
}

int bq_batched_tri_closest_f3(const bq_bvh3f *bvhs, const uint32_t *triOffsets, const int32_t *tris,
                              const float *verts, const float *queries, const uint32_t *queryOffsets,
                              uint32_t numSegs, uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg,
                              int32_t *ids, float *sqrDist, float *P, uint32_t *deviceErr, const bq_allocator *alloc,
                              bq_stream_t stream)
{
  if (numQueries && (!bvhs || !triOffsets || !tris || !verts || !queries || !queryOffsets || !ids || !sqrDist))
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  Alloc al = make_alloc(alloc, stream);
  return batched_tri_closest(bvhs, triOffsets, tris, verts, queries, queryOffsets, numSegs, numQueries, maxSqrDist,
                             qcfg, ids, sqrDist, P, deviceErr, al);
}

int bq_autotune_batched_knn_f3(const bq_box3f *boxes, const float *points, const uint32_t *segOffsets,
                               uint32_t numSegs, uint32_t numPrims, const float *queries, const uint32_t *queryOffsets,
                               uint32_t numQueries, int k, bq_tuning *best, const bq_allocator *alloc,
                               bq_stream_t stream)
{
  if (!boxes || !points || !segOffsets || !queries || !queryOffsets || !best)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL argument");
  Alloc al = make_alloc(alloc, stream);
  return autotune_batched_knn(boxes, points, segOffsets, numSegs, numPrims, queries, queryOffsets, numQueries, k,
                              best, al);
}

int bq_autotune_query_f3(const bq_box3f *boxes, const float *points, uint32_t numPrims, const float *queries,
                         uint32_t numQueries, int k, bq_tuning *best, const bq_allocator *alloc, bq_stream_t stream)
{
  if (!boxes || !points || !queries || !best) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL argument");
  Alloc al = make_alloc(alloc, stream);
  return autotune_query(boxes, points, numPrims, queries, numQueries, k, best, al);
}

int bq_tri_boxes_f3(const int32_t *tris, const float *verts, uint32_t numTris, bq_box3f *boxes, bq_stream_t stream)
{
  if (numTris && (!tris || !verts || !boxes)) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  return tri_boxes(tris, verts, numTris, boxes, (cudaStream_t)stream);
}

int bq_points_to_boxes_f3(const float *points, uint32_t numPoints, bq_box3f *boxes, bq_stream_t stream)
{
  if (numPoints && (!points || !boxes)) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  return points_to_boxes(points, numPoints, boxes, (cudaStream_t)stream);
}

} // extern "C"
