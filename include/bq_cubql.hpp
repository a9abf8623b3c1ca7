// bq_cubql.hpp -- drop-in C++ front end with cuBQL's own call signatures.
//
// Include this after (or instead of) the cuBQL builder header and call the
// functions in namespace bq_cubql the way cuBQL's are called; the work runs
// in libbq.so (include/bq.h).  The functions are templates over the
// caller's types, so cuBQL's headers are not needed to compile this file,
// but the types must have cuBQL's layout (checked by static_assert):
//
//   BinaryBVH<float,3>   {Node *nodes; uint32 numNodes; uint32 *primIDs;
//                         uint32 numPrims}, Node = 32 bytes   (cuBQL/bvh.h:71-111)
//   box_t<float,3>       24 bytes                              (cuBQL/math/box.h:60-179)
//   BuildConfig          {int maxAllowedLeafSize, makeLeafThreshold, buildMethod}
//                                                              (cuBQL/bvh.h:31-64)
//   GpuMemoryResource    virtual malloc(void**, size_t, cudaStream_t),
//                        virtual free(void*, cudaStream_t)     (cuBQL/builder/cuda.h:31-78)
//
// Error behaviour follows the reference: a failing call reports the
// message and raises SIGINT (cuBQL/math/common.h:134-149) unless
// BQ_CUBQL_THROW is defined, in which case it throws std::runtime_error.
#pragma once

#include <cuda_runtime_api.h>

#include <csignal>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "bq.h"

namespace bq_cubql {

inline void check(int status, const char *what)
{
  if (status == BQ_OK) return;
  std::string msg = std::string(what) + ": " + bq_last_error_string();
#ifdef BQ_CUBQL_THROW
  throw std::runtime_error(msg);
#else
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::raise(SIGINT);
#endif
}

// bq_allocator that forwards to a cuBQL GpuMemoryResource
template <class MemRes>
struct ResourceAdapter {
  static int mallocFn(void *ctx, void **ptr, size_t size, bq_stream_t s)
  {
    return static_cast<MemRes *>(ctx)->malloc(ptr, size, (cudaStream_t)s) == cudaSuccess ? 0 : 1;
  }
  static int freeFn(void *ctx, void *ptr, bq_stream_t s)
  {
    return static_cast<MemRes *>(ctx)->free(ptr, (cudaStream_t)s) == cudaSuccess ? 0 : 1;
  }
  static bq_allocator make(MemRes &m) { return bq_allocator{&m, &mallocFn, &freeFn, 0}; }
};

template <class BVH>
inline bq_bvh3f to_c(const BVH &b)
{
  static_assert(sizeof(typename BVH::Node) == 32, "BinaryBVH<float,3>::Node layout");
  return bq_bvh3f{(bq_node3f *)b.nodes, b.numNodes, b.primIDs, b.numPrims};
}

template <class BVH>
inline void from_c(BVH &b, const bq_bvh3f &c)
{
  b.nodes = (typename BVH::Node *)c.nodes;
  b.numNodes = c.numNodes;
  b.primIDs = c.primIDs;
  b.numPrims = c.numPrims;
}

template <class Cfg>
inline bq_build_config to_c_cfg(const Cfg &c)
{
  return bq_build_config{c.maxAllowedLeafSize, c.makeLeafThreshold, (int)c.buildMethod};
}

/*! cuBQL::gpuBuilder(WideBVH<float,3,W>&) (cuBQL/builder/cuda.h:100-116):
    a binary spatial-median build collapsed into a W-wide tree (W = 4, 8) */
template <template <typename, int, int> class WideBVH, typename T, int D, int W, class Box, class Cfg, class MemRes>
inline void gpuBuilder(WideBVH<T, D, W> &bvh, const Box *boxes, uint32_t numBoxes, Cfg cfg, cudaStream_t s,
                       MemRes &mem)
{
  static_assert(sizeof(Box) == 24, "box_t<float,3> layout");
  static_assert(sizeof(typename WideBVH<T, D, W>::Node) == 32 * W, "WideBVH<float,3,W>::Node layout");
  bq_wide_bvh3f c{};
  bq_build_config cc = to_c_cfg(cfg);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_build_wide_f3(&c, W, (const bq_box3f *)boxes, numBoxes, &cc, &a, s), "gpuBuilder(WideBVH)");
  bvh.nodes = (typename WideBVH<T, D, W>::Node *)c.nodes;
  bvh.numNodes = c.numNodes;
  bvh.primIDs = c.primIDs;
  bvh.numPrims = c.numPrims;
}

/*! cuBQL::gpuBuilder (cuBQL/builder/cuda.h:91-99): spatial median */
template <class BVH, class Box, class Cfg, class MemRes>
inline void gpuBuilder(BVH &bvh, const Box *boxes, uint32_t numBoxes, Cfg cfg, cudaStream_t s, MemRes &mem)
{
  static_assert(sizeof(Box) == 24, "box_t<float,3> layout");
  bq_bvh3f c{};
  bq_build_config cc = to_c_cfg(cfg);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_build_spatial_median_f3(&c, (const bq_box3f *)boxes, numBoxes, &cc, &a, s), "gpuBuilder");
  from_c(bvh, c);
}

namespace cuda {
/*! cuBQL::cuda::radixBuilder (cuBQL/builder/cuda.h:134-140) */
template <class BVH, class Box, class Cfg, class MemRes>
inline void radixBuilder(BVH &bvh, const Box *boxes, uint32_t numPrims, Cfg cfg, cudaStream_t s, MemRes &mem)
{
  static_assert(sizeof(Box) == 24, "box_t<float,3> layout");
  bq_bvh3f c{};
  bq_build_config cc = to_c_cfg(cfg);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_build_morton63_f3(&c, (const bq_box3f *)boxes, numPrims, &cc, &a, s), "radixBuilder");
  from_c(bvh, c);
}

/*! cuBQL::cuda::sahBuilder (cuBQL/builder/cuda.h:118-129): binned SAH */
template <class BVH, class Box, class Cfg, class MemRes>
inline void sahBuilder(BVH &bvh, const Box *boxes, uint32_t numPrims, Cfg cfg, cudaStream_t s, MemRes &mem)
{
  static_assert(sizeof(Box) == 24, "box_t<float,3> layout");
  bq_bvh3f c{};
  bq_build_config cc = to_c_cfg(cfg);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_build_sah_f3(&c, (const bq_box3f *)boxes, numPrims, &cc, &a, s), "sahBuilder");
  from_c(bvh, c);
}

/*! cuBQL::cuda::rebinRadixBuilder (cuBQL/builder/cuda.h:143-154) */
template <class BVH, class Box, class Cfg, class MemRes>
inline void rebinRadixBuilder(BVH &bvh, const Box *boxes, uint32_t numPrims, Cfg cfg, cudaStream_t s, MemRes &mem)
{
  static_assert(sizeof(Box) == 24, "box_t<float,3> layout");
  bq_bvh3f c{};
  bq_build_config cc = to_c_cfg(cfg);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_build_rebin_morton30_f3(&c, (const bq_box3f *)boxes, numPrims, &cc, &a, s), "rebinRadixBuilder");
  from_c(bvh, c);
}

/*! cuBQL::cuda::free (cuBQL/builder/cuda.h:158-161) */
template <class BVH, class MemRes>
inline void free(BVH &bvh, cudaStream_t s, MemRes &mem)
{
  bq_bvh3f c = to_c(bvh);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_free_f3(&c, &a, s), "free");
  cudaStreamSynchronize(s);  // cuda::free synchronises (gpu_builder.h:86)
  from_c(bvh, c);
}

/*! cuBQL::cuda::free(WideBVH&) (cuBQL/builder/cuda/wide_gpu_builder.h:217-231) */
template <template <typename, int, int> class WideBVH, typename T, int D, int W, class MemRes>
inline void free(WideBVH<T, D, W> &bvh, cudaStream_t s, MemRes &mem)
{
  bq_wide_bvh3f c{(bq_wide_child3f *)bvh.nodes, bvh.numNodes, bvh.primIDs, bvh.numPrims};
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_wide_free_f3(&c, &a, s), "free(WideBVH)");
  cudaStreamSynchronize(s);
  bvh.nodes = nullptr;
  bvh.numNodes = 0;
  bvh.primIDs = nullptr;
  bvh.numPrims = 0;
}
} // namespace cuda

/*! gpuBuilder_impl::refit (cuBQL/builder/cuda/sm_builder.h:677-693) */
template <class BVH, class Box, class MemRes>
inline void refit(BVH &bvh, const Box *boxes, cudaStream_t s, MemRes &mem)
{
  bq_bvh3f c = to_c(bvh);
  bq_allocator a = ResourceAdapter<MemRes>::make(mem);
  check(bq_refit_f3(&c, (const bq_box3f *)boxes, &a, s), "refit");
}

namespace points {
/*! batched cuBQL::points::findClosest: one call for all queries; ids -1
    where nothing is strictly closer than maxSqrDist.  Ties go to the
    lowest primID unless tieMode is BQ_TIES_REFERENCE. */
template <class BVH, class Vec>
inline void findClosest(const BVH &bvh, const Vec *points, const Vec *queries, uint32_t numQueries, int32_t *ids,
                        float *sqrDist, float maxSqrDist = INFINITY, cudaStream_t s = 0,
                        int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_bvh3f c = to_c(bvh);
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_closest_point_f3(&c, (const float *)points, (const float *)queries, numQueries, maxSqrDist, &q, ids,
                            sqrDist, nullptr, s),
        "findClosest");
}

/*! batched cuBQL::points::findClosest(WideBVH<float,3,W>) (findClosest.h:363-386) */
template <template <typename, int, int> class WideBVH, typename T, int D, int W, class Vec>
inline void findClosest(const WideBVH<T, D, W> &bvh, const Vec *points, const Vec *queries, uint32_t numQueries,
                        int32_t *ids, float *sqrDist, float maxSqrDist = INFINITY, cudaStream_t s = 0,
                        int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_wide_bvh3f c{(bq_wide_child3f *)bvh.nodes, bvh.numNodes, bvh.primIDs, bvh.numPrims};
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_wide_closest_point_f3(&c, W, (const float *)points, (const float *)queries, numQueries, maxSqrDist, &q,
                                 ids, sqrDist, nullptr, s),
        "findClosest(WideBVH)");
}

/*! batched cuBQL::points::findKNN; ids/sqrDist are numQueries*k */
template <class BVH, class Vec>
inline void findKNN(const BVH &bvh, const Vec *points, const Vec *queries, uint32_t numQueries, int k, int32_t *ids,
                    float *sqrDist, int32_t *numFound, float maxSqrDist = INFINITY, cudaStream_t s = 0,
                    int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_bvh3f c = to_c(bvh);
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_knn_f3(&c, (const float *)points, (const float *)queries, numQueries, k, maxSqrDist, &q, ids, sqrDist,
                  numFound, nullptr, s),
        "findKNN");
}

/*! batched cuBQL::points::findClosest_exludeID (findClosest.h:278-305):
    query i never returns prim excludeIds[i] (-1: nothing excluded) */
template <class BVH, class Vec>
inline void findClosest_exludeID(const BVH &bvh, const Vec *points, const Vec *queries, uint32_t numQueries,
                                 const int32_t *excludeIds, int32_t *ids, float *sqrDist,
                                 float maxSqrDist = INFINITY, cudaStream_t s = 0, int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_bvh3f c = to_c(bvh);
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_closest_point_exclude_id_f3(&c, (const float *)points, (const float *)queries, numQueries, excludeIds,
                                       maxSqrDist, &q, ids, sqrDist, nullptr, s),
        "findClosest_exludeID");
}

/*! batched cuBQL::points::findClosest_exludeSelf (findClosest.h:307-334):
    data points equal to the query point are skipped */
template <class BVH, class Vec>
inline void findClosest_exludeSelf(const BVH &bvh, const Vec *points, const Vec *queries, uint32_t numQueries,
                                   int32_t *ids, float *sqrDist, float maxSqrDist = INFINITY, cudaStream_t s = 0,
                                   int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_bvh3f c = to_c(bvh);
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_closest_point_exclude_self_f3(&c, (const float *)points, (const float *)queries, numQueries, maxSqrDist,
                                         &q, ids, sqrDist, nullptr, s),
        "findClosest_exludeSelf");
}
} // namespace points

namespace triangles {
/*! batched cuBQL::triangles::findClosest (queries/triangles/findClosest.h:132-152)
    over an indexed mesh: tris holds 3 vertex indices per triangle into
    verts (float triples), where the reference's Triangle array holds the
    3 vertices themselves; ids, sqrDist and the closest points P (may be
    NULL) per query, -1 / +inf where nothing is closer than maxSqrDist */
template <class BVH, class Vec>
inline void findClosest(const BVH &bvh, const int32_t *tris, const Vec *verts, const Vec *queries,
                        uint32_t numQueries, int32_t *ids, float *sqrDist, Vec *P = nullptr,
                        float maxSqrDist = INFINITY, cudaStream_t s = 0, int tieMode = BQ_TIES_LOWEST_ID)
{
  static_assert(sizeof(Vec) == 12, "vec3f layout");
  bq_bvh3f c = to_c(bvh);
  bq_query_config q{tieMode, 0, 0, 1, 0};
  check(bq_tri_closest_f3(&c, tris, (const float *)verts, (const float *)queries, numQueries, maxSqrDist, &q, ids,
                          sqrDist, (float *)P, nullptr, s),
        "triangles::findClosest");
}
} // namespace triangles

namespace fixedBoxQuery {
/*! batched cuBQL::fixedBoxQuery::forEachPrim (traversal/fixedBoxQuery.h:139-156)
    with a lambda that keeps prims whose box overlaps the query box.  First
    pass: counts[i] = the number of such prims for queryBoxes[i]. */
template <class BVH, class Box>
inline void countPrims(const BVH &bvh, const Box *boxes, const Box *queryBoxes, uint32_t numQueries,
                       uint32_t *counts, cudaStream_t s = 0)
{
  static_assert(sizeof(Box) == 24, "box3f layout");
  bq_bvh3f c = to_c(bvh);
  check(bq_box_query_count_f3(&c, (const bq_box3f *)boxes, (const bq_box3f *)queryBoxes, numQueries, counts,
                              nullptr, s),
        "fixedBoxQuery::countPrims");
}

/*! second pass: the prims of query i go to ids[offsets[i] ..], in the
    order forEachPrim visits them; offsets is the exclusive prefix sum of
    the counts and `capacity` the length of ids */
template <class BVH, class Box>
inline void findPrims(const BVH &bvh, const Box *boxes, const Box *queryBoxes, uint32_t numQueries,
                      const uint32_t *offsets, uint64_t capacity, int32_t *ids, cudaStream_t s = 0)
{
  static_assert(sizeof(Box) == 24, "box3f layout");
  bq_bvh3f c = to_c(bvh);
  check(bq_box_query_f3(&c, (const bq_box3f *)boxes, (const bq_box3f *)queryBoxes, numQueries, offsets, capacity,
                        ids, nullptr, s),
        "fixedBoxQuery::findPrims");
}
} // namespace fixedBoxQuery

} // namespace bq_cubql
