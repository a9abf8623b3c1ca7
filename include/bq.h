/*
 * bq.h -- C ABI of the B200-native BVH build-and-query library (libbq.so).
 *
 * Drop-in for the BinaryBVH<float,3> build-and-query path of cuBQL
 * (Ssz990220/cuBQL).  Every entry point:
 *   - runs on the caller's CUDA stream (`bq_stream_t` is a cudaStream_t;
 *     NULL is the legacy default stream),
 *   - takes DEVICE pointers for all array arguments,
 *   - returns an int status (BQ_OK or one of the BQ_ERR_* codes below);
 *     bq_last_error_string() gives the message of the calling thread's
 *     last failure.  Nothing aborts or raises.
 * Mutable global state kept between calls:
 *   - the per-thread error string;
 *   - the flag that records that the default stream-ordered pool's
 *     release threshold was raised (set once per device);
 *   - the phase profiler's event pool (bq_profile_*, per thread, only
 *     while profiling is enabled);
 *   - a small pinned host buffer per thread that the builders read their
 *     device-side counters back into (allocated on first use);
 *   - the fixed scratch array of bq_refit_noalloc_f3 (shared by all of
 *     its calls; see there);
 *   - the count of bq_debug_inject_sort_timeout (a test hook, 0 unless a
 *     test sets it).
 * Apart from bq_refit_noalloc_f3, calls on different streams may run
 * concurrently.
 *
 * Memory layout (identical to the reference, so trees built here can be
 * traversed by the reference's device code and vice versa):
 *   bq_box3f   == cuBQL::box3f              (cuBQL/math/box.h:60-179), 24 B
 *   bq_node3f  == BinaryBVH<float,3>::Node  (cuBQL/bvh.h:78-102), 32 B,
 *                 offsetAndCount = offset (bits 0..47) | count (bits 48..63);
 *                 count 0 = inner node whose children are nodes[offset],
 *                 nodes[offset+1]; count > 0 = leaf holding
 *                 primIDs[offset .. offset+count).
 *                 Node 0 is the root, node 1 is unused.
 *   bq_bvh3f   == BinaryBVH<float,3>        (cuBQL/bvh.h:71-111)
 */
#ifndef BQ_H
#define BQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BQ_VERSION 100

/* status codes */
#define BQ_OK 0
#define BQ_ERR_INVALID_ARGUMENT 1 /* bad pointer, size, alignment or config */
#define BQ_ERR_CUDA 2             /* a CUDA runtime call failed */
#define BQ_ERR_ALLOC 3            /* the allocator returned an error */
#define BQ_ERR_STACK_OVERFLOW 4   /* a query exceeded even the deep fallback stack */
#define BQ_ERR_TIMEOUT 5          /* a bounded device-side wait gave up */
#define BQ_ERR_UNSUPPORTED 6

/* build methods (cuBQL/bvh.h:38-55 BuildConfig::BuildMethod) */
#define BQ_SPATIAL_MEDIAN 0
#define BQ_SAH 1 /* binned surface-area heuristic (BuildConfig::SAH) */
#define BQ_ELH 2 /* edge-length heuristic (BuildConfig::ELH) */
#define BQ_MORTON63 16 /* cuda::radixBuilder */
#define BQ_MORTON30 17 /* cuda::rebinRadixBuilder */

/* query tie rules */
#define BQ_TIES_LOWEST_ID 0 /* equal FP32 distances -> lowest primID (default) */
#define BQ_TIES_REFERENCE 1 /* exactly the reference's traversal-order rules */

typedef void *bq_stream_t; /* cudaStream_t */

typedef struct bq_box3f {
  float lower[3];
  float upper[3];
} bq_box3f;

typedef struct bq_node3f {
  float lower[3];
  float upper[3];
  uint64_t offsetAndCount;
} bq_node3f;

typedef struct bq_bvh3f {
  bq_node3f *nodes;
  uint32_t numNodes;
  uint32_t *primIDs;
  uint32_t numPrims;
} bq_bvh3f;

/* mirrors cuBQL::BuildConfig (cuBQL/bvh.h:31-64) */
typedef struct bq_build_config {
  int maxAllowedLeafSize; /* default 1<<15 */
  int makeLeafThreshold;  /* 0 = builder default (1) */
  int buildMethod;        /* BQ_SPATIAL_MEDIAN, BQ_SAH or BQ_ELH (bq_build_spatial_median_f3 only) */
} bq_build_config;

/* replaces cuBQL::GpuMemoryResource (cuBQL/builder/cuda.h:31-78).
   NULL = cudaMallocAsync / cudaFreeAsync on the call's stream.  Frees are
   stream-ordered: free(ctx, ptr, stream) may be called while work queued
   on `stream` still uses ptr, so the memory must not go to other streams
   before that work completes (as with cudaFreeAsync). */
typedef struct bq_allocator {
  void *ctx;
  int (*malloc)(void *ctx, void **ptr, size_t size, bq_stream_t stream); /* 0 on success */
  int (*free)(void *ctx, void *ptr, bq_stream_t stream);
  /* 0 (the default of a zero-initialised struct): every allocation, the
     call's temporaries included, goes through malloc/free, as with the
     reference's GpuMemoryResource.  1: only the arrays handed back (tree
     nodes, primIDs) do; temporaries come from the library's stream-ordered
     pool (cudaMallocAsync), which saves a callback per temporary. */
  int scratchFromPool;
} bq_allocator;

/* traversal knobs; NULL = defaults (ties lowest-ID, Morton-ordered
   queries, autotuned launch shape) */
typedef struct bq_query_config {
  int tieMode;       /* BQ_TIES_LOWEST_ID or BQ_TIES_REFERENCE */
  int stackDepth;    /* fast-path stack entries: 32, 64 or 128 (0 = 64) */
  int blockSize;     /* threads per block: 64..512 (0 = 128) */
  int reorder;       /* 1 = process queries in Morton order, 0 = input order */
  int queriesPerWarp;/* one thread per query; queries a warp takes per work grab in the
                        persistent batched kernel (multiple of 32, <= 1024; 0 = 32) */
  int lanesPerQuery; /* bq_knn_f3 only.  0 or 1: one thread per query, its top-k list in
                        that thread's registers.  4, 8, 16 or 32 (at least k): a group of
                        that many lanes per query walks the tree together and holds the
                        sorted top-k list one candidate per lane; a new candidate is
                        placed by one ballot and moved in by one warp shuffle */
} bq_query_config;

/* ---------------------------------------------------------------- */
/* builders                                                           */
/* ---------------------------------------------------------------- */

/* Morton/radix builder with 63-bit keys.  Replaces
   cuBQL::cuda::radixBuilder<float,3> (cuBQL/builder/cuda.h:134-140,
   implementation cuBQL/builder/cuda/radix.h:591-771).  The tree equals
   the reference's node for node after BFS renumbering.  Empty boxes
   (lower.x > upper.x) are left out.  Allocates bvh->nodes and
   bvh->primIDs with `alloc`.  Synchronises `stream` once, after the
   sort, to learn the valid-prim count, the sort's status and whether
   long runs of equal keys need their extra pass (and once more at the end
   when they do); otherwise the bottom-up agglomeration is still running
   on `stream` when the call returns (stream-ordered, as the reference's
   builder returns before its refit completes). */
int bq_build_morton63_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                         const bq_allocator *alloc, bq_stream_t stream);

/* Rebinning Morton builder with 30-bit keys.  Replaces
   cuBQL::cuda::rebinRadixBuilder<float,3> (cuBQL/builder/cuda.h:143-154,
   implementation cuBQL/builder/cuda/rebinMortonBuilder.h:1161-1488).
   Runs of more than 32 prims with equal keys get new keys over their own
   centroid bounds (stable sort); smaller ones are rebinned with the
   reference's exchange sort.  The tree and prim order equal the
   reference's after BFS renumbering for inputs without empty boxes.
   Where the reference would rebin forever (a run whose centroid bounds
   are narrower than 1e-20 but not a point) the rebin depth stops at 40
   and the run is split by position. */
int bq_build_rebin_morton30_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                               const bq_allocator *alloc, bq_stream_t stream);

/* Replaces cuBQL::gpuBuilder<float,3> (cuBQL/builder/cuda.h:91-99,
   cuBQL/builder/cuda/gpu_builder.h:31-67): cfg->buildMethod
   BQ_SPATIAL_MEDIAN (default) is the spatial-median builder
   (cuBQL/builder/cuda/sm_builder.h:469-614), BQ_SAH the SAH builder
   (as bq_build_sah_f3), BQ_ELH the edge-length-heuristic builder
   (cuBQL/builder/cuda/elh_builder.h:420-556: the SAH builder with 8 bins
   per axis, bins at (c - lo) / (hi - lo) and edge-length sums as the cost
   measure).  Other values give BQ_ERR_INVALID_ARGUMENT. */
int bq_build_spatial_median_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                               const bq_allocator *alloc, bq_stream_t stream);

/* Binned SAH builder.  Replaces cuBQL::cuda::sahBuilder<float,3>
   (cuBQL/builder/cuda.h:118-129, cuBQL/builder/cuda/sah_builder.h:
   320-538): 16 centroid bins per axis, evaluateSAH's leaf-versus-split
   costs with surfaceArea, prims with bin >= the split bin to the right.
   The tree equals the reference's after BFS renumbering; leaves list their
   prims in ascending primID order.  A node the heuristic would make a
   leaf of more than 65535 prims (the reference's 16-bit count wraps) is
   split in halves by position.  makeLeafThreshold 0 and 1 are the same. */
int bq_build_sah_f3(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t numPrims, const bq_build_config *cfg,
                    const bq_allocator *alloc, bq_stream_t stream);

/* Recomputes every node box bottom-up from `boxes`.  Replaces
   gpuBuilder_impl::refit (cuBQL/builder/cuda/sm_builder.h:677-693).
   Every index read from the tree is range-checked on the device: an inner
   node whose children are not in [2, numNodes), a leaf whose prims are not
   in [0, numPrims), or a cycle of parent links gives
   BQ_ERR_INVALID_ARGUMENT (the bad access is skipped, never made).  To
   report that, the call waits for the refit to finish; while the stream is
   being captured into a graph it does not wait and reports nothing.
   primIDs must index `boxes`. */
int bq_refit_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_allocator *alloc, bq_stream_t stream);

/* bq_refit_f3 without any device allocation (no counterpart in the
   reference).  For callers that may not allocate device memory when they
   refit: an application that reserved all GPU memory for its own pool up
   front, a real-time loop where cudaMalloc could stall or fail mid-frame,
   or a framework that only permits allocation during its set-up.  Its
   scratch (two words per node) is one fixed array inside the library,
   sized for BQ_NOALLOC_REFIT_MAX_NODES nodes (8 MiB); larger trees are
   rejected with BQ_ERR_INVALID_ARGUMENT.
   Set-up: call it once per device, with that device current and
   numNodes == 0 (the other fields are not read), during set-up, before
   any stream capture and before reserving the rest of the GPU's memory.
   That call places the array on the device (with the CUDA runtime's
   default lazy module loading nothing is placed before) and loads the
   kernels; the device then holds the 8 MiB until the process exits.
   All calls share the array and each call clears what it needs: calls
   that overlap on the GPU race, so serialise them.  Like bq_refit_f3 it
   range-checks the tree and waits for the refit to finish. */
#define BQ_NOALLOC_REFIT_MAX_NODES (1u << 20)
int bq_refit_noalloc_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, bq_stream_t stream);

/* Frees a tree built by this library.  Replaces cuBQL::cuda::free
   (cuBQL/builder/cuda.h:158-161, cuBQL/builder/cuda/gpu_builder.h:79-90). */
int bq_free_f3(bq_bvh3f *bvh, const bq_allocator *alloc, bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* wide BVHs: WideBVH<float,3,W> (cuBQL/bvh.h:113-141), W = 4 or 8    */
/* ---------------------------------------------------------------- */
/* One child slot of a wide node (WideBVH::Node::Child, cuBQL/bvh.h:124-131),
   32 B: the child's box, then one 64-bit word with bit 0 = valid,
   bits 1..45 = offset (the wide node id of an inner child, or the first
   primIDs index of a leaf), bits 46..61 = count (0: inner child).  A wide
   node is W consecutive slots; unused slots have valid = 0, an empty box
   (+inf lower, -inf upper), offset 0xFFFFFFFF and count 0xFFFF, as the
   reference writes them.  Node 0 is the root. */
typedef struct bq_wide_child3f {
  float lower[3];
  float upper[3];
  uint64_t validOffsetCount;
} bq_wide_child3f;

/* == WideBVH<float,3,W> (nodes: numNodes * W slots) */
typedef struct bq_wide_bvh3f {
  bq_wide_child3f *nodes;
  uint32_t numNodes;
  uint32_t *primIDs;
  uint32_t numPrims;
} bq_wide_bvh3f;

/* Spatial-median build collapsed into a width-W tree.  Replaces
   cuBQL::gpuBuilder(WideBVH<float,3,W>&, ...) (cuBQL/builder/cuda.h:104-113,
   cuBQL/builder/cuda/wide_gpu_builder.h:162-213): every inner binary node
   at a depth that is a multiple of log2(W) becomes a wide node whose
   slots are the frontier of its treelet, in the reference's slot order.
   Wide nodes are numbered by the index of their binary root (the
   reference numbers them in atomic order, so its numbering varies from
   run to run).  Synchronises the stream. */
int bq_build_wide_f3(bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes, uint32_t numPrims,
                     const bq_build_config *cfg, const bq_allocator *alloc, bq_stream_t stream);

/* Collapses an existing binary tree (any builder) into a width-W tree
   with its own copy of the primIDs; `binary` stays valid.  Synchronises
   the stream. */
int bq_collapse_wide_f3(bq_wide_bvh3f *wide, int width, const bq_bvh3f *binary, const bq_allocator *alloc,
                        bq_stream_t stream);

/* Frees a wide tree.  Replaces cuBQL::cuda::free(WideBVH&)
   (cuBQL/builder/cuda/wide_gpu_builder.h:217-231). */
int bq_wide_free_f3(bq_wide_bvh3f *bvh, const bq_allocator *alloc, bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* queries (batched; the reference offers per-thread device functions */
/* that user kernels call one thread per query)                        */
/* ---------------------------------------------------------------- */

/* Closest data point per query.  Replaces a user kernel calling
   cuBQL::points::findClosest (cuBQL/queries/points/findClosest.h:336-360)
   once per query, e.g. testing/points/closestPoint.cu:37-58.
   ids[q] = closest primID or -1 if none within maxSqrDist (strictly
   closer); sqrDist[q] = its FP32 squared distance or +inf. */
int bq_closest_point_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                        float maxSqrDist, const bq_query_config *qcfg, int32_t *ids, float *sqrDist,
                        const bq_allocator *alloc, bq_stream_t stream);

/* Closest data point per query, skipping one prim per query: excludeIds
   (device array of numQueries ints) names the prim query q must not return
   (-1: none).  Replaces cuBQL::points::findClosest_exludeID
   (cuBQL/queries/points/findClosest.h:278-305) in a user kernel; the
   typical use is "nearest other point" with the data points as queries. */
int bq_closest_point_exclude_id_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                                   const int32_t *excludeIds, float maxSqrDist, const bq_query_config *qcfg,
                                   int32_t *ids, float *sqrDist, const bq_allocator *alloc, bq_stream_t stream);

/* Closest data point per query among the points not equal to the query
   (every coordinate equal).  Replaces cuBQL::points::findClosest_exludeSelf
   (cuBQL/queries/points/findClosest.h:307-334) in a user kernel. */
int bq_closest_point_exclude_self_f3(const bq_bvh3f *bvh, const float *points, const float *queries,
                                     uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                                     float *sqrDist, const bq_allocator *alloc, bq_stream_t stream);

/* Fixed-box query, first pass: counts[q] = the number of prims whose box
   (boxes: the boxes the tree was built over) overlaps queryBoxes[q]
   (closed intervals, box_t::overlaps, cuBQL/math/box.h:208-212).  Replaces
   a user kernel calling cuBQL::fixedBoxQuery::forEachPrim
   (cuBQL/traversal/fixedBoxQuery.h:143-156) with a lambda that tests the
   prim's box.  Synchronises the stream (reports a traversal that would
   need more than 128 stack entries as BQ_ERR_STACK_OVERFLOW). */
int bq_box_query_count_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t numQueries,
                          uint32_t *counts, const bq_allocator *alloc, bq_stream_t stream);

/* Fixed-box query, second pass: the ids of query q go to
   ids[offsets[q] .. offsets[q+1]) (offsets: the exclusive prefix sum of the
   first pass's counts; the last query ends at `capacity`, the length of
   ids), in the reference's visiting order (forEachLeaf, depth first, first
   child first).  Synchronises the stream. */
int bq_box_query_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes, uint32_t numQueries,
                    const uint32_t *offsets, uint64_t capacity, int32_t *ids, const bq_allocator *alloc,
                    bq_stream_t stream);

/* Fixed-box query in one traversal (same results as the two calls above):
   the first slabCap ids of query q go to slab[q*slabCap ..], all its count
   to counts[q]; the queries with more than slabCap prims are listed in
   overflow[1 ..] (overflow[0] = how many; the array holds numQueries + 1
   entries).  Synchronises the stream. */
int bq_box_query_slab_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t numQueries, uint32_t slabCap, int32_t *slab, uint32_t *counts, uint32_t *overflow,
                         const bq_allocator *alloc, bq_stream_t stream);

/* Second step of the one-traversal query: the ids of query q go to
   ids[offsets[q] .. offsets[q] + counts[q]) (offsets: the exclusive prefix
   sum of counts; capacity: the length of ids) -- copied from its slab row,
   or, for the listed queries, by traversing again.  Synchronises the
   stream. */
int bq_box_query_gather_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                           uint32_t numQueries, uint32_t slabCap, const int32_t *slab, const uint32_t *counts,
                           const uint32_t *overflow, const uint32_t *offsets, uint64_t capacity, int32_t *ids,
                           const bq_allocator *alloc, bq_stream_t stream);

/* Closest data point per query over a wide tree.  Replaces a user kernel
   calling cuBQL::points::findClosest(WideBVH<float,3,W>, ...)
   (cuBQL/queries/points/findClosest.h:365-386, traversal
   cuBQL/traversal/shrinkingRadiusQuery.h:553-636).  Same contract as
   bq_closest_point_f3; with BQ_TIES_REFERENCE the answer equals the
   reference's on the same wide tree (same slot sort, same numbering). */
int bq_wide_closest_point_f3(const bq_wide_bvh3f *bvh, int width, const float *points, const float *queries,
                             uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                             float *sqrDist, const bq_allocator *alloc, bq_stream_t stream);

/* Fixed-box query over a wide tree (cuBQL::fixedBoxQuery::forEachPrim for
   WideBVH, cuBQL/traversal/fixedBoxQuery.h:161-277: depth first, slots
   in order), two passes as bq_box_query_count_f3 / bq_box_query_f3. */
int bq_wide_box_query_count_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                               const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t *counts,
                               const bq_allocator *alloc, bq_stream_t stream);
int bq_wide_box_query_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes, const bq_box3f *queryBoxes,
                         uint32_t numQueries, const uint32_t *offsets, uint64_t capacity, int32_t *ids,
                         const bq_allocator *alloc, bq_stream_t stream);
/* The one-traversal form over a wide tree: as bq_box_query_slab_f3 /
   bq_box_query_gather_f3. */
int bq_wide_box_query_slab_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                              const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t slabCap, int32_t *slab,
                              uint32_t *counts, uint32_t *overflow, const bq_allocator *alloc, bq_stream_t stream);
int bq_wide_box_query_gather_f3(const bq_wide_bvh3f *bvh, int width, const bq_box3f *boxes,
                                const bq_box3f *queryBoxes, uint32_t numQueries, uint32_t slabCap,
                                const int32_t *slab, const uint32_t *counts, const uint32_t *overflow,
                                const uint32_t *offsets, uint64_t capacity, int32_t *ids, const bq_allocator *alloc,
                                bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* test hook                                                          */
/* ---------------------------------------------------------------- */
/* The next `count` radix sorts (of any call, any thread) start with the
   first pass's first tile holding back its digit totals, so every
   look-back wait on it runs out after a short spin (a few milliseconds)
   instead of the normal limit: the pass aborts, the sort's output is
   overwritten with in-range values (keys 0, values 0..n-1) and the call
   returns BQ_ERR_TIMEOUT.  Exercises the bounded-wait error path without
   any fault; no counterpart in the reference.  0 switches it off. */
int bq_debug_inject_sort_timeout(int count);

/* ---------------------------------------------------------------- */
/* binary-dump files (host only, no GPU)                              */
/* ---------------------------------------------------------------- */
/* The format of cuBQL::samples::loadBinary / saveBinary
   (samples/common/IO.h:27-58): an 8-byte element count N, then N raw
   elements of itemBytes each.  With out == NULL only *count is set;
   otherwise N must not exceed capacity (elements). */
int bq_load_binary(const char *path, size_t itemBytes, void *out, uint64_t capacity, uint64_t *count);
int bq_save_binary(const char *path, const void *data, uint64_t count, size_t itemBytes);

/* A file of vec_t<double,dims> points (what the reference's point
   generator writes) loaded as float points: loadBinary followed by
   convert<float,dims> (samples/common/IO.h:60-68), each coordinate
   rounded to the nearest float.  out holds capacity*dims floats. */
int bq_load_points_f64_as_f32(const char *path, int dims, float *out, uint64_t capacity, uint64_t *count);

/* k nearest data points per query (1 <= k <= 64), ascending by squared
   distance.  Replaces cuBQL::points::findKNN
   (cuBQL/queries/points/knn.h:75-116).  ids/sqrDist are numQueries*k
   (row per query; unfilled slots -1 / +inf); numFound may be NULL. */
int bq_knn_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries, int k,
              float maxSqrDist, const bq_query_config *qcfg, int32_t *ids, float *sqrDist, int32_t *numFound,
              const bq_allocator *alloc, bq_stream_t stream);

/* Closest triangle per query over an indexed mesh (tris: int32 triples
   into verts: float triples).  Replaces cuBQL::triangles::findClosest
   (cuBQL/queries/triangles/findClosest.h:132-152).  P may be NULL. */
int bq_tri_closest_f3(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries,
                      uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, int32_t *ids,
                      float *sqrDist, float *P, const bq_allocator *alloc, bq_stream_t stream);

/* Adjoint of bq_tri_closest_f3's sqrDist: given gradSqr (dL/dsqrDist per
   query) and the forward's ids, writes gradQueries (numQueries*3) and
   OVERWRITES gradVerts (numVerts*3).  Vertex contributions are sorted by
   vertex id and summed in a fixed order: no float atomics, bitwise
   reproducible.  No counterpart in the reference (it has no gradients). */
int bq_tri_distance_bwd_f3(const int32_t *tris, const float *verts, uint32_t numVerts, const float *queries,
                           uint32_t numQueries, const int32_t *ids, const float *gradSqr, float *gradQueries,
                           float *gradVerts, const bq_allocator *alloc, bq_stream_t stream);

/* Traversal visit counts of a query batch, the measurement behind the
   query rooflines.  Replaces the reference's traversal-step counters
   (testing/bvh/buildQual.h:65-126 NUM_TRAVERSAL_STEPS,
   testing/bvh/checkBuilders.cu:110-143 node/prim visit counts).  The same
   traversal as bq_closest_point_f3 (k == 0) or bq_knn_f3 (k in [1, 64]),
   or bq_tri_closest_f3 for the _tri_ form, is run once more, counting; the
   answers are discarded.  counts (HOST array of 3): [0] inner nodes
   expanded (each loads both 32-byte children), [1] node admin words
   loaded (16 B: the root and every stack entry descended), [2] prims
   tested.  Waits for the stream. */
int bq_query_visit_counts_f3(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t numQueries,
                             int k, float maxSqrDist, const bq_query_config *qcfg, uint64_t *counts,
                             const bq_allocator *alloc, bq_stream_t stream);
int bq_tri_visit_counts_f3(const bq_bvh3f *bvh, const int32_t *tris, const float *verts, const float *queries,
                           uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg, uint64_t *counts,
                           const bq_allocator *alloc, bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* batches of clouds (no counterpart in the reference, which builds    */
/* and queries one cloud per call)                                      */
/* ---------------------------------------------------------------- */

/* Builds one Morton63 BVH per cloud for numSegs clouds stored back to
   back: cloud s owns boxes[segOffsets[s] .. segOffsets[s+1]) (segOffsets:
   device array of numSegs+1 entries, segOffsets[numSegs] == numPrims).
   Each cloud's tree is exactly bq_build_morton63_f3's tree for that cloud
   alone.  Outputs go to caller buffers: nodes (2*numPrims entries; cloud s
   uses the block starting at 2*segOffsets[s]), primIDs (numPrims entries,
   cloud-local ids) and bvhs (device array of numSegs descriptors pointing
   into those buffers).  Every box must be non-empty.  No host
   synchronisation: the call can be captured in a CUDA graph (use the
   NULL allocator or a capture-safe one).  deviceErr (may be NULL) receives
   BQ device error bits; it is not read back. */
int bq_batched_build_morton63_f3(const bq_box3f *boxes, const uint32_t *segOffsets, uint32_t numSegs,
                                 uint32_t numPrims, const bq_build_config *cfg, bq_node3f *nodes, uint32_t *primIDs,
                                 bq_bvh3f *bvhs, uint32_t *deviceErr, const bq_allocator *alloc, bq_stream_t stream);

/* k nearest points per query over a batch built by the call above.
   Queries are stored cloud by cloud (queryOffsets: device, numSegs+1
   entries); query q of cloud s searches only cloud s (whose points start
   at points + 3*pointOffsets[s]).  ids are cloud-local.  A persistent
   work-stealing kernel answers the whole batch; qcfg->queriesPerWarp
   (a multiple of 32, default 32) is the number of queries a warp takes
   per grab.  No host synchronisation. */
int bq_batched_knn_f3(const bq_bvh3f *bvhs, const uint32_t *pointOffsets, const float *points, const float *queries,
                      const uint32_t *queryOffsets, uint32_t numSegs, uint32_t numQueries, int k, float maxSqrDist,
                      const bq_query_config *qcfg, int32_t *ids, float *sqrDist, int32_t *numFound,
                      uint32_t *deviceErr, const bq_allocator *alloc, bq_stream_t stream);

/* Refits every tree of a batch (after its boxes moved): segOffsets,
   nodes, primIDs and bvhs as produced by bq_batched_build_morton63_f3;
   boxes holds the batch's boxes back to back.  One launch pair for all
   trees, no host synchronisation. */
int bq_batched_refit_f3(const bq_bvh3f *bvhs, const uint32_t *segOffsets, uint32_t numSegs, uint32_t numPrims,
                        bq_node3f *nodes, const uint32_t *primIDs, const bq_box3f *boxes, const bq_allocator *alloc,
                        bq_stream_t stream);

/* Closest triangle per query over a batch of meshes built with
   bq_batched_build_morton63_f3 over triangle boxes: mesh s owns triangles
   tris[triOffsets[s] .. triOffsets[s+1]) (int32 vertex indices into one
   shared verts array); its queries are queries[queryOffsets[s] ..
   queryOffsets[s+1]).  ids are GLOBAL triangle indices (so
   bq_tri_distance_bwd_f3 can run on the shared arrays); -1 / +inf when
   nothing is within maxSqrDist.  No host synchronisation. */
int bq_batched_tri_closest_f3(const bq_bvh3f *bvhs, const uint32_t *triOffsets, const int32_t *tris,
                              const float *verts, const float *queries, const uint32_t *queryOffsets,
                              uint32_t numSegs, uint32_t numQueries, float maxSqrDist, const bq_query_config *qcfg,
                              int32_t *ids, float *sqrDist, float *P, uint32_t *deviceErr, const bq_allocator *alloc,
                              bq_stream_t stream);

/* Launch-shape autotuner for a batched build + kNN workload: times every
   combination of leaf threshold {1,2,4,8}, stack depth {32,64}, block
   size {64,128} and queries per warp {32,128} on the given inputs (CUDA
   events, after one warm-up) and returns the fastest.  With the default
   tie rule the answers do not depend on these knobs, only the time. */
typedef struct bq_tuning {
  int makeLeafThreshold;
  int stackDepth;
  int blockSize;
  int queriesPerWarp;
  float buildMs;
  float queryMs;
} bq_tuning;
int bq_autotune_batched_knn_f3(const bq_box3f *boxes, const float *points, const uint32_t *segOffsets,
                               uint32_t numSegs, uint32_t numPrims, const float *queries, const uint32_t *queryOffsets,
                               uint32_t numQueries, int k, bq_tuning *best, const bq_allocator *alloc,
                               bq_stream_t stream);

/* The same for one tree: Morton builds with leaf threshold {1,2,4,8},
   each queried with stack depth {32,64,128} x block size {64,128}, closest
   point (k == 0) or kNN (k in [1, 64]); best->queriesPerWarp is 32 (the
   single-tree kernels take one query per thread).  The fastest build +
   query is returned with its two times. */
int bq_autotune_query_f3(const bq_box3f *boxes, const float *points, uint32_t numPrims, const float *queries,
                         uint32_t numQueries, int k, bq_tuning *best, const bq_allocator *alloc, bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* input helpers                                                      */
/* ---------------------------------------------------------------- */

/* boxes[t] = bounds of triangle t (Triangle::bounds(),
   cuBQL/queries/triangles/Triangle.h:40-41). */
int bq_tri_boxes_f3(const int32_t *tris, const float *verts, uint32_t numTris, bq_box3f *boxes, bq_stream_t stream);

/* boxes[i] = the degenerate box of point i (box3f().including(p), as
   testing/points/closestPoint.cu:22-29 prepares point data). */
int bq_points_to_boxes_f3(const float *points, uint32_t numPoints, bq_box3f *boxes, bq_stream_t stream);

/* ---------------------------------------------------------------- */
/* misc                                                               */
/* ---------------------------------------------------------------- */
const char *bq_last_error_string(void);
int bq_version(void);

/* Phase profiler, the counterpart of the reference's CUBQL_PROFILE
   switch (cuBQL/builder/cuda/sm_builder.h:24-66, 505-607).  While enabled,
   every library call brackets its kernel phases with CUDA events on its
   stream; totals are kept per calling thread and per phase name.  The
   returned name stays valid until the next bq_profile_reset(). */
int bq_profile_enable(int on);
int bq_profile_reset(void);
int bq_profile_count(void);
int bq_profile_entry(int index, const char **name, uint64_t *launches, double *ms);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* BQ_H */
