// ref_gpu.cu -- C entry points over the reference library's own GPU code.
//
// TEST / BASELINE INFRASTRUCTURE ONLY.  Compiled by oracle/build_ref.sh
// with nvcc for sm_100a directly against the unmodified reference headers
// (never copied into this repository) into oracle/_ref/libref_gpu.so.
// The parity tests use it as the ground truth the CUDA library must match
// bit for bit; the comparison benchmark times it as "the reference's
// generic kernels compiled for sm_100a".
//
// All entry points take and return HOST arrays and manage device memory
// themselves, except the timing functions, which report CUDA-event times.
//
// Reference code wrapped here:
//   cuBQL::gpuBuilder           cuBQL/builder/cuda/gpu_builder.h:31-67
//   cuBQL::cuda::radixBuilder   cuBQL/builder/cuda/radix.h:760-771
//   cuBQL::cuda::rebinRadixBuilder cuBQL/builder/cuda/rebinMortonBuilder.h:1478-1487
//   points::findClosest / findKNN, triangles::findClosest (device functions,
//   launched one thread per query as testing/points/closestPoint.cu:37-58)
//   fixedBoxQuery::forEachPrim  cuBQL/traversal/fixedBoxQuery.h:139-156, with
//   a lambda that keeps prims whose box overlaps the query box
//   gpuBuilder(WideBVH<float,3,W>&) cuBQL/builder/cuda/wide_gpu_builder.h:162-213,
//   points::findClosest(WideBVH) and fixedBoxQuery::forEachPrim(WideBVH)
#define CUBQL_GPU_BUILDER_IMPLEMENTATION 1
#include "cuBQL/bvh.h"
#include "cuBQL/builder/cuda/radix.h"
#include "cuBQL/builder/cuda/rebinMortonBuilder.h"
#include "cuBQL/queries/points/findClosest.h"
#include "cuBQL/queries/points/knn.h"
#include "cuBQL/queries/triangles/findClosest.h"
#include "cuBQL/traversal/fixedBoxQuery.h"

#include <cstdio>
#include <vector>

using namespace cuBQL;

#define RCHECK(x)                                                                  \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      fprintf(stderr, "ref_gpu: %s failed: %s\n", #x, cudaGetErrorString(e_));     \
      return -1;                                                                   \
    }                                                                              \
  } while (0)

namespace {
template <typename T>
T *dalloc_copy(const T *h, size_t n)
{
  T *d = nullptr;
  if (cudaMalloc((void **)&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
  if (n && h) cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
  return d;
}

struct DeviceTree {
  bvh3f bvh;
  int upload(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims)
  {
    bvh.nodes = (bvh3f::Node *)dalloc_copy((const char *)nodes, sizeof(bvh3f::Node) * (size_t)numNodes);
    bvh.primIDs = dalloc_copy(primIDs, numPrims);
    bvh.numNodes = numNodes;
    bvh.numPrims = numPrims;
    return (bvh.nodes && bvh.primIDs) ? 0 : -1;
  }
  ~DeviceTree()
  {
    cudaFree(bvh.nodes);
    cudaFree(bvh.primIDs);
  }
};

__global__ void k_closest(bvh3f bvh, const vec3f *pts, const vec3f *qs, int nq, float maxSqr, int *ids,
                          float *dists)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  int id = points::findClosest(bvh, pts, qs[tid], maxSqr);
  ids[tid] = id;
  dists[tid] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[tid]);
}

// excl != nullptr: findClosest_exludeID(excl[tid]); else findClosest_exludeSelf
__global__ void k_closest_exclude(bvh3f bvh, const vec3f *pts, const vec3f *qs, int nq, float maxSqr,
                                  const int *excl, int *ids, float *dists)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  int id = excl ? points::findClosest_exludeID(excl[tid], bvh, pts, qs[tid], maxSqr)
                : points::findClosest_exludeSelf(bvh, pts, qs[tid], maxSqr);
  ids[tid] = id;
  dists[tid] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[tid]);
}

// offsets == nullptr: count pass (counts[tid]); else fill ids[offsets[tid]..]
__global__ void k_box(bvh3f bvh, const box3f *boxes, const box3f *qb, int nq, const unsigned long long *offsets,
                      unsigned *counts, int *ids)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  const box3f q = qb[tid];
  unsigned c = 0;
  auto perPrim = [&](uint32_t primID) -> int {
    if (q.overlaps(boxes[primID])) {
      if (offsets) ids[offsets[tid] + c] = (int)primID;
      c++;
    }
    return CUBQL_CONTINUE_TRAVERSAL;
  };
  fixedBoxQuery::forEachPrim(perPrim, bvh, q);
  counts[tid] = c;
}

// evaluateSAH and surfaceArea of the reference, for pinning their FMA shapes
static_assert(sizeof(sahBuilder_impl::SAHBins) == 1536, "SAHBins layout");
__global__ void k_sah_pin(const sahBuilder_impl::SAHBins *bins, int nb, int *dims, int *splitBins,
                          const box3f *boxes, int nbox, float *areas)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid < nb) {
    int splitDim = -1, splitBin = 0;
    sahBuilder_impl::evaluateSAH(splitDim, splitBin, bins[tid]);
    dims[tid] = splitDim;
    splitBins[tid] = splitDim < 0 ? 0 : splitBin;
  }
  if (tid < nbox) areas[tid] = surfaceArea(boxes[tid]);
}

static_assert(sizeof(elhBuilder_impl::ELHBins<float, 3>) == 768, "ELHBins layout");
__global__ void k_elh_pin(const elhBuilder_impl::ELHBins<float, 3> *bins, int nb, int *dims, int *splitBins)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nb) return;
  int splitDim = -1, splitBin = 0;
  elhBuilder_impl::evaluateELH<float, 3>(splitDim, splitBin, bins[tid]);
  dims[tid] = splitDim;
  splitBins[tid] = splitDim < 0 ? 0 : splitBin;
}

template <int KMAX>
__global__ void k_knn(bvh3f bvh, const vec3f *pts, const vec3f *qs, int nq, int k, float maxSqr, int *ids,
                      float *dists, int *numFound)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  knn::Candidate c[KMAX];
  knn::Result r = points::findKNN(c, k, bvh, pts, qs[tid], maxSqr);
  for (int j = 0; j < k; j++) {
    ids[(size_t)tid * k + j] = j < r.numFound ? c[j].primID : -1;
    dists[(size_t)tid * k + j] = j < r.numFound ? c[j].sqrDist : INFINITY;
  }
  numFound[tid] = r.numFound;
}

__global__ void k_tri(bvh3f bvh, const Triangle *tris, const vec3f *qs, int nq, float maxSqr, int *ids,
                      float *dists, vec3f *P)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  triangles::FCPResult r;
  r.clear(maxSqr);
  r.P = vec3f(0.f, 0.f, 0.f);
  triangles::findClosest(r, bvh, tris, qs[tid]);
  ids[tid] = r.primID;
  dists[tid] = r.primID < 0 ? INFINITY : r.sqrDist;
  P[tid] = r.P;
}

__global__ void k_pin(const vec3f *a, const vec3f *b, const box3f *bx, int n, float *pp, float *pbox)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  pp[tid] = fSqrDistance_rd(a[tid], b[tid]);
  pbox[tid] = shrinkingRadiusQuery::fSqrDistance_rd(a[tid], bx[tid]);
}

__global__ void k_points_to_boxes(const vec3f *pts, box3f *boxes, int n)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  boxes[tid] = box3f().including(pts[tid]);
}

// ---- wide trees ----
template <int W>
using wbvh = WideBVH<float, 3, W>;
static_assert(sizeof(wbvh<4>::Node) == 4 * 32 && sizeof(wbvh<8>::Node) == 8 * 32, "wide node layout");

template <int W>
struct DeviceWide {
  wbvh<W> bvh;
  int upload(const void *slots, uint32_t numWide, const uint32_t *primIDs, uint32_t numPrims)
  {
    bvh.nodes = (typename wbvh<W>::Node *)dalloc_copy((const char *)slots, sizeof(typename wbvh<W>::Node) * numWide);
    bvh.primIDs = dalloc_copy(primIDs, numPrims);
    bvh.numNodes = numWide;
    bvh.numPrims = numPrims;
    return (bvh.nodes && bvh.primIDs) ? 0 : -1;
  }
  ~DeviceWide()
  {
    cudaFree(bvh.nodes);
    cudaFree(bvh.primIDs);
  }
};

template <int W>
__global__ void k_wide_closest(wbvh<W> bvh, const vec3f *pts, const vec3f *qs, int nq, float maxSqr, int *ids,
                               float *dists)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  int id = points::findClosest(bvh, pts, qs[tid], maxSqr);
  ids[tid] = id;
  dists[tid] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[tid]);
}

template <int W>
__global__ void k_wide_box(wbvh<W> bvh, const box3f *boxes, const box3f *qb, int nq,
                           const unsigned long long *offsets, unsigned *counts, int *ids)
{
  int tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= nq) return;
  const box3f q = qb[tid];
  unsigned c = 0;
  auto perPrim = [&](uint32_t primID) -> int {
    if (q.overlaps(boxes[primID])) {
      if (offsets) ids[offsets[tid] + c] = (int)primID;
      c++;
    }
    return CUBQL_CONTINUE_TRAVERSAL;
  };
  fixedBoxQuery::forEachPrim(perPrim, bvh, q);
  counts[tid] = c;
}

template <int W>
int build_wide_t(const float *boxes, uint32_t n, int thr, void *slotsOut, uint32_t *primsOut, uint32_t *numWide,
                 uint32_t *numPrims)
{
  box3f *d_boxes = dalloc_copy((const box3f *)boxes, n);
  if (!d_boxes) return -1;
  wbvh<W> bvh;
  BuildConfig cfg;
  cfg.makeLeafThreshold = thr;
  gpuBuilder(bvh, d_boxes, n, cfg);
  RCHECK(cudaDeviceSynchronize());
  *numWide = bvh.numNodes;
  *numPrims = bvh.numPrims;
  if (bvh.numNodes)
    RCHECK(cudaMemcpy(slotsOut, bvh.nodes, sizeof(typename wbvh<W>::Node) * bvh.numNodes, cudaMemcpyDeviceToHost));
  if (bvh.numPrims) RCHECK(cudaMemcpy(primsOut, bvh.primIDs, sizeof(uint32_t) * bvh.numPrims, cudaMemcpyDeviceToHost));
  cuBQL::cuda::free(bvh);
  cudaFree(d_boxes);
  return 0;
}

template <int W>
int wide_closest_t(const void *slots, uint32_t numWide, const uint32_t *primIDs, uint32_t numPrims,
                   const float *points, uint32_t np, const float *queries, uint32_t nq, float maxSqr, int32_t *ids,
                   float *dists)
{
  DeviceWide<W> t;
  if (t.upload(slots, numWide, primIDs, numPrims)) return -1;
  vec3f *dp = dalloc_copy((const vec3f *)points, np), *dq = dalloc_copy((const vec3f *)queries, nq);
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  k_wide_closest<W><<<(nq + 127) / 128, 128>>>(t.bvh, dp, dq, (int)nq, maxSqr, di, dd);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(ids, di, sizeof(int) * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(dists, dd, sizeof(float) * nq, cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dq); cudaFree(di); cudaFree(dd);
  return 0;
}

template <int W>
int wide_box_t(const void *slots, uint32_t numWide, const uint32_t *primIDs, uint32_t numPrims, const float *boxes,
               uint32_t nb, const float *queryBoxes, uint32_t nq, uint32_t *counts, const uint64_t *offsets,
               int32_t *ids)
{
  DeviceWide<W> t;
  if (t.upload(slots, numWide, primIDs, numPrims)) return -1;
  box3f *db = dalloc_copy((const box3f *)boxes, nb), *dq = dalloc_copy((const box3f *)queryBoxes, nq);
  unsigned *dc = dalloc_copy<unsigned>(nullptr, nq);
  unsigned long long *doff = ids ? dalloc_copy((const unsigned long long *)offsets, nq + 1) : nullptr;
  const size_t total = ids ? offsets[nq] : 0;
  int *di = ids ? dalloc_copy<int>(nullptr, total) : nullptr;
  k_wide_box<W><<<(nq + 127) / 128, 128>>>(t.bvh, db, dq, (int)nq, doff, dc, di);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(counts, dc, sizeof(unsigned) * nq, cudaMemcpyDeviceToHost);
  if (ids && total) cudaMemcpy(ids, di, sizeof(int) * total, cudaMemcpyDeviceToHost);
  cudaFree(db); cudaFree(dq); cudaFree(dc);
  if (doff) cudaFree(doff);
  if (di) cudaFree(di);
  return 0;
}

template <int W>
float time_wide_query_t(const float *points, uint32_t n, int thr, const float *queries, uint32_t nq, int reps)
{
  vec3f *dp = dalloc_copy((const vec3f *)points, n), *dq = dalloc_copy((const vec3f *)queries, nq);
  box3f *db = dalloc_copy<box3f>(nullptr, n);
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  if (!dp || !dq || !db || !di || !dd) return -1.f;
  k_points_to_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  wbvh<W> bvh;
  BuildConfig cfg;
  cfg.makeLeafThreshold = thr;
  gpuBuilder(bvh, db, n, cfg);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1.f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    cudaEventRecord(e0);
    k_wide_closest<W><<<(nq + 127) / 128, 128>>>(bvh, dp, dq, (int)nq, INFINITY, di, dd);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cuBQL::cuda::free(bvh);
  cudaFree(dp); cudaFree(dq); cudaFree(db); cudaFree(di); cudaFree(dd);
  return total / (reps > 0 ? reps : 1);
}

// CUDA-event time of gpuBuilder(WideBVH<float,3,W>&) (free not timed)
template <int W>
float time_wide_build_t(const box3f *db, uint32_t n, int thr, int reps)
{
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  BuildConfig cfg;
  cfg.makeLeafThreshold = thr;
  for (int r = -1; r < reps; r++) {
    wbvh<W> w;
    cudaEventRecord(e0);
    gpuBuilder(w, db, n, cfg);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
    cuBQL::cuda::free(w);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return total / (reps > 0 ? reps : 1);
}

int run_build(int method, const box3f *d_boxes, uint32_t n, int leafThr, bvh3f &bvh)
{
  BuildConfig cfg;
  cfg.makeLeafThreshold = leafThr;
  if (method == 5)
    cuBQL::cuda::sahBuilder(bvh, d_boxes, n, cfg);
  else if (method == 6) {  // gpuBuilder with BuildConfig::ELH (gpu_builder.h:54-59)
    cfg.buildMethod = BuildConfig::ELH;
    gpuBuilder(bvh, d_boxes, n, cfg);
  }
  else if (method == 0)
    cuBQL::cuda::radixBuilder(bvh, d_boxes, n, cfg);
  else if (method == 1)
    gpuBuilder(bvh, d_boxes, n, cfg);
  else
    cuBQL::cuda::rebinRadixBuilder(bvh, d_boxes, n, cfg);
  return 0;
}
} // namespace

extern "C" {

int ref_gpu_node_size(void) { return (int)sizeof(bvh3f::Node); }

// method: 0 radixBuilder, 1 gpuBuilder (spatial median), 2 rebinRadixBuilder,
// 5 cuda::sahBuilder, 6 gpuBuilder with BuildConfig::ELH.
// nodesOut must hold 2n+2 nodes, primIDsOut n entries.
int ref_gpu_build(int method, const float *boxes, uint32_t n, int makeLeafThreshold, void *nodesOut,
                  uint32_t *primIDsOut, uint32_t *numNodes, uint32_t *numPrims)
{
  box3f *d_boxes = dalloc_copy((const box3f *)boxes, n);
  if (!d_boxes) return -1;
  bvh3f bvh;
  run_build(method, d_boxes, n, makeLeafThreshold, bvh);
  RCHECK(cudaDeviceSynchronize());
  *numNodes = bvh.numNodes;
  *numPrims = bvh.numPrims;
  if (bvh.numNodes) RCHECK(cudaMemcpy(nodesOut, bvh.nodes, sizeof(bvh3f::Node) * bvh.numNodes, cudaMemcpyDeviceToHost));
  if (bvh.numPrims) RCHECK(cudaMemcpy(primIDsOut, bvh.primIDs, sizeof(uint32_t) * bvh.numPrims, cudaMemcpyDeviceToHost));
  if (bvh.numNodes) cuBQL::cuda::free(bvh);
  cudaFree(d_boxes);
  return 0;
}

int ref_gpu_closest(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                    const float *points, uint32_t np, const float *queries, uint32_t nq, float maxSqr, int32_t *ids,
                    float *dists)
{
  DeviceTree t;
  if (t.upload(nodes, numNodes, primIDs, numPrims)) return -1;
  vec3f *dp = dalloc_copy((const vec3f *)points, np), *dq = dalloc_copy((const vec3f *)queries, nq);
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  k_closest<<<(nq + 127) / 128, 128>>>(t.bvh, dp, dq, (int)nq, maxSqr, di, dd);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(ids, di, sizeof(int) * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(dists, dd, sizeof(float) * nq, cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dq); cudaFree(di); cudaFree(dd);
  return 0;
}

int ref_gpu_closest_exclude(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                            const float *points, uint32_t np, const float *queries, uint32_t nq, float maxSqr,
                            const int32_t *excludeIds, int32_t *ids, float *dists)
{
  DeviceTree t;
  if (t.upload(nodes, numNodes, primIDs, numPrims)) return -1;
  vec3f *dp = dalloc_copy((const vec3f *)points, np), *dq = dalloc_copy((const vec3f *)queries, nq);
  int *dx = excludeIds ? dalloc_copy((const int *)excludeIds, nq) : nullptr;
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  k_closest_exclude<<<(nq + 127) / 128, 128>>>(t.bvh, dp, dq, (int)nq, maxSqr, dx, di, dd);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(ids, di, sizeof(int) * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(dists, dd, sizeof(float) * nq, cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dq); cudaFree(di); cudaFree(dd);
  if (dx) cudaFree(dx);
  return 0;
}

// Both passes of the reference box query; offsets (nq+1) and ids are host
// arrays sized by the caller after a count-only call (ids == NULL).
int ref_gpu_box_query(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                      const float *boxes, uint32_t nb, const float *queryBoxes, uint32_t nq, uint32_t *counts,
                      const uint64_t *offsets, int32_t *ids)
{
  DeviceTree t;
  if (t.upload(nodes, numNodes, primIDs, numPrims)) return -1;
  box3f *db = dalloc_copy((const box3f *)boxes, nb), *dq = dalloc_copy((const box3f *)queryBoxes, nq);
  unsigned *dc = dalloc_copy<unsigned>(nullptr, nq);
  unsigned long long *doff = ids ? dalloc_copy((const unsigned long long *)offsets, nq + 1) : nullptr;
  const size_t total = ids ? offsets[nq] : 0;
  int *di = ids ? dalloc_copy<int>(nullptr, total) : nullptr;
  k_box<<<(nq + 127) / 128, 128>>>(t.bvh, db, dq, (int)nq, doff, dc, di);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(counts, dc, sizeof(unsigned) * nq, cudaMemcpyDeviceToHost);
  if (ids && total) cudaMemcpy(ids, di, sizeof(int) * total, cudaMemcpyDeviceToHost);
  cudaFree(db); cudaFree(dq); cudaFree(dc);
  if (doff) cudaFree(doff);
  if (di) cudaFree(di);
  return 0;
}

int ref_gpu_knn(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                const float *points, uint32_t np, const float *queries, uint32_t nq, int k, float maxSqr,
                int32_t *ids, float *dists, int32_t *numFound)
{
  if (k < 1 || k > 64) return -1;
  DeviceTree t;
  if (t.upload(nodes, numNodes, primIDs, numPrims)) return -1;
  vec3f *dp = dalloc_copy((const vec3f *)points, np), *dq = dalloc_copy((const vec3f *)queries, nq);
  int *di = dalloc_copy<int>(nullptr, (size_t)nq * k), *dn = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, (size_t)nq * k);
  if (k <= 16)
    k_knn<16><<<(nq + 127) / 128, 128>>>(t.bvh, dp, dq, (int)nq, k, maxSqr, di, dd, dn);
  else
    k_knn<64><<<(nq + 127) / 128, 128>>>(t.bvh, dp, dq, (int)nq, k, maxSqr, di, dd, dn);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(ids, di, sizeof(int) * nq * k, cudaMemcpyDeviceToHost);
  cudaMemcpy(dists, dd, sizeof(float) * nq * k, cudaMemcpyDeviceToHost);
  cudaMemcpy(numFound, dn, sizeof(int) * nq, cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dq); cudaFree(di); cudaFree(dd); cudaFree(dn);
  return 0;
}

int ref_gpu_tri_closest(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                        const int32_t *tris, uint32_t nt, const float *verts, const float *queries, uint32_t nq,
                        float maxSqr, int32_t *ids, float *dists, float *P)
{
  DeviceTree t;
  if (t.upload(nodes, numNodes, primIDs, numPrims)) return -1;
  std::vector<Triangle> T(nt);
  const vec3f *V = (const vec3f *)verts;
  for (uint32_t i = 0; i < nt; i++) {
    T[i].a = V[tris[3 * i + 0]];
    T[i].b = V[tris[3 * i + 1]];
    T[i].c = V[tris[3 * i + 2]];
  }
  Triangle *dt = dalloc_copy(T.data(), nt);
  vec3f *dq = dalloc_copy((const vec3f *)queries, nq), *dP = dalloc_copy<vec3f>(nullptr, nq);
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  k_tri<<<(nq + 127) / 128, 128>>>(t.bvh, dt, dq, (int)nq, maxSqr, di, dd, dP);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(ids, di, sizeof(int) * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(dists, dd, sizeof(float) * nq, cudaMemcpyDeviceToHost);
  if (P) cudaMemcpy(P, dP, sizeof(vec3f) * nq, cudaMemcpyDeviceToHost);
  cudaFree(dt); cudaFree(dq); cudaFree(dP); cudaFree(di); cudaFree(dd);
  return 0;
}

// The two distance expressions the reference's device code uses, evaluated
// by the reference's own functions, to pin their FMA contraction.
int ref_gpu_pin(const float *a, const float *b, const float *boxes, uint32_t n, float *pp, float *pbox)
{
  vec3f *da = dalloc_copy((const vec3f *)a, n), *db = dalloc_copy((const vec3f *)b, n);
  box3f *dbx = dalloc_copy((const box3f *)boxes, n);
  float *d1 = dalloc_copy<float>(nullptr, n), *d2 = dalloc_copy<float>(nullptr, n);
  k_pin<<<(n + 127) / 128, 128>>>(da, db, dbx, (int)n, d1, d2);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(pp, d1, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(pbox, d2, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(da); cudaFree(db); cudaFree(dbx); cudaFree(d1); cudaFree(d2);
  return 0;
}

// Times the reference's GPU builders on point boxes already resident in
// device memory: one warm-up build, then `reps` builds, CUDA events around
// each (the builders' own host syncs included, as a user sees them).
// ms_out receives the mean build time.
int ref_gpu_time_build(int method, const float *points, uint32_t n, int makeLeafThreshold, int reps,
                       float *ms_out)
{
  vec3f *dp = dalloc_copy((const vec3f *)points, n);
  box3f *db = dalloc_copy<box3f>(nullptr, n);
  if (!dp || !db) return -1;
  k_points_to_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  RCHECK(cudaDeviceSynchronize());
  if (method == 3 || method == 4) {  // gpuBuilder into a WideBVH<float,3,4|8>
    *ms_out = method == 3 ? time_wide_build_t<4>(db, n, makeLeafThreshold, reps)
                          : time_wide_build_t<8>(db, n, makeLeafThreshold, reps);
    cudaFree(dp);
    cudaFree(db);
    return *ms_out < 0.f ? -1 : 0;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    bvh3f bvh;
    cudaEventRecord(e0);
    run_build(method, db, n, makeLeafThreshold, bvh);
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
    cuBQL::cuda::free(bvh);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dp);
  cudaFree(db);
  *ms_out = total / (reps > 0 ? reps : 1);
  return 0;
}

// As ref_gpu_time_build, over given boxes (e.g. triangle boxes)
int ref_gpu_time_build_boxes(int method, const float *boxes, uint32_t n, int makeLeafThreshold, int reps,
                             float *ms_out)
{
  box3f *db = dalloc_copy((const box3f *)boxes, n);
  if (!db) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    bvh3f bvh;
    cudaEventRecord(e0);
    run_build(method, db, n, makeLeafThreshold, bvh);
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
    cuBQL::cuda::free(bvh);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(db);
  *ms_out = total / (reps > 0 ? reps : 1);
  return 0;
}

// Times one-thread-per-query reference kernels over a tree built with
// `method` on the points: kind 0 closest point, kind k>0 kNN with that k.
int ref_gpu_time_query(int method, const float *points, uint32_t n, int makeLeafThreshold, const float *queries,
                       uint32_t nq, int kind, int reps, float *ms_out)
{
  vec3f *dp = dalloc_copy((const vec3f *)points, n), *dq = dalloc_copy((const vec3f *)queries, nq);
  box3f *db = dalloc_copy<box3f>(nullptr, n);
  int k = kind > 0 ? kind : 1;
  int *di = dalloc_copy<int>(nullptr, (size_t)nq * k), *dn = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, (size_t)nq * k);
  if (!dp || !dq || !db || !di || !dn || !dd) return -1;
  k_points_to_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  bvh3f bvh;
  run_build(method, db, n, makeLeafThreshold, bvh);
  RCHECK(cudaDeviceSynchronize());
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    cudaEventRecord(e0);
    if (kind == -1)
      k_closest_exclude<<<(nq + 127) / 128, 128>>>(bvh, dp, dq, (int)nq, INFINITY, nullptr, di, dd);
    else if (kind == 0)
      k_closest<<<(nq + 127) / 128, 128>>>(bvh, dp, dq, (int)nq, INFINITY, di, dd);
    else if (k <= 16)
      k_knn<16><<<(nq + 127) / 128, 128>>>(bvh, dp, dq, (int)nq, k, INFINITY, di, dd, dn);
    else
      k_knn<64><<<(nq + 127) / 128, 128>>>(bvh, dp, dq, (int)nq, k, INFINITY, di, dd, dn);
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cuBQL::cuda::free(bvh);
  cudaFree(dp); cudaFree(dq); cudaFree(db); cudaFree(di); cudaFree(dn); cudaFree(dd);
  *ms_out = total / (reps > 0 ? reps : 1);
  return 0;
}

// Times the reference's per-thread triangles::findClosest kernel
// (<<<ceil(Q/128),128>>>) over a tree built with `method` on the triangle
// boxes; the tree build is not timed.
int ref_gpu_time_tri(int method, const int32_t *tris, uint32_t nt, const float *verts, const float *queries,
                     uint32_t nq, int reps, float *ms_out)
{
  std::vector<Triangle> T(nt);
  std::vector<box3f> B(nt);
  const vec3f *V = (const vec3f *)verts;
  for (uint32_t i = 0; i < nt; i++) {
    T[i].a = V[tris[3 * i + 0]];
    T[i].b = V[tris[3 * i + 1]];
    T[i].c = V[tris[3 * i + 2]];
    B[i] = box3f().including(T[i].a).including(T[i].b).including(T[i].c);
  }
  Triangle *dt = dalloc_copy(T.data(), nt);
  box3f *db = dalloc_copy(B.data(), nt);
  vec3f *dq = dalloc_copy((const vec3f *)queries, nq), *dP = dalloc_copy<vec3f>(nullptr, nq);
  int *di = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, nq);
  if (!dt || !db || !dq || !dP || !di || !dd) return -1;
  bvh3f bvh;
  run_build(method, db, nt, 0, bvh);
  RCHECK(cudaDeviceSynchronize());
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    cudaEventRecord(e0);
    k_tri<<<(nq + 127) / 128, 128>>>(bvh, dt, dq, (int)nq, INFINITY, di, dd, dP);
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cuBQL::cuda::free(bvh);
  cudaFree(dt); cudaFree(db); cudaFree(dq); cudaFree(dP); cudaFree(di); cudaFree(dd);
  *ms_out = total / (reps > 0 ? reps : 1);
  return 0;
}

// Times the reference's way of serving a batch of clouds: for every cloud,
// radixBuilder over its point boxes, then its per-thread findKNN kernel
// (<<<ceil(Q/128),128>>>) over its queries, then cuda::free; one CUDA event
// pair around the whole loop (the builder's own host syncs included).
// Points and queries are stored back to back; off / qoff hold numSegs+1
// offsets each.
int ref_gpu_time_batched_knn(const float *points, const uint32_t *off, const float *queries, const uint32_t *qoff,
                             uint32_t numSegs, int k, float *ms_out)
{
  const uint32_t n = off[numSegs], nq = qoff[numSegs];
  vec3f *dp = dalloc_copy((const vec3f *)points, n), *dq = dalloc_copy((const vec3f *)queries, nq);
  box3f *db = dalloc_copy<box3f>(nullptr, n);
  int *di = dalloc_copy<int>(nullptr, (size_t)nq * k), *dn = dalloc_copy<int>(nullptr, nq);
  float *dd = dalloc_copy<float>(nullptr, (size_t)nq * k);
  if (!dp || !dq || !db || !di || !dn || !dd || k > 16) return -1;
  k_points_to_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  RCHECK(cudaDeviceSynchronize());
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < 1; r++) {  // one warm-up loop, one timed loop
    cudaEventRecord(e0);
    for (uint32_t c = 0; c < numSegs; c++) {
      const uint32_t cn = off[c + 1] - off[c], cq = qoff[c + 1] - qoff[c];
      bvh3f bvh;
      cuBQL::cuda::radixBuilder(bvh, db + off[c], cn, BuildConfig());
      k_knn<16><<<(cq + 127) / 128, 128>>>(bvh, dp + off[c], dq + qoff[c], (int)cq, k, INFINITY,
                                         di + (size_t)qoff[c] * k, dd + (size_t)qoff[c] * k, dn + qoff[c]);
      cuBQL::cuda::free(bvh);
    }
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&total, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dp); cudaFree(dq); cudaFree(db); cudaFree(di); cudaFree(dn); cudaFree(dd);
  *ms_out = total;
  return 0;
}

// Times the reference box query (count kernel + fill kernel, offsets from
// an untimed count pass) over a tree of `method` built on point boxes.
int ref_gpu_time_box_query(int method, const float *points, uint32_t n, int makeLeafThreshold,
                           const float *queryBoxes, uint32_t nq, int reps, float *ms_out, uint64_t *total_out)
{
  vec3f *dp = dalloc_copy((const vec3f *)points, n);
  box3f *db = dalloc_copy<box3f>(nullptr, n), *dq = dalloc_copy((const box3f *)queryBoxes, nq);
  unsigned *dc = dalloc_copy<unsigned>(nullptr, nq);
  unsigned long long *doff = dalloc_copy<unsigned long long>(nullptr, nq + 1);
  if (!dp || !db || !dq || !dc || !doff) return -1;
  k_points_to_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  bvh3f bvh;
  run_build(method, db, n, makeLeafThreshold, bvh);
  k_box<<<(nq + 127) / 128, 128>>>(bvh, db, dq, (int)nq, nullptr, dc, nullptr);
  RCHECK(cudaDeviceSynchronize());
  std::vector<unsigned> hc(nq);
  std::vector<unsigned long long> ho(nq + 1, 0);
  cudaMemcpy(hc.data(), dc, sizeof(unsigned) * nq, cudaMemcpyDeviceToHost);
  for (uint32_t i = 0; i < nq; i++) ho[i + 1] = ho[i] + hc[i];
  cudaMemcpy(doff, ho.data(), sizeof(unsigned long long) * (nq + 1), cudaMemcpyHostToDevice);
  int *di = dalloc_copy<int>(nullptr, ho[nq]);
  if (!di) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float total = 0.f;
  for (int r = -1; r < reps; r++) {
    cudaEventRecord(e0);
    k_box<<<(nq + 127) / 128, 128>>>(bvh, db, dq, (int)nq, nullptr, dc, nullptr);
    k_box<<<(nq + 127) / 128, 128>>>(bvh, db, dq, (int)nq, doff, dc, di);
    cudaEventRecord(e1);
    RCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0) total += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cuBQL::cuda::free(bvh);
  cudaFree(dp); cudaFree(db); cudaFree(dq); cudaFree(dc); cudaFree(doff); cudaFree(di);
  *ms_out = total / (reps > 0 ? reps : 1);
  *total_out = ho[nq];
  return 0;
}

int ref_gpu_sah_pin(const void *bins, int nb, int *dims, int *splitBins, const float *boxes, int nbox, float *areas)
{
  auto *db = dalloc_copy((const sahBuilder_impl::SAHBins *)bins, nb);
  box3f *dbox = dalloc_copy((const box3f *)boxes, nbox);
  int *dd = dalloc_copy<int>(nullptr, nb), *ds = dalloc_copy<int>(nullptr, nb);
  float *da = dalloc_copy<float>(nullptr, nbox);
  const int n = nb > nbox ? nb : nbox;
  k_sah_pin<<<(n + 127) / 128, 128>>>(db, nb, dd, ds, dbox, nbox, da);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(dims, dd, sizeof(int) * nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(splitBins, ds, sizeof(int) * nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(areas, da, sizeof(float) * nbox, cudaMemcpyDeviceToHost);
  cudaFree(db); cudaFree(dbox); cudaFree(dd); cudaFree(ds); cudaFree(da);
  return 0;
}

int ref_gpu_elh_pin(const void *bins, int nb, int *dims, int *splitBins)
{
  auto *db = dalloc_copy((const elhBuilder_impl::ELHBins<float, 3> *)bins, nb);
  int *dd = dalloc_copy<int>(nullptr, nb), *ds = dalloc_copy<int>(nullptr, nb);
  k_elh_pin<<<(nb + 127) / 128, 128>>>(db, nb, dd, ds);
  RCHECK(cudaDeviceSynchronize());
  cudaMemcpy(dims, dd, sizeof(int) * nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(splitBins, ds, sizeof(int) * nb, cudaMemcpyDeviceToHost);
  cudaFree(db); cudaFree(dd); cudaFree(ds);
  return 0;
}

// ---- wide trees (W = 4 or 8) ----
// slotsOut holds (2n+2)*W slots, primsOut n entries
int ref_gpu_build_wide(int W, const float *boxes, uint32_t n, int thr, void *slotsOut, uint32_t *primsOut,
                       uint32_t *numWide, uint32_t *numPrims)
{
  if (W == 4) return build_wide_t<4>(boxes, n, thr, slotsOut, primsOut, numWide, numPrims);
  if (W == 8) return build_wide_t<8>(boxes, n, thr, slotsOut, primsOut, numWide, numPrims);
  return -1;
}

int ref_gpu_wide_closest(int W, const void *slots, uint32_t numWide, const uint32_t *primIDs, uint32_t numPrims,
                         const float *points, uint32_t np, const float *queries, uint32_t nq, float maxSqr,
                         int32_t *ids, float *dists)
{
  if (W == 4) return wide_closest_t<4>(slots, numWide, primIDs, numPrims, points, np, queries, nq, maxSqr, ids, dists);
  if (W == 8) return wide_closest_t<8>(slots, numWide, primIDs, numPrims, points, np, queries, nq, maxSqr, ids, dists);
  return -1;
}

int ref_gpu_wide_box_query(int W, const void *slots, uint32_t numWide, const uint32_t *primIDs, uint32_t numPrims,
                           const float *boxes, uint32_t nb, const float *queryBoxes, uint32_t nq, uint32_t *counts,
                           const uint64_t *offsets, int32_t *ids)
{
  if (W == 4) return wide_box_t<4>(slots, numWide, primIDs, numPrims, boxes, nb, queryBoxes, nq, counts, offsets, ids);
  if (W == 8) return wide_box_t<8>(slots, numWide, primIDs, numPrims, boxes, nb, queryBoxes, nq, counts, offsets, ids);
  return -1;
}

int ref_gpu_time_wide_query(int W, const float *points, uint32_t n, int thr, const float *queries, uint32_t nq,
                            int reps, float *ms_out)
{
  float ms = W == 4 ? time_wide_query_t<4>(points, n, thr, queries, nq, reps)
                    : (W == 8 ? time_wide_query_t<8>(points, n, thr, queries, nq, reps) : -1.f);
  *ms_out = ms;
  return ms < 0.f ? -1 : 0;
}

} // extern "C"
