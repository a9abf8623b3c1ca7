// ref_shim.cu -- the drop-in check: the reference's own types and device
// query code running on trees built by libbq through include/bq_cubql.hpp.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/build_ref.sh against the
// unmodified reference headers into oracle/_ref/libref_shim.so, linked to
// cubql_b200/libbq.so.  For the same boxes it
//   1. builds with cuBQL::cuda::radixBuilder (the reference),
//   2. builds with bq_cubql::cuda::radixBuilder (this library, called with
//      the reference's BinaryBVH, box3f, BuildConfig and GpuMemoryResource),
//   3. runs the reference's points::findClosest kernel on BOTH trees,
// so a test can check that the reference's traversal reads our tree and
// answers exactly as on its own tree.  ref_shim_compare_more does the same
// for cuda::sahBuilder and gpuBuilder(WideBVH<float,3,4>&) (the
// reference's binary and wide findClosest kernels on both trees), and runs
// bq_cubql::triangles::findClosest against the reference's per-thread
// triangles::findClosest kernel on the reference's own tree.
#define CUBQL_GPU_BUILDER_IMPLEMENTATION 1
#include "cuBQL/bvh.h"
#include "cuBQL/builder/cuda/radix.h"
#include "cuBQL/queries/points/findClosest.h"
#include "cuBQL/queries/triangles/findClosest.h"

#include "bq_cubql.hpp"

#include <vector>

using namespace cuBQL;

namespace {
__global__ void k_boxes(const vec3f *pts, box3f *boxes, int n)
{
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i < n) boxes[i] = box3f().including(pts[i]);
}

__global__ void k_query(bvh3f bvh, const vec3f *pts, const vec3f *qs, int nq, int *ids, float *d)
{
  int t = threadIdx.x + blockIdx.x * blockDim.x;
  if (t >= nq) return;
  int id = points::findClosest(bvh, pts, qs[t], INFINITY);
  ids[t] = id;
  d[t] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[t]);
}

template <int W>
__global__ void k_wide_query(WideBVH<float, 3, W> bvh, const vec3f *pts, const vec3f *qs, int nq, int *ids, float *d)
{
  int t = threadIdx.x + blockIdx.x * blockDim.x;
  if (t >= nq) return;
  int id = points::findClosest(bvh, pts, qs[t], INFINITY);
  ids[t] = id;
  d[t] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[t]);
}

__global__ void k_tri_query(bvh3f bvh, const Triangle *tris, const vec3f *qs, int nq, int *ids, float *d)
{
  int t = threadIdx.x + blockIdx.x * blockDim.x;
  if (t >= nq) return;
  triangles::FCPResult r;
  r.clear(INFINITY);
  triangles::findClosest(r, bvh, tris, qs[t]);
  ids[t] = r.primID;
  d[t] = r.primID < 0 ? INFINITY : r.sqrDist;
}

__global__ void k_tri_boxes(const Triangle *tris, box3f *boxes, int n)
{
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i < n) boxes[i] = box3f().including(tris[i].a).including(tris[i].b).including(tris[i].c);
}
} // namespace

// ids/d: 6 rows of max(nq, ntq): [0] reference findClosest on the reference's
// SAH tree, [1] on ours; [2] reference wide findClosest on the reference's
// WideBVH<4>, [3] on ours; [4] reference triangles::findClosest kernel on the
// reference's radix tree of the triangles, [5] bq_cubql::triangles::findClosest
// (reference tie rule) on the same tree.  numNodes: SAH ref/ours, wide ref/ours.
extern "C" int ref_shim_compare_more(const float *points, uint32_t n, const float *queries, uint32_t nq,
                                     const int32_t *tris, uint32_t nt, const float *verts, uint32_t nv,
                                     const float *tq, uint32_t ntq, int32_t *ids, float *d, uint32_t *numNodes)
{
  const uint32_t row = nq > ntq ? nq : ntq;
  vec3f *dp, *dq, *dv, *dtq;
  box3f *db, *dtb;
  Triangle *dtri;
  int32_t *dti;
  int *di;
  float *dd;
  cudaMalloc(&dp, 12ull * n);
  cudaMalloc(&dq, 12ull * nq);
  cudaMalloc(&db, 24ull * n);
  cudaMalloc(&dv, 12ull * nv);
  cudaMalloc(&dtq, 12ull * ntq);
  cudaMalloc(&dtb, 24ull * nt);
  cudaMalloc(&dtri, sizeof(Triangle) * (size_t)nt);
  cudaMalloc(&dti, 12ull * nt);
  cudaMalloc(&di, 4ull * row);
  cudaMalloc(&dd, 4ull * row);
  cudaMemcpy(dp, points, 12ull * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dq, queries, 12ull * nq, cudaMemcpyHostToDevice);
  cudaMemcpy(dv, verts, 12ull * nv, cudaMemcpyHostToDevice);
  cudaMemcpy(dtq, tq, 12ull * ntq, cudaMemcpyHostToDevice);
  cudaMemcpy(dti, tris, 12ull * nt, cudaMemcpyHostToDevice);
  std::vector<Triangle> T(nt);
  for (uint32_t i = 0; i < nt; i++) {
    T[i].a = ((const vec3f *)verts)[tris[3 * i]];
    T[i].b = ((const vec3f *)verts)[tris[3 * i + 1]];
    T[i].c = ((const vec3f *)verts)[tris[3 * i + 2]];
  }
  cudaMemcpy(dtri, T.data(), sizeof(Triangle) * (size_t)nt, cudaMemcpyHostToDevice);
  k_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  k_tri_boxes<<<(nt + 127) / 128, 128>>>(dtri, dtb, (int)nt);
  auto fetch = [&](int r, uint32_t cnt) {
    cudaMemcpy(ids + (size_t)r * row, di, 4ull * cnt, cudaMemcpyDeviceToHost);
    cudaMemcpy(d + (size_t)r * row, dd, 4ull * cnt, cudaMemcpyDeviceToHost);
  };
  // SAH: the reference's builder and ours through the shim
  bvh3f sref, sours;
  cuBQL::cuda::sahBuilder(sref, db, n, BuildConfig());
  bq_cubql::cuda::sahBuilder(sours, db, n, BuildConfig(), 0, defaultGpuMemResource());
  numNodes[0] = sref.numNodes;
  numNodes[1] = sours.numNodes;
  k_query<<<(nq + 127) / 128, 128>>>(sref, dp, dq, (int)nq, di, dd);
  fetch(0, nq);
  k_query<<<(nq + 127) / 128, 128>>>(sours, dp, dq, (int)nq, di, dd);
  fetch(1, nq);
  cuBQL::cuda::free(sref);
  bq_cubql::cuda::free(sours, 0, defaultGpuMemResource());
  // WideBVH<float,3,4>: gpuBuilder(WideBVH&) of the reference and ours
  WideBVH<float, 3, 4> wref, wours;
  cuBQL::gpuBuilder(wref, db, n, BuildConfig());
  bq_cubql::gpuBuilder(wours, db, n, BuildConfig(), 0, defaultGpuMemResource());
  numNodes[2] = wref.numNodes;
  numNodes[3] = wours.numNodes;
  k_wide_query<4><<<(nq + 127) / 128, 128>>>(wref, dp, dq, (int)nq, di, dd);
  fetch(2, nq);
  k_wide_query<4><<<(nq + 127) / 128, 128>>>(wours, dp, dq, (int)nq, di, dd);
  fetch(3, nq);
  cuBQL::cuda::free(wref);
  bq_cubql::cuda::free(wours, 0, defaultGpuMemResource());
  // triangles: the reference's kernel and the batched shim call on one tree
  bvh3f tref;
  cuBQL::cuda::radixBuilder(tref, dtb, nt, BuildConfig());
  k_tri_query<<<(ntq + 127) / 128, 128>>>(tref, dtri, dtq, (int)ntq, di, dd);
  fetch(4, ntq);
  bq_cubql::triangles::findClosest(tref, dti, dv, dtq, ntq, di, dd, (vec3f *)nullptr, INFINITY, 0,
                                   BQ_TIES_REFERENCE);
  fetch(5, ntq);
  cuBQL::cuda::free(tref);
  int ok = cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
  cudaFree(dp); cudaFree(dq); cudaFree(db); cudaFree(dv); cudaFree(dtq); cudaFree(dtb); cudaFree(dtri);
  cudaFree(dti); cudaFree(di); cudaFree(dd);
  return ok;
}

extern "C" int ref_shim_compare(const float *points, uint32_t n, const float *queries, uint32_t nq, int32_t *refIds,
                                float *refD, int32_t *ourIds, float *ourD, uint32_t *numNodes)
{
  vec3f *dp, *dq;
  box3f *db;
  int *di;
  float *dd;
  cudaMalloc(&dp, 12ull * n);
  cudaMalloc(&dq, 12ull * nq);
  cudaMalloc(&db, 24ull * n);
  cudaMalloc(&di, 4ull * nq);
  cudaMalloc(&dd, 4ull * nq);
  cudaMemcpy(dp, points, 12ull * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dq, queries, 12ull * nq, cudaMemcpyHostToDevice);
  k_boxes<<<(n + 127) / 128, 128>>>(dp, db, (int)n);
  bvh3f ref, ours;
  cuBQL::cuda::radixBuilder(ref, db, n, BuildConfig());
  bq_cubql::cuda::radixBuilder(ours, db, n, BuildConfig(), 0, defaultGpuMemResource());
  numNodes[0] = ref.numNodes;
  numNodes[1] = ours.numNodes;
  k_query<<<(nq + 127) / 128, 128>>>(ref, dp, dq, (int)nq, di, dd);
  cudaMemcpy(refIds, di, 4ull * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(refD, dd, 4ull * nq, cudaMemcpyDeviceToHost);
  k_query<<<(nq + 127) / 128, 128>>>(ours, dp, dq, (int)nq, di, dd);
  cudaMemcpy(ourIds, di, 4ull * nq, cudaMemcpyDeviceToHost);
  cudaMemcpy(ourD, dd, 4ull * nq, cudaMemcpyDeviceToHost);
  int ok = cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
  cuBQL::cuda::free(ref);
  bq_cubql::cuda::free(ours, 0, defaultGpuMemResource());
  cudaFree(dp); cudaFree(dq); cudaFree(db); cudaFree(di); cudaFree(dd);
  return ok;
}
