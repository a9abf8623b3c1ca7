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
// answers exactly as on its own tree.
#define CUBQL_GPU_BUILDER_IMPLEMENTATION 1
#include "cuBQL/bvh.h"
#include "cuBQL/builder/cuda/radix.h"
#include "cuBQL/queries/points/findClosest.h"

#include "bq_cubql.hpp"

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
} // namespace

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
