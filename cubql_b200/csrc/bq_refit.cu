// bq_refit.cu -- bq_refit_f3: bottom-up refit of any BinaryBVH<float,3>
// (kernels in bq_refit.cuh), scratch from the caller's allocator.
//
// Replaces gpuBuilder_impl::refit (cuBQL/builder/cuda/sm_builder.h:677-693).
// The builders call it on trees they made themselves (check = false: no
// wait).  For a caller's tree (check = true) the call reads the kernels'
// range-check word back, so a malformed tree is reported as
// BQ_ERR_INVALID_ARGUMENT; that read waits for the stream, and is skipped
// while the stream is being captured into a graph.
#include "bq_refit.cuh"

namespace bq {

int refit(const bq_bvh3f *bvh, const bq_box3f *boxes, Alloc &al, bool check)
{
  const uint32_t nn = bvh->numNodes;
  if (nn == 0) return BQ_OK;
  TempSet tmp(al);
  uint32_t *scratch = nullptr;
  BQ_TRY(tmp.get(&scratch, 2ull * nn + 1));
  uint32_t *parent = scratch, *counter = scratch + nn, *err = scratch + 2ull * nn;
  {
    ProfScope ps("refit", al.s, 3);
    launch_refit((Node *)bvh->nodes, nn, bvh->primIDs, bvh->numPrims, boxes, parent, counter, err, al.s);
  }
  BQ_CUDA(cudaGetLastError());
  if (!check) return BQ_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  BQ_CUDA(cudaStreamIsCapturing(al.s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return BQ_OK;
  uint32_t h = 0;
  BQ_CUDA(cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, al.s));
  BQ_CUDA(cudaStreamSynchronize(al.s));
  if (h & DEV_ERR_RANGE)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "malformed tree: a child, prim range or parent chain is out of range");
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
