// bq_noalloc.cu -- a refit that allocates no device memory.
//
// Who needs it: callers that are not allowed to allocate device memory
// at the moment they refit.  Examples are an application that reserved all
// GPU memory for its own pool up front, a real-time loop where a
// cudaMalloc could stall or fail part-way through a frame, and a framework
// that only permits allocation during its own set-up phase.
// bq_refit_f3 needs two scratch words per node (parent link and arrival
// counter) and takes them from an allocator on every call.  This variant
// takes them from one fixed array in the library's own device memory
// instead, and runs the same range-checked kernels (bq_refit.cuh).
//
// The array (refitScratch below) is a file-scope __device__ variable
// sized for BQ_NOALLOC_REFIT_MAX_NODES nodes, 8 MiB.  This file is its own
// CUDA module, and with lazy module loading (the CUDA runtime's default)
// the module -- and with it the 8 MiB -- is only placed on a device when
// something first needs it there.  A call with numNodes == 0 (the set-up
// call) does exactly that for the current device: it looks the array up
// and loads both kernels, then returns.  Make that call during set-up,
// before any stream capture and before reserving the rest of the GPU's
// memory; from then on the device holds the array until the process exits.
// The address is looked up again on every call (a host-side lookup), so a
// device that was reset and set up again gets the array's new address.
// All calls share the array and each call rewrites it:
// - the links, counters and the error word are cleared by the call itself;
// - two calls that overlap on the GPU (different streams, or different
//   host threads) race on the array and corrupt each other's boxes, so
//   serialise them.
// Nothing here calls cudaMalloc, cudaFree or any allocating routine.
#include "bq_refit.cuh"

namespace bq {
namespace {

// parent links in [0, MAX), arrival counters in [MAX, 2*MAX), the
// range-check word at 2*MAX
constexpr size_t NA_WORDS = 2ull * BQ_NOALLOC_REFIT_MAX_NODES + 64;
static __device__ __align__(256) uint32_t refitScratch[NA_WORDS];

// device address of refitScratch on the current device (loads this
// module there if it is not loaded yet), and both kernels loaded
int scratch_address(uint32_t **out)
{
  void *p = nullptr;
  BQ_CUDA(cudaGetSymbolAddress(&p, refitScratch));
  cudaFuncAttributes fa;
  BQ_CUDA(cudaFuncGetAttributes(&fa, k_refit_init));
  BQ_CUDA(cudaFuncGetAttributes(&fa, k_refit_parents));
  BQ_CUDA(cudaFuncGetAttributes(&fa, k_refit_climb));
  *out = (uint32_t *)p;
  return BQ_OK;
}

} // namespace
} // namespace bq

extern "C" int bq_refit_noalloc_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, bq_stream_t stream)
{
  using namespace bq;
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  const uint32_t nn = bvh->numNodes;
  if (nn > BQ_NOALLOC_REFIT_MAX_NODES)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "tree has " + std::to_string(nn) +
                                                  " nodes; the allocation-free refit handles at most " +
                                                  std::to_string(BQ_NOALLOC_REFIT_MAX_NODES));
  uint32_t *scratch = nullptr;
  BQ_TRY(scratch_address(&scratch));
  if (nn == 0) return BQ_OK;  // the set-up call
  if (!bvh->nodes || !bvh->primIDs || !boxes) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t *parent = scratch, *counter = scratch + BQ_NOALLOC_REFIT_MAX_NODES;
  uint32_t *err = scratch + 2ull * BQ_NOALLOC_REFIT_MAX_NODES;
  launch_refit((Node *)bvh->nodes, nn, bvh->primIDs, bvh->numPrims, boxes, parent, counter, err, s);
  BQ_CUDA(cudaGetLastError());
  // the range-check word, read into host memory (no device allocation)
  uint32_t h = 0;
  BQ_CUDA(cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, s));
  BQ_CUDA(cudaStreamSynchronize(s));
  if (h & DEV_ERR_RANGE)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "malformed tree: a child, prim range or parent chain is out of range");
  return BQ_OK;
}
