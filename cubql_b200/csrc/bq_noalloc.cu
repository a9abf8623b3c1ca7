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
// instead.
//
// The array (refitScratch below) is a file-scope __device__ variable
// sized for BQ_NOALLOC_REFIT_MAX_NODES nodes, 8 MiB.  Every GPU that loads
// the library holds those 8 MiB until the process exits.  Its device
// address is looked up once per device, with that device current, on the
// first call made on that device.  Make that first call before any stream
// capture.  All calls share the array and each call rewrites it:
// - the arrival counters are cleared by the call itself;
// - two calls that overlap on the GPU (different streams, or different
//   host threads) race on the array and corrupt each other's boxes, so
//   serialise them.
// Nothing here calls cudaMalloc, cudaFree or any allocating routine.
#include <mutex>

#include <cuda/atomic>

#include "bq_internal.cuh"

namespace bq {
namespace {

constexpr uint32_t NA_NO_PARENT = 0xffffffffu;

// parent links in [0, MAX), arrival counters in [MAX, 2*MAX)
static __device__ __align__(256) uint32_t refitScratch[2u * BQ_NOALLOC_REFIT_MAX_NODES];

__global__ void k_na_parents(const Node *__restrict__ nodes, uint32_t numNodes, uint32_t *__restrict__ scratch)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes) return;
  uint32_t *parent = scratch, *counter = scratch + BQ_NOALLOC_REFIT_MAX_NODES;
  counter[i] = 0;  // left over from the previous call
  if (i == 0) parent[0] = NA_NO_PARENT;
  if (i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  if (admin_count(a) == 0) {
    const uint64_t off = admin_offset(a);
    if (off + 1 < numNodes) {
      parent[off] = i;
      parent[off + 1] = i;
    }
  }
}

__global__ void k_na_climb(Node *nodes, uint32_t numNodes, const uint32_t *__restrict__ primIDs,
                           const bq_box3f *__restrict__ boxes, uint32_t *scratch)
{
  const uint32_t *parent = scratch;
  uint32_t *counter = scratch + BQ_NOALLOC_REFIT_MAX_NODES;
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes || i == 1) return;
  const uint64_t a = node_admin(nodes[i]);
  const uint32_t cnt = admin_count(a);
  if (cnt == 0) return;
  const uint64_t off = admin_offset(a);
  float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
  for (uint32_t j = 0; j < cnt; j++) {
    const bq_box3f b = boxes[primIDs[off + j]];
    lx = fminf(lx, b.lower[0]); ly = fminf(ly, b.lower[1]); lz = fminf(lz, b.lower[2]);
    hx = fmaxf(hx, b.upper[0]); hy = fmaxf(hy, b.upper[1]); hz = fmaxf(hz, b.upper[2]);
  }
  nodes[i] = make_node(lx, ly, lz, hx, hy, hz, a);
  while (true) {
    const uint32_t p = parent[i];
    if (p == NA_NO_PARENT) return;
    // device-scope release of this node's box / acquire of the sibling's
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> arrived(counter[p]);
    if (arrived.fetch_add(1u, cuda::memory_order_acq_rel) == 0) return;  // the sibling finishes this parent
    const float4 pb = __ldcg(&nodes[p].b);  // from L2: the box half of this word is being written
    const uint64_t pa = ((uint64_t)__float_as_uint(pb.w) << 32) | __float_as_uint(pb.z);
    const uint64_t c0 = admin_offset(pa);
    const Node sib = ldcg_node(nodes + (c0 == i ? c0 + 1 : c0));
    if (c0 == i) {  // union in child order (left, right)
      lx = fminf(lx, sib.a.x); ly = fminf(ly, sib.a.y); lz = fminf(lz, sib.a.z);
      hx = fmaxf(hx, sib.a.w); hy = fmaxf(hy, sib.b.x); hz = fmaxf(hz, sib.b.y);
    } else {
      lx = fminf(sib.a.x, lx); ly = fminf(sib.a.y, ly); lz = fminf(sib.a.z, lz);
      hx = fmaxf(sib.a.w, hx); hy = fmaxf(sib.b.x, hy); hz = fmaxf(sib.b.y, hz);
    }
    nodes[p] = make_node(lx, ly, lz, hx, hy, hz, pa);
    i = p;
  }
}

// device address of refitScratch, looked up once per device
int scratch_address(uint32_t **out)
{
  static std::mutex m;
  static uint32_t *addr[64] = {};
  int dev = 0;
  BQ_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BQ_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> g(m);
  if (!addr[dev]) {
    void *p = nullptr;
    BQ_CUDA(cudaGetSymbolAddress(&p, refitScratch));
    addr[dev] = (uint32_t *)p;
  }
  *out = addr[dev];
  return BQ_OK;
}

} // namespace
} // namespace bq

extern "C" int bq_refit_noalloc_f3(const bq_bvh3f *bvh, const bq_box3f *boxes, bq_stream_t stream)
{
  using namespace bq;
  if (!bvh) return set_error(BQ_ERR_INVALID_ARGUMENT, "bvh is NULL");
  const uint32_t nn = bvh->numNodes;
  if (nn == 0) return BQ_OK;
  if (nn > BQ_NOALLOC_REFIT_MAX_NODES)
    return set_error(BQ_ERR_INVALID_ARGUMENT, "tree has " + std::to_string(nn) +
                                                  " nodes; the allocation-free refit handles at most " +
                                                  std::to_string(BQ_NOALLOC_REFIT_MAX_NODES));
  if (!bvh->nodes || !bvh->primIDs || !boxes) return set_error(BQ_ERR_INVALID_ARGUMENT, "NULL array argument");
  uint32_t *scratch = nullptr;
  BQ_TRY(scratch_address(&scratch));
  cudaStream_t s = (cudaStream_t)stream;
  Node *nodes = (Node *)bvh->nodes;
  k_na_parents<<<div_up(nn, 256), 256, 0, s>>>(nodes, nn, scratch);
  k_na_climb<<<div_up(nn, 128), 128, 0, s>>>(nodes, nn, bvh->primIDs, boxes, scratch);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}
