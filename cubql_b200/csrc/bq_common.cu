// bq_common.cu -- error reporting, allocation and a device exclusive scan.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <string>
#include <vector>

#include "bq_internal.cuh"

namespace bq {

static thread_local std::string g_lastError;

int set_error(int code, const std::string &msg)
{
  g_lastError = msg;
  return code;
}

int cuda_error(cudaError_t e, const char *what)
{
  return set_error(BQ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int Alloc::malloc_bytes(void **p, size_t bytes)
{
  *p = nullptr;
  if (a && a->malloc) {
    if (a->malloc(a->ctx, p, bytes, (bq_stream_t)s) != 0 || !*p)
      return set_error(BQ_ERR_ALLOC, "allocator failed to provide " + std::to_string(bytes) + " bytes");
    return BQ_OK;
  }
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(BQ_ERR_ALLOC, std::string("cudaMallocAsync(") + std::to_string(bytes) +
                                       " bytes): " + cudaGetErrorString(e));
  }
  return BQ_OK;
}

int Alloc::free_bytes(void *p)
{
  if (!p) return BQ_OK;
  if (a && a->free) return a->free(a->ctx, p, (bq_stream_t)s) == 0 ? BQ_OK : set_error(BQ_ERR_ALLOC, "free failed");
  cudaError_t e = cudaFreeAsync(p, s);
  return e == cudaSuccess ? BQ_OK : cuda_error(e, "cudaFreeAsync");
}

int Alloc::scratch_malloc(void **p, size_t bytes)
{
  if (a && a->scratchFromPool) {
    Alloc pool{nullptr, s};
    return pool.malloc_bytes(p, bytes);
  }
  return malloc_bytes(p, bytes);
}

int Alloc::scratch_free(void *p)
{
  if (a && a->scratchFromPool) {
    Alloc pool{nullptr, s};
    return pool.free_bytes(p);
  }
  return free_bytes(p);
}

void *host_readback_buffer(size_t bytes)
{
  struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    ~Buf()
    {
      if (p) cudaFreeHost(p);
    }
  };
  static thread_local Buf b;
  if (bytes > b.cap) {
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
    void *q = nullptr;
    if (cudaMallocHost(&q, std::max(bytes, (size_t)256)) != cudaSuccess) {
      cudaGetLastError();  // not sticky: clear it
      return nullptr;
    }
    b.p = q;
    b.cap = std::max(bytes, (size_t)256);
  }
  return b.p;
}

int num_sms()
{
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

// ------------------------------------------------------------------
// exclusive scan of u32: per-block sums -> scan of block sums (one
// block, looping) -> per-block scan plus offset.  No inter-block waits.
// ------------------------------------------------------------------
namespace {
constexpr int SCAN_BLOCK = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ uint32_t warp_incl(uint32_t x)
{
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// block-wide exclusive scan of one value per thread (blockDim = 256)
__device__ __forceinline__ uint32_t block_excl(uint32_t v, uint32_t *sh, uint32_t *total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = warp_incl(v);
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < 8 ? sh[lane] : 0;
    w = warp_incl(w);
    if (lane < 8) sh[lane] = w;
  }
  __syncthreads();
  uint32_t base = warp ? sh[warp - 1] : 0;
  *total = sh[7];
  __syncthreads();
  return base + x - v;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const uint32_t *in, uint32_t nMax, const uint32_t *nDev,
                                                            uint32_t *blockSums)
{
  griddep_wait();
  __shared__ uint32_t sh[8];
  const uint32_t n = nDev ? min(*nDev, nMax) : nMax;  // never past the buffers
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    uint64_t idx = base + (uint64_t)i * SCAN_BLOCK + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  uint32_t total;
  block_excl(s, sh, &total);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_blocks(uint32_t *blockSums, int numBlocks, uint32_t *dTotal)
{
  griddep_wait();
  __shared__ uint32_t sh[8];
  uint32_t carry = 0;
  for (int b0 = 0; b0 < numBlocks; b0 += SCAN_BLOCK) {
    int i = b0 + threadIdx.x;
    uint32_t v = i < numBlocks ? blockSums[i] : 0;
    uint32_t total;
    uint32_t ex = block_excl(v, sh, &total);
    if (i < numBlocks) blockSums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0 && dTotal) *dTotal = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_final(const uint32_t *in, uint32_t *out, uint32_t nMax,
                                                           const uint32_t *nDev, const uint32_t *blockOffsets)
{
  griddep_wait();
  __shared__ uint32_t sh[8];
  const uint32_t n = nDev ? min(*nDev, nMax) : nMax;  // never past the buffers
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    uint64_t idx = base + i;
    v[i] = idx < n ? in[idx] : 0;
    s += v[i];
  }
  uint32_t total;
  uint32_t run = block_excl(s, sh, &total) + blockOffsets[blockIdx.x];
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    uint64_t idx = base + i;
    if (idx < n) out[idx] = run;
    run += v[i];
  }
}
} // namespace

int exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint32_t nMax, const uint32_t *nDev, uint32_t *dTotal,
                       Alloc &al)
{
  if (nMax == 0) {
    if (dTotal) BQ_CUDA(cudaMemsetAsync(dTotal, 0, 4, al.s));
    return BQ_OK;
  }
  // k_scan_reduce strides by SCAN_BLOCK within a tile while k_scan_final
  // takes SCAN_ITEMS consecutive items per thread: both cover exactly the
  // same SCAN_TILE-element range per block, so the block sums agree.
  const int numBlocks = div_up(nMax, SCAN_TILE);
  TempSet tmp(al);
  uint32_t *sums = nullptr;
  BQ_TRY(tmp.get(&sums, numBlocks));
  launch_pdl(k_scan_reduce, dim3(numBlocks), dim3(SCAN_BLOCK), 0, al.s, in, nMax, nDev, sums);
  launch_pdl(k_scan_blocks, dim3(1), dim3(SCAN_BLOCK), 0, al.s, sums, numBlocks, dTotal);
  launch_pdl(k_scan_final, dim3(numBlocks), dim3(SCAN_BLOCK), 0, al.s, in, out, nMax, nDev, sums);
  BQ_CUDA(cudaGetLastError());
  return BQ_OK;
}

// ------------------------------------------------------------------
// phase profiler
// ------------------------------------------------------------------
namespace {
std::atomic<int> g_profOn{0};
struct Pending {
  const char *name;
  cudaEvent_t e0, e1;
  int launches;
};
struct ProfTotals {
  std::string name;
  uint64_t launches = 0, calls = 0;
  double ms = 0.0;
};
thread_local std::vector<Pending> t_pending;
thread_local std::vector<ProfTotals> t_totals;
thread_local std::vector<cudaEvent_t> t_eventPool;

cudaEvent_t get_event()
{
  if (!t_eventPool.empty()) {
    cudaEvent_t e = t_eventPool.back();
    t_eventPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
} // namespace

bool prof_enabled() { return g_profOn.load(std::memory_order_relaxed) != 0; }

void prof_record(const char *name, cudaStream_t s, bool begin, int launches)
{
  if (begin) {
    Pending p{name, get_event(), nullptr, launches};
    cudaEventRecord(p.e0, s);
    t_pending.push_back(p);
    return;
  }
  for (auto it = t_pending.rbegin(); it != t_pending.rend(); ++it) {
    if (it->name == name && it->e1 == nullptr) {
      it->e1 = get_event();
      cudaEventRecord(it->e1, s);
      return;
    }
  }
}

void prof_flush()
{
  for (auto &p : t_pending) {
    if (!p.e1) continue;
    float ms = 0.f;
    cudaEventSynchronize(p.e1);
    cudaEventElapsedTime(&ms, p.e0, p.e1);
    ProfTotals *tot = nullptr;
    for (auto &t : t_totals)
      if (t.name == p.name) tot = &t;
    if (!tot) {
      t_totals.push_back(ProfTotals{p.name});
      tot = &t_totals.back();
    }
    tot->launches += p.launches;
    tot->calls += 1;
    tot->ms += ms;
    t_eventPool.push_back(p.e0);
    t_eventPool.push_back(p.e1);
  }
  std::vector<Pending> keep;
  for (auto &p : t_pending)
    if (!p.e1) keep.push_back(p);
  t_pending.swap(keep);
}

} // namespace bq

extern "C" {

int bq_profile_enable(int on)
{
  bq::g_profOn.store(on ? 1 : 0);
  return BQ_OK;
}

int bq_profile_reset(void)
{
  bq::prof_flush();
  bq::t_totals.clear();
  return BQ_OK;
}

int bq_profile_count(void)
{
  bq::prof_flush();
  return (int)bq::t_totals.size();
}

int bq_profile_entry(int i, const char **name, uint64_t *launches, double *ms)
{
  bq::prof_flush();
  if (i < 0 || i >= (int)bq::t_totals.size()) return bq::set_error(BQ_ERR_INVALID_ARGUMENT, "profile index");
  *name = bq::t_totals[i].name.c_str();
  *launches = bq::t_totals[i].launches;
  *ms = bq::t_totals[i].ms;
  return BQ_OK;
}

const char *bq_last_error_string(void) { return bq::g_lastError.c_str(); }

int bq_version(void) { return BQ_VERSION; }

} // extern "C"
