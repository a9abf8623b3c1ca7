// bq_internal.cuh -- shared device/host helpers of libbq (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <utility>

#include "../../include/bq.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libbq is written for sm_100a (B200) only"
#endif

namespace bq {

// ------------------------------------------------------------------
// errors: every entry point returns a status and records a message
// ------------------------------------------------------------------
int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);

#define BQ_CUDA(x)                                  \
  do {                                              \
    cudaError_t e_ = (x);                           \
    if (e_ != cudaSuccess) return ::bq::cuda_error(e_, #x); \
  } while (0)

#define BQ_TRY(x)                 \
  do {                            \
    int s_ = (x);                 \
    if (s_ != BQ_OK) return s_;   \
  } while (0)

// device-side error bits (or-ed into a per-call status word)
enum : uint32_t {
  DEV_ERR_TIMEOUT = 1u,        // a bounded spin wait gave up
  DEV_ERR_STACK = 2u,          // a deep-stack fallback query still overflowed
  DEV_ERR_RANGE = 4u,          // an index fell outside its buffer (skipped)
};

// ------------------------------------------------------------------
// allocation through the caller's bq_allocator (or cudaMallocAsync)
// ------------------------------------------------------------------
struct Alloc {
  const bq_allocator *a;
  cudaStream_t s;
  int malloc_bytes(void **p, size_t bytes);
  int free_bytes(void *p);
  // temporaries: from the caller's allocator, or from the pool when it
  // asks for that (bq_allocator::scratchFromPool)
  int scratch_malloc(void **p, size_t bytes);
  int scratch_free(void *p);
  template <typename T>
  int get(T **p, size_t count) { return malloc_bytes((void **)p, sizeof(T) * (count ? count : 1)); }
};

// Carves one allocation into 256-byte aligned pieces (first pass: sizing
// with base == nullptr; second pass: the pointers)
struct Carver {
  char *base;
  size_t off = 0;
  explicit Carver(void *b) : base((char *)b) {}
  template <typename T>
  void take(T **p, size_t count)
  {
    off = (off + 255) & ~(size_t)255;
    *p = base ? (T *)(base + off) : nullptr;
    off += sizeof(T) * (count ? count : 1);
  }
};

// RAII list of temporaries freed (stream-ordered) at scope exit
struct TempSet {
  Alloc &al;
  void *ptrs[32];
  int n = 0;
  explicit TempSet(Alloc &a) : al(a) {}
  template <typename T>
  int get(T **p, size_t count)
  {
    int s = al.scratch_malloc((void **)p, sizeof(T) * (count ? count : 1));
    if (s == BQ_OK) ptrs[n++] = (void *)*p;
    return s;
  }
  ~TempSet()
  {
    for (int i = n - 1; i >= 0; i--) al.scratch_free(ptrs[i]);
  }
};

// ------------------------------------------------------------------
// node layout: BinaryBVH<float,3>::Node as two 16-byte halves
//   a = lower.x lower.y lower.z upper.x
//   b = upper.y upper.z admin.lo admin.hi
// ------------------------------------------------------------------
struct __align__(16) Node {
  float4 a, b;
};
static_assert(sizeof(Node) == 32, "node size");
static_assert(sizeof(bq_node3f) == 32, "C node size");
static_assert(sizeof(bq_box3f) == 24, "C box size");

__host__ __device__ inline uint64_t make_admin(uint64_t offset, uint32_t count)
{
  return offset | ((uint64_t)count << 48);
}

__device__ __forceinline__ uint64_t node_admin(const Node &n)
{
  return ((uint64_t)__float_as_uint(n.b.w) << 32) | __float_as_uint(n.b.z);
}
__device__ __forceinline__ uint32_t admin_count(uint64_t a) { return (uint32_t)(a >> 48); }
__device__ __forceinline__ uint64_t admin_offset(uint64_t a) { return a & 0xFFFFFFFFFFFFull; }

__device__ __forceinline__ Node make_node(float lx, float ly, float lz, float hx, float hy, float hz, uint64_t admin)
{
  Node n;
  n.a = make_float4(lx, ly, lz, hx);
  n.b = make_float4(hy, hz, __uint_as_float((uint32_t)admin), __uint_as_float((uint32_t)(admin >> 32)));
  return n;
}

// read-only, L1-cached 32-byte node load (two 16-byte vector loads)
__device__ __forceinline__ Node ldg_node(const Node *p)
{
  Node n;
  n.a = __ldg(&p->a);
  n.b = __ldg(&p->b);
  return n;
}

// L2-only load (for data written by other blocks of the same kernel)
__device__ __forceinline__ Node ldcg_node(const Node *p)
{
  Node n;
  n.a = __ldcg(&p->a);
  n.b = __ldcg(&p->b);
  return n;
}

// L2 eviction priority (createpolicy): a kernel that streams data it
// touches once (evict_first) past data it reads at random and may hit
// again keeps more of the latter in L2
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// read-only load with an L2 policy
__device__ __forceinline__ uint32_t ldg_u32_policy(const uint32_t *p, uint64_t pol)
{
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
// 32-byte node store with an L2 policy (two 16-byte stores)
__device__ __forceinline__ void st_node_policy(Node *p, const Node &n, uint64_t pol)
{
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(&p->a), "f"(n.a.x), "f"(n.a.y),
               "f"(n.a.z), "f"(n.a.w), "l"(pol)
               : "memory");
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(&p->b), "f"(n.b.x), "f"(n.b.y),
               "f"(n.b.z), "f"(n.b.w), "l"(pol)
               : "memory");
}

// ------------------------------------------------------------------
// order-preserving float <-> int32 (min/max over encoded ints equals a
// total-order min/max over the floats; -0 < +0)
// ------------------------------------------------------------------
__host__ __device__ __forceinline__ int32_t enc_f(float f)
{
#ifdef __CUDA_ARCH__
  int32_t b = __float_as_int(f);
#else
  int32_t b;
  memcpy(&b, &f, 4);
#endif
  return (b & (int32_t)0x80000000) ? (b ^ 0x7fffffff) : b;
}
__host__ __device__ __forceinline__ float dec_f(int32_t b)
{
  b = (b & (int32_t)0x80000000) ? (b ^ 0x7fffffff) : b;
#ifdef __CUDA_ARCH__
  return __int_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

// Block-wide min/max of encoded coordinates, merged into lohi[0..2] (min)
// and lohi[3..5] (max) with one atomic per block and component.  Every
// thread of the block (BLOCK threads, full warps) must call it.
template <int BLOCK>
__device__ __forceinline__ void block_merge_bounds(const int32_t lo[3], const int32_t hi[3], int32_t *lohi)
{
  __shared__ int32_t sRed[6][BLOCK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int32_t mn = __reduce_min_sync(0xffffffffu, lo[d]);
    const int32_t mx = __reduce_max_sync(0xffffffffu, hi[d]);
    if (lane == 0) { sRed[d][warp] = mn; sRed[3 + d][warp] = mx; }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const bool isMin = threadIdx.x < 3;
    int32_t v = isMin ? INT_MAX : INT_MIN;
    for (int w = 0; w < BLOCK / 32; w++) v = isMin ? min(v, sRed[threadIdx.x][w]) : max(v, sRed[threadIdx.x][w]);
    if (isMin && v != INT_MAX) atomicMin(&lohi[threadIdx.x], v);
    if (!isMin && v != INT_MIN) atomicMax(&lohi[threadIdx.x], v);
  }
}

// ------------------------------------------------------------------
// squared distances with the FMA shapes the reference's device code
// compiles to (pinned against the reference kernels on B200):
//   fSqrDistance_rd(vec3f,vec3f) = x*x+y*y+z*z
//     (cuBQL/math/conservativeDistances.h:60-100)
//   shrinkingRadiusQuery::fSqrDistance_rd(vec3f,box3f) = dot(v,v)
//     (cuBQL/traversal/shrinkingRadiusQuery.h:253-259, vec.h:459-466)
// Written with explicit intrinsics so surrounding code cannot change
// the contraction.
// ------------------------------------------------------------------
__device__ __forceinline__ float sqr_pp(float px, float py, float pz, float qx, float qy, float qz)
{
  const float x = __fsub_rn(px, qx), y = __fsub_rn(py, qy), z = __fsub_rn(pz, qz);
  return __fmaf_rn(z, z, __fmaf_rn(x, x, __fmul_rn(y, y)));
}

__device__ __forceinline__ float sqr_pbox(float qx, float qy, float qz, float lx, float ly, float lz, float hx,
                                          float hy, float hz)
{
  const float vx = __fsub_rn(fminf(fmaxf(qx, lx), hx), qx);
  const float vy = __fsub_rn(fminf(fmaxf(qy, ly), hy), qy);
  const float vz = __fsub_rn(fminf(fmaxf(qz, lz), hz), qz);
  return __fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx)));
}

// ------------------------------------------------------------------
// Morton helpers: 21 bits spread to every third bit of a u64
// ------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t spread21(uint64_t x)
{
  x &= 0x1fffffull;
  x = (x | (x << 32)) & 0x001f00000000ffffull;
  x = (x | (x << 16)) & 0x001f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// 10 bits spread to every third bit of a u32
__host__ __device__ __forceinline__ uint32_t spread10(uint32_t x)
{
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// quantised cell as in the reference's Quantizer<float,D>::quantize
// (cuBQL/builder/cuda/radix.h:55-62): float->uint truncation
// (saturating, NaN -> 0), clamped to 2^bits - 1
__device__ __forceinline__ uint32_t quant_cell(float c, float bias, float scale, uint32_t maxCell)
{
  const float f = __fmul_rn(__fsub_rn(c, bias), scale);
  return min(__float2uint_rz(f), maxCell);
}

// per-build summary of the Morton build: the centroid bounds, valid count
// and quantizer (written by block 0 of the key pass) and the device error
// word (zeroed by the bounds pass)
struct BuildState {
  int32_t cbLo[3], cbHi[3];  // encoded centroid bounds of valid prims
  uint32_t numValid;
  float bias[3];
  float scale;
  uint32_t err;               // DEV_ERR_* bits
};

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

int num_sms();
// a pinned host buffer of at least `bytes`, one per host thread (reused by
// every call of that thread; nullptr if pinned memory cannot be had): the
// builders' read-backs of their device counters land here directly instead
// of being staged through pageable memory
void *host_readback_buffer(size_t bytes);

// ------------------------------------------------------------------
// phase profiler (the counterpart of the reference's CUBQL_PROFILE,
// cuBQL/builder/cuda/sm_builder.h:24-66): when enabled, CUDA events
// bracket each named phase on the call's stream; prof_flush() (after the
// stream synchronised) turns them into per-name launch counts and times.
// Off by default; costs one branch per phase when off.
// ------------------------------------------------------------------
// ------------------------------------------------------------------
// programmatic dependent launch (sm_90 and later): a kernel launched with
// launch_pdl may be scheduled as soon as the previous kernel on the stream
// has let its blocks finish, before that grid has fully completed; it
// must call griddep_wait() before it touches any memory the previous
// kernels write or read.  griddep_wait() returns at once in a kernel
// launched the ordinary way, so a kernel that calls it first thing may be
// launched either way.
// ------------------------------------------------------------------
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

bool prof_enabled();
void prof_record(const char *name, cudaStream_t s, bool begin, int launches);
void prof_flush();
struct ProfScope {
  const char *name;
  cudaStream_t s;
  int launches;
  bool on;
  ProfScope(const char *n, cudaStream_t st, int nLaunches = 1) : name(n), s(st), launches(nLaunches), on(prof_enabled())
  {
    if (on) prof_record(name, s, true, launches);
  }
  ~ProfScope()
  {
    if (on) prof_record(name, s, false, launches);
  }
};

// ------------------------------------------------------------------
// one-block scans of short per-level arrays kept in shared memory (the
// spatial-median and SAH level loops)
// ------------------------------------------------------------------
constexpr int BQ_SCAN_THREADS = 1024;
constexpr uint32_t BQ_SCAN_SMEM_MAX = 56u * 1024u;  // longest array such a scan keeps in shared memory

// Exclusive scan of s[0 .. L) in place by one block of BQ_SCAN_THREADS
// threads (each a contiguous segment); returns the total.  sWarp: 33 words.
__device__ __forceinline__ uint32_t block_scan_smem(uint32_t *s, uint32_t L, uint32_t *sWarp)
{
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t per = (L + BQ_SCAN_THREADS - 1) / BQ_SCAN_THREADS;
  const uint32_t b = min(t * per, L), e = min(b + per, L);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; i++) sum += s[i];
  uint32_t x = sum;  // inclusive scan over the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if ((int)lane >= o) x += y;
  }
  if (lane == 31) sWarp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = sWarp[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if ((int)lane >= o) wi += y;
    }
    sWarp[lane] = wi - w;
    if (lane == 31) sWarp[32] = wi;
  }
  __syncthreads();
  uint32_t run = sWarp[warp] + x - sum;
  for (uint32_t i = b; i < e; i++) {
    const uint32_t v = s[i];
    s[i] = run;
    run += v;
  }
  const uint32_t total = sWarp[32];
  __syncthreads();
  return total;
}

// ------------------------------------------------------------------
// onesweep LSD radix sort (bq_sort.cu)
// ------------------------------------------------------------------
// Sorts (key, value) pairs by bits [beginBit, endBit) of the key, stably.
// keys/vals are double buffers: input in [0], result in [*outSel].
// The element count is nDev[0] when nDev is given (nMax bounds it),
// else nMax.  dHist (optional) holds the per-pass 256-bin digit
// histograms, already counted by the producer of the keys.
// ctlWs (optional): onesweep_ctl_words(nMax, beginBit, endBit) words of
// device memory, zeroed by the caller, that the sort uses for its
// look-back state instead of allocating them.
int onesweep_sort_u64(uint64_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al,
                      uint32_t *ctlWs = nullptr);
size_t onesweep_ctl_words(uint32_t nMax, int beginBit, int endBit);
int onesweep_sort_u32(uint32_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al);

// exclusive scan of u32 values (reduce-then-scan, no waits); total -> *dTotal
int exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint32_t nMax, const uint32_t *nDev, uint32_t *dTotal,
                       Alloc &al);

} // namespace bq
