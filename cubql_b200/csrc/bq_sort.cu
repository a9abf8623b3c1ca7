// bq_sort.cu -- onesweep LSD radix sort for (key, u32 value) pairs.
//
// Stands in for cub::DeviceRadixSort::SortPairs / SortKeys at the
// reference's call sites (cuBQL/builder/cuda/radix.h:666-687,
// sm_builder.h:572-580).  Same contract: ascending, stable.
//
// One kernel launch per 8-bit digit.  Each 256-thread block takes the next
// tile of TILE = 256*ITEMS pairs (tile order from an atomic counter, so a
// tile only ever waits on tiles that already started):
//   1. loads its keys (warp-contiguous, coalesced),
//   2. ranks them stably with __match_any_sync: per warp, per round of 32
//      consecutive keys, peers with the same digit share one update of a
//      warp-private digit histogram in shared memory,
//   3. publishes its 256 digit counts and resolves its global digit
//      offsets by decoupled look-back over earlier tiles (one thread per
//      digit; every wait is bounded and aborts the whole pass on timeout),
//   4. reorders keys (then values) through shared memory so the global
//      writes are runs of consecutive addresses per digit.
// The per-pass digit histograms come from one counting pass over all
// digits (or from the producer of the keys, see *_prehist).
#include <algorithm>

#include "bq_internal.cuh"

namespace bq {
namespace {

constexpr int SORT_BLOCK = 256;
constexpr int SORT_WARPS = SORT_BLOCK / 32;
constexpr uint32_t ST_AGG = 1u << 30;
constexpr uint32_t ST_INC = 2u << 30;
constexpr uint32_t ST_VAL = (1u << 30) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 22;  // x >= 64 ns sleep => ~0.3 s per wait at most

__device__ __forceinline__ uint32_t lanemask_lt()
{
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p)
{
  return *(const volatile uint32_t *)p;
}

template <typename KeyT>
__device__ __forceinline__ uint32_t digit_of(KeyT k, int shift)
{
  return (uint32_t)(k >> shift) & 0xffu;
}

// exclusive scan of v over the 256 threads of the block; returns the
// exclusive prefix, writes the total to *total (all threads)
__device__ __forceinline__ uint32_t block_excl_scan_256(uint32_t v, uint32_t *warpSums, uint32_t *total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < SORT_WARPS ? warpSums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < SORT_WARPS) warpSums[lane] = w;  // inclusive
  }
  __syncthreads();
  uint32_t warpBase = warp ? warpSums[warp - 1] : 0;
  *total = warpSums[SORT_WARPS - 1];
  __syncthreads();
  return warpBase + x - v;
}

// ------------------------------------------------------------------
// counting pass: histograms of every digit position at once
// ------------------------------------------------------------------
template <typename KeyT>
__global__ void __launch_bounds__(256) k_histogram(const KeyT *__restrict__ keys, uint32_t nHost,
                                                   const uint32_t *nDev, int beginBit, int numPasses,
                                                   uint32_t *__restrict__ hist)
{
  const uint32_t n = nDev ? *nDev : nHost;
  extern __shared__ uint32_t sh[];  // numPasses * 256
  for (int i = threadIdx.x; i < numPasses * 256; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    KeyT k = keys[i];
    for (int p = 0; p < numPasses; p++) atomicAdd(&sh[p * 256 + digit_of(k, beginBit + 8 * p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < numPasses * 256; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// ------------------------------------------------------------------
// one onesweep digit pass
// ------------------------------------------------------------------
struct PassCtl {
  uint32_t *status;    // numTiles * 256 look-back words for this pass
  uint32_t *tileCtr;   // dynamic tile counter for this pass
  uint32_t *abort;     // shared abort flag (all passes)
  uint32_t *err;       // caller's device error word
  const uint32_t *hist;// 256 counters of this pass's digit
};

template <typename KeyT, int ITEMS>
__global__ void __launch_bounds__(SORT_BLOCK, 4) k_onesweep(const KeyT *__restrict__ keysIn, KeyT *__restrict__ keysOut,
                                                            const uint32_t *__restrict__ valsIn,
                                                            uint32_t *__restrict__ valsOut, uint32_t nHost,
                                                            const uint32_t *nDev, int shift, PassCtl ctl)
{
  const uint32_t n = nDev ? *nDev : nHost;
  constexpr int TILE = SORT_BLOCK * ITEMS;
  constexpr int WARP_ITEMS = 32 * ITEMS;
  // dynamic shared memory: keys [TILE], then values [TILE]; the per-warp
  // digit histograms live in the value region until the local positions
  // are known (they are dead before the first value is stored)
  extern __shared__ __align__(16) unsigned char smem[];
  KeyT *sKeys = (KeyT *)smem;
  uint32_t *sVals = (uint32_t *)(smem + sizeof(KeyT) * TILE);
  uint32_t *sWarpHist = sVals;  // SORT_WARPS * 257 <= TILE
  __shared__ uint32_t sTileStart[256];
  __shared__ uint32_t sGlobalBase[256];
  __shared__ uint32_t sWarpSums[SORT_WARPS];
  __shared__ uint32_t sTile;
  __shared__ uint32_t sBad;
  static_assert(SORT_WARPS * 257 <= TILE, "histograms must fit in the value region");

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    sTile = atomicAdd(ctl.tileCtr, 1u);
    sBad = 0;
  }
  for (int i = threadIdx.x; i < SORT_WARPS * 257; i += SORT_BLOCK) sWarpHist[i] = 0;
  __syncthreads();
  const uint32_t tile = sTile;
  const uint64_t warpBase = (uint64_t)tile * TILE + (uint64_t)warp * WARP_ITEMS;

  // 1. keys (warp-contiguous sub-tiles, coalesced)
  KeyT key[ITEMS];
#pragma unroll
  for (int r = 0; r < ITEMS; r++) {
    const uint64_t idx = warpBase + (uint64_t)r * 32 + lane;
    key[r] = idx < n ? keysIn[idx] : (KeyT)0;
  }

  // 2. stable ranking inside each warp
  uint32_t *wh = sWarpHist + warp * 257;
  const uint32_t ltMask = lanemask_lt();
  uint32_t pos[ITEMS];  // rank within warp and digit, later the tile-local position
#pragma unroll
  for (int r = 0; r < ITEMS; r++) {
    const bool valid = warpBase + (uint64_t)r * 32 + lane < n;
    const uint32_t d = valid ? digit_of(key[r], shift) : 256u;  // 256: never written
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t base = wh[d];
    __syncwarp();
    if ((peers & ~(ltMask | (1u << lane))) == 0) wh[d] = base + __popc(peers);  // highest lane of the group
    __syncwarp();
    pos[r] = base + __popc(peers & ltMask);
  }
  __syncthreads();

  // per digit (thread d): warp-exclusive offsets and tile totals
  const int d = threadIdx.x;
  uint32_t cnt = 0;
#pragma unroll
  for (int w = 0; w < SORT_WARPS; w++) {
    const uint32_t c = sWarpHist[w * 257 + d];
    sWarpHist[w * 257 + d] = cnt;
    cnt += c;
  }
  uint32_t tileTotal;
  sTileStart[d] = block_excl_scan_256(cnt, sWarpSums, &tileTotal);
  uint32_t histTotal;
  const uint32_t gStart = block_excl_scan_256(ctl.hist[d], sWarpSums, &histTotal);

  // 3. decoupled look-back (thread d owns digit d)
  uint32_t *st = ctl.status;
  if (tile == 0) {
    __stcg(&st[d], ST_INC | cnt);
    sGlobalBase[d] = gStart;
  } else {
    __stcg(&st[(uint64_t)tile * 256 + d], ST_AGG | cnt);
    uint32_t excl = 0;
    int64_t j = (int64_t)tile - 1;
    bool bad = false;
    while (j >= 0) {
      uint32_t v = ld_volatile(&st[(uint64_t)j * 256 + d]);
      uint32_t spins = 0;
      while ((v & ~ST_VAL) == 0) {
        if (++spins > SPIN_LIMIT || ld_volatile(ctl.abort)) {
          bad = true;
          break;
        }
        __nanosleep(64);
        v = ld_volatile(&st[(uint64_t)j * 256 + d]);
      }
      if (bad) break;
      excl += v & ST_VAL;
      if (v & ST_INC) break;
      j--;
    }
    if (bad) {
      atomicOr(ctl.abort, 1u);
      atomicOr(ctl.err, DEV_ERR_TIMEOUT);
      sBad = 1;
    } else {
      __stcg(&st[(uint64_t)tile * 256 + d], ST_INC | (excl + cnt));
    }
    sGlobalBase[d] = gStart + excl;
  }
  __syncthreads();
  if (sBad) return;  // a wait timed out: leave the output untouched, report

  // 4. tile-local positions; then keys and values through shared memory
#pragma unroll
  for (int r = 0; r < ITEMS; r++) {
    const bool valid = warpBase + (uint64_t)r * 32 + lane < n;
    const uint32_t dd = digit_of(key[r], shift);
    pos[r] = valid ? sTileStart[dd] + sWarpHist[warp * 257 + dd] + pos[r] : 0xffffffffu;
  }
  __syncthreads();  // histograms dead: the value region may be written now
#pragma unroll
  for (int r = 0; r < ITEMS; r++)
    if (pos[r] != 0xffffffffu) sKeys[pos[r]] = key[r];
  uint32_t val[ITEMS];
#pragma unroll
  for (int r = 0; r < ITEMS; r++) {
    const uint64_t idx = warpBase + (uint64_t)r * 32 + lane;
    val[r] = pos[r] != 0xffffffffu ? valsIn[idx] : 0u;
  }
#pragma unroll
  for (int r = 0; r < ITEMS; r++)
    if (pos[r] != 0xffffffffu) sVals[pos[r]] = val[r];
  __syncthreads();
  // 5. scatter: consecutive tile positions of one digit go to consecutive
  // global positions
#pragma unroll 4
  for (int r = 0; r < ITEMS; r++) {
    const uint32_t p = threadIdx.x + r * SORT_BLOCK;
    if (p < tileTotal) {
      const KeyT k = sKeys[p];
      const uint32_t dd = digit_of(k, shift);
      const uint32_t g = sGlobalBase[dd] + (p - sTileStart[dd]);
      if (g < n) {
        keysOut[g] = k;
        valsOut[g] = sVals[p];
      } else {
        atomicOr(ctl.err, DEV_ERR_RANGE);
      }
    }
  }
}

template <typename KeyT>
int onesweep_impl(KeyT *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit, int endBit,
                  const uint32_t *preHist, int *outSel, uint32_t *dErr, Alloc &al)
{
  constexpr int ITEMS = 16;
  constexpr int TILE = SORT_BLOCK * ITEMS;
  *outSel = 0;
  if ((nMax <= 1 && !nDev) || nMax == 0 || endBit <= beginBit) return BQ_OK;
  const int numPasses = (endBit - beginBit + 7) / 8;
  const int numTiles = div_up(nMax, TILE);
  TempSet tmp(al);
  uint32_t *hist = nullptr, *ctl = nullptr;
  // ctl layout: [status: numPasses*numTiles*256][tileCtr: numPasses][abort: 1]
  const size_t statusWords = (size_t)numPasses * numTiles * 256;
  BQ_TRY(tmp.get(&ctl, statusWords + numPasses + 1));
  BQ_CUDA(cudaMemsetAsync(ctl, 0, sizeof(uint32_t) * (statusWords + numPasses + 1), al.s));
  if (preHist) {
    hist = const_cast<uint32_t *>(preHist);
  } else {
    BQ_TRY(tmp.get(&hist, (size_t)numPasses * 256));
    BQ_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * numPasses * 256, al.s));
    int grid = std::max(1, std::min(div_up(nMax, 256 * 8), num_sms() * 8));
    ProfScope ps(sizeof(KeyT) == 8 ? "sort.histogram64" : "sort.histogram32", al.s);
    k_histogram<KeyT><<<grid, 256, sizeof(uint32_t) * numPasses * 256, al.s>>>(keys[0], nMax, nDev, beginBit,
                                                                                numPasses, hist);
    BQ_CUDA(cudaGetLastError());
  }
  const size_t smemBytes = (sizeof(KeyT) + sizeof(uint32_t)) * TILE;
  BQ_CUDA(cudaFuncSetAttribute(k_onesweep<KeyT, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes));
  int sel = 0;
  for (int p = 0; p < numPasses; p++) {
    PassCtl c;
    c.status = ctl + (size_t)p * numTiles * 256;
    c.tileCtr = ctl + statusWords + p;
    c.abort = ctl + statusWords + numPasses;
    c.err = dErr;
    c.hist = hist + p * 256;
    ProfScope ps(sizeof(KeyT) == 8 ? "sort.onesweep64" : "sort.onesweep32", al.s);
    k_onesweep<KeyT, ITEMS><<<numTiles, SORT_BLOCK, smemBytes, al.s>>>(keys[sel], keys[sel ^ 1], vals[sel],
                                                                       vals[sel ^ 1], nMax, nDev, beginBit + 8 * p, c);
    BQ_CUDA(cudaGetLastError());
    sel ^= 1;
  }
  *outSel = sel;
  return BQ_OK;
}

} // namespace

int onesweep_sort_u64(uint64_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al)
{
  return onesweep_impl<uint64_t>(keys, vals, nMax, nDev, beginBit, endBit, dHist, outSel, dErr, al);
}

int onesweep_sort_u32(uint32_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al)
{
  return onesweep_impl<uint32_t>(keys, vals, nMax, nDev, beginBit, endBit, dHist, outSel, dErr, al);
}

} // namespace bq
