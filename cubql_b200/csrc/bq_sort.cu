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
//   2. ranks them stably: per warp, per round of 32 consecutive keys, the
//      lanes holding the same digit (found with __match_any_sync, or with
//      nine ballots when the warp's first round shows many distinct digits:
//      match-any gets slower the more groups a round has) share one update
//      of a warp-private digit histogram in shared memory; each warp runs
//      two such chains (first and second half of its keys) interleaved,
//   3. publishes its 256 digit counts and resolves its global digit
//      offsets by decoupled look-back over earlier tiles (one thread per
//      digit; every wait is bounded and aborts the whole pass on timeout),
//   4. reorders keys (then values) through shared memory so the global
//      writes are runs of consecutive addresses per digit.
// The per-pass digit histograms come from one counting pass over all
// digits (or from the producer of the keys, see *_prehist).
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "bq_internal.cuh"

namespace bq {
namespace {

constexpr int SORT_BLOCK = 256;
constexpr int SORT_ITEMS = 16;  // keys a thread ranks per tile
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


// lanes holding the same value v in [0, 512): nine ballots (warp multi-split)
__device__ __forceinline__ uint32_t match9(uint32_t v)
{
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; b++) {
    const bool bit = (v >> b) & 1u;
    const uint32_t m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

// a warp whose first round holds more distinct digits than this ranks the
// rest of its keys with ballots instead of match-any
constexpr int MATCH_GROUPS_MAX = 12;

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
  uint32_t spinLimit;  // polls of one look-back wait before it gives up
  int holdTile0;       // test hook: tile 0 never publishes (every wait on it runs out)
};

// WORD: -1 ranks on the whole key; 0 / 1 on the low / high 32-bit word of a
// 64-bit key when the pass's digit lies inside that word.  Ranking on one
// word holds half the registers (no spills at 64 registers a thread); the
// whole keys are read again, from L2, when they are staged for the scatter.
template <typename KeyT, int ITEMS, int WORD>
__global__ void __launch_bounds__(SORT_BLOCK, 4) k_onesweep(const KeyT *__restrict__ keysIn, KeyT *__restrict__ keysOut,
                                                            const uint32_t *__restrict__ valsIn,
                                                            uint32_t *__restrict__ valsOut, uint32_t nHost,
                                                            const uint32_t *nDev, int shift, PassCtl ctl)
{
  griddep_wait();  // the previous pass (or the keys' producer) has finished
  const uint32_t n = nDev ? *nDev : nHost;
  constexpr int TILE = SORT_BLOCK * ITEMS;
  constexpr int WARP_ITEMS = 32 * ITEMS;
  // dynamic shared memory: keys [TILE], then values [TILE]; the digit
  // histograms (two per warp) overlay both until the local positions are
  // known (they are dead before the first key is stored)
  extern __shared__ __align__(16) unsigned char smem[];
  KeyT *sKeys = (KeyT *)smem;
  uint32_t *sVals = (uint32_t *)(smem + sizeof(KeyT) * TILE);
  uint32_t *sWarpHist = (uint32_t *)smem;  // SORT_WARPS * 2 histograms of 257
  __shared__ uint32_t sTileStart[256];
  __shared__ uint32_t sGlobalBase[256];
  __shared__ uint32_t sWarpSums[SORT_WARPS];
  __shared__ uint32_t sTile;
  __shared__ uint32_t sBad;
  constexpr int NHIST = SORT_WARPS * 2;
  constexpr int HALF = ITEMS / 2;
  static_assert(ITEMS % 2 == 0, "two ranking chains of ITEMS/2 rounds");
  static_assert(TILE <= 0xffff, "tile positions are packed in 16 bits");
  static_assert(NHIST * 257 * 4 <= (sizeof(KeyT) + 4) * TILE, "histograms must fit in the tile buffers");

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    sTile = atomicAdd(ctl.tileCtr, 1u);
    sBad = 0;
  }
  for (int i = threadIdx.x; i < NHIST * 257; i += SORT_BLOCK) sWarpHist[i] = 0;
  __syncthreads();
  const uint32_t tile = sTile;
  const uint64_t warpBase = (uint64_t)tile * TILE + (uint64_t)warp * WARP_ITEMS;

  // 1. keys (warp-contiguous sub-tiles, coalesced), or the word of each key
  // that holds the digit
  static_assert(WORD < 0 || sizeof(KeyT) == 8, "word ranking is for 64-bit keys");
  using RankT = typename std::conditional<(WORD >= 0), uint32_t, KeyT>::type;
  const int rshift = WORD == 1 ? shift - 32 : shift;
  RankT key[ITEMS];
#pragma unroll
  for (int r = 0; r < ITEMS; r++) {
    const uint64_t idx = warpBase + (uint64_t)r * 32 + lane;
    if constexpr (WORD >= 0)
      key[r] = idx < n ? __ldg(reinterpret_cast<const uint32_t *>(keysIn) + 2 * idx + WORD) : 0u;
    else
      key[r] = idx < n ? keysIn[idx] : (KeyT)0;
  }

  // 2. stable ranking inside each warp, as two independent chains (rounds
  // [0, HALF) and [HALF, ITEMS), each with its own digit histogram) so that
  // the shared-memory round trips of one overlap those of the other
  uint32_t *wh0 = sWarpHist + (2 * warp) * 257;
  uint32_t *wh1 = wh0 + 257;
  const uint32_t ltMask = lanemask_lt();
  const uint32_t geMask = ~ltMask;
  // pos2[r]: low half for item r, high half for item r + HALF -- the rank
  // within (warp, chain, digit), later the tile-local position (< 2^16;
  // 0xffff marks an item past the end)
  uint32_t pos2[HALF];
  bool byBallot = false;  // warp-uniform, chosen in round 0
#pragma unroll
  for (int r = 0; r < HALF; r++) {
    const bool v0 = warpBase + (uint64_t)r * 32 + lane < n;
    const bool v1 = warpBase + (uint64_t)(r + HALF) * 32 + lane < n;
    const uint32_t d0 = v0 ? digit_of(key[r], rshift) : 256u;  // 256: padding slot, never read back
    const uint32_t d1 = v1 ? digit_of(key[r + HALF], rshift) : 256u;
    uint32_t p0, p1;
    if (r == 0) {
      p0 = __match_any_sync(0xffffffffu, d0);
      p1 = __match_any_sync(0xffffffffu, d1);
      const uint32_t groups = __popc(__ballot_sync(0xffffffffu, (p0 & geMask) == (1u << lane)));
      byBallot = groups > MATCH_GROUPS_MAX;
    } else if (byBallot) {
      p0 = match9(d0);
      p1 = match9(d1);
    } else {
      p0 = __match_any_sync(0xffffffffu, d0);
      p1 = __match_any_sync(0xffffffffu, d1);
    }
    const uint32_t b0 = wh0[d0];
    const uint32_t b1 = wh1[d1];
    __syncwarp();
    if ((p0 & geMask) == (1u << lane)) wh0[d0] = b0 + __popc(p0);  // highest lane of the group
    if ((p1 & geMask) == (1u << lane)) wh1[d1] = b1 + __popc(p1);
    __syncwarp();
    pos2[r] = (b0 + __popc(p0 & ltMask)) | ((b1 + __popc(p1 & ltMask)) << 16);
  }
  __syncthreads();

  // per digit (thread d): warp-exclusive offsets and tile totals
  const int d = threadIdx.x;
  uint32_t cnt = 0;
#pragma unroll
  for (int h = 0; h < NHIST; h++) {  // (warp, chain) in tile order
    const uint32_t c = sWarpHist[h * 257 + d];
    sWarpHist[h * 257 + d] = cnt;
    cnt += c;
  }
  uint32_t tileTotal;
  sTileStart[d] = block_excl_scan_256(cnt, sWarpSums, &tileTotal);
  uint32_t histTotal;
  const uint32_t gStart = block_excl_scan_256(ctl.hist[d], sWarpSums, &histTotal);

  // 3. decoupled look-back (thread d owns digit d)
  uint32_t *st = ctl.status;
  if (tile == 0) {
    if (!ctl.holdTile0) __stcg(&st[d], ST_INC | cnt);
    sGlobalBase[d] = gStart - sTileStart[d];  // global position = this + tile position
  } else {
    __stcg(&st[(uint64_t)tile * 256 + d], ST_AGG | cnt);
    uint32_t excl = 0;
    int64_t j = (int64_t)tile - 1;
    bool bad = false;
    while (j >= 0) {
      uint32_t v = ld_volatile(&st[(uint64_t)j * 256 + d]);
      uint32_t spins = 0;
      while ((v & ~ST_VAL) == 0) {
        if (++spins > ctl.spinLimit || ld_volatile(ctl.abort)) {
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
    sGlobalBase[d] = gStart + excl - sTileStart[d];
  }
  __syncthreads();
  if (sBad) return;  // a wait timed out: k_sort_repair overwrites the output, the caller reports

  // 4. tile-local positions; then keys and values through shared memory
#pragma unroll
  for (int r = 0; r < HALF; r++) {
    uint32_t lo = pos2[r] & 0xffffu, hi = pos2[r] >> 16;
    const bool v0 = warpBase + (uint64_t)r * 32 + lane < n;
    const bool v1 = warpBase + (uint64_t)(r + HALF) * 32 + lane < n;
    const uint32_t d0 = digit_of(key[r], rshift), d1 = digit_of(key[r + HALF], rshift);
    lo = v0 ? sTileStart[d0] + sWarpHist[(2 * warp) * 257 + d0] + lo : 0xffffu;
    hi = v1 ? sTileStart[d1] + sWarpHist[(2 * warp + 1) * 257 + d1] + hi : 0xffffu;
    pos2[r] = lo | (hi << 16);
  }
  __syncthreads();  // histograms dead: the tile buffers may be written now
  // the whole keys, read again (from L2): the ranking copies are dead after
  // the positions, so nothing is held in registers across the look-back
#pragma unroll
  for (int r = 0; r < HALF; r++) {
    const uint32_t lo = pos2[r] & 0xffffu, hi = pos2[r] >> 16;
    const uint64_t i0 = warpBase + (uint64_t)r * 32 + lane, i1 = warpBase + (uint64_t)(r + HALF) * 32 + lane;
    if (lo != 0xffffu) sKeys[lo] = keysIn[i0];
    if (hi != 0xffffu) sKeys[hi] = keysIn[i1];
  }
  uint32_t val[ITEMS];
#pragma unroll
  for (int r = 0; r < HALF; r++) {
    const uint64_t i0 = warpBase + (uint64_t)r * 32 + lane, i1 = warpBase + (uint64_t)(r + HALF) * 32 + lane;
    val[r] = (pos2[r] & 0xffffu) != 0xffffu ? valsIn[i0] : 0u;
    val[r + HALF] = (pos2[r] >> 16) != 0xffffu ? valsIn[i1] : 0u;
  }
#pragma unroll
  for (int r = 0; r < HALF; r++) {
    const uint32_t lo = pos2[r] & 0xffffu, hi = pos2[r] >> 16;
    if (lo != 0xffffu) sVals[lo] = val[r];
    if (hi != 0xffffu) sVals[hi] = val[r + HALF];
  }
  __syncthreads();
  // 5. scatter: consecutive tile positions of one digit go to consecutive
  // global positions
#pragma unroll 4
  for (int r = 0; r < ITEMS; r++) {
    const uint32_t p = threadIdx.x + r * SORT_BLOCK;
    if (p < tileTotal) {
      const KeyT k = sKeys[p];
      const uint32_t dd = digit_of(k, shift);
      const uint32_t g = sGlobalBase[dd] + p;  // unsigned wrap-around is intended
      if (g < n) {
        keysOut[g] = k;
        valsOut[g] = sVals[p];
      } else {
        atomicOr(ctl.err, DEV_ERR_RANGE);
      }
    }
  }
}

// After the last pass.  A tile whose look-back gave up leaves its part of
// that pass's output unwritten, so if any pass gave up (or scattered out of
// range) the final output is overwritten with keys 0 and values 0..n-1:
// the caller reports the error, and whatever runs on the stream before it
// looks sees only in-range values.  Otherwise every thread returns at once.
template <typename KeyT>
__global__ void k_sort_repair(KeyT *__restrict__ keys, uint32_t *__restrict__ vals, uint32_t nHost,
                              const uint32_t *nDev, const uint32_t *abort, const uint32_t *err)
{
  griddep_wait();
  if (ld_volatile(abort) == 0 && (!err || (ld_volatile(err) & DEV_ERR_RANGE) == 0)) return;
  const uint32_t n = nDev ? *nDev : nHost;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = (KeyT)0;
    vals[i] = (uint32_t)i;
  }
}

// test hook (bq_debug_inject_sort_timeout): sorts left to start with a held tile 0
std::atomic<int> g_injectSortTimeout{0};
constexpr uint32_t INJECTED_SPIN_LIMIT = 4096;

template <typename KeyT>
int onesweep_impl(KeyT *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit, int endBit,
                  const uint32_t *preHist, int *outSel, uint32_t *dErr, Alloc &al, uint32_t *ctlWs)
{
  constexpr int ITEMS = SORT_ITEMS;
  constexpr int TILE = SORT_BLOCK * ITEMS;
  *outSel = 0;
  if ((nMax <= 1 && !nDev) || nMax == 0 || endBit <= beginBit) return BQ_OK;
  const int numPasses = (endBit - beginBit + 7) / 8;
  const int numTiles = div_up(nMax, TILE);
  TempSet tmp(al);
  uint32_t *hist = nullptr, *ctl = ctlWs;
  // ctl layout: [status: numPasses*numTiles*256][tileCtr: numPasses][abort: 1]
  const size_t statusWords = (size_t)numPasses * numTiles * 256;
  if (!ctl) {  // a caller's workspace comes zeroed
    BQ_TRY(tmp.get(&ctl, statusWords + numPasses + 1));
    BQ_CUDA(cudaMemsetAsync(ctl, 0, sizeof(uint32_t) * (statusWords + numPasses + 1), al.s));
  }
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
  // the test hook is taken by the first sort that runs after it was set
  int inject = g_injectSortTimeout.load();
  while (inject > 0 && !g_injectSortTimeout.compare_exchange_weak(inject, inject - 1)) {
  }
  const size_t smemBytes = (sizeof(KeyT) + sizeof(uint32_t)) * TILE;
  BQ_CUDA(cudaFuncSetAttribute(k_onesweep<KeyT, ITEMS, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smemBytes));
  if constexpr (sizeof(KeyT) == 8) {
    BQ_CUDA(cudaFuncSetAttribute(k_onesweep<KeyT, ITEMS, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smemBytes));
    BQ_CUDA(cudaFuncSetAttribute(k_onesweep<KeyT, ITEMS, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smemBytes));
  }
  int sel = 0;
  for (int p = 0; p < numPasses; p++) {
    PassCtl c;
    c.status = ctl + (size_t)p * numTiles * 256;
    c.tileCtr = ctl + statusWords + p;
    c.abort = ctl + statusWords + numPasses;
    c.err = dErr;
    c.hist = hist + p * 256;
    c.spinLimit = inject > 0 ? INJECTED_SPIN_LIMIT : SPIN_LIMIT;
    c.holdTile0 = inject > 0 && p == 0 && numTiles > 1;
    ProfScope ps(sizeof(KeyT) == 8 ? "sort.onesweep64" : "sort.onesweep32", al.s);
    const int sh = beginBit + 8 * p;
    // the 32-bit word of a 64-bit key that holds this pass's digit, if one does
    const int word = sizeof(KeyT) != 8 ? -1 : sh >= 32 ? 1 : sh + 8 <= 32 ? 0 : -1;
    // each pass may be scheduled while the one before drains (it waits for
    // it before its first access)
    auto launch = [&](auto kernel) {
      return launch_pdl(kernel, dim3(numTiles), dim3(SORT_BLOCK), smemBytes, al.s, (const KeyT *)keys[sel],
                        keys[sel ^ 1], (const uint32_t *)vals[sel], vals[sel ^ 1], nMax, nDev, sh, c);
    };
    cudaError_t le = cudaSuccess;
    if constexpr (sizeof(KeyT) == 8) {
      le = word == 1 ? launch(k_onesweep<KeyT, ITEMS, 1>)
                     : word == 0 ? launch(k_onesweep<KeyT, ITEMS, 0>) : launch(k_onesweep<KeyT, ITEMS, -1>);
    } else {
      le = launch(k_onesweep<KeyT, ITEMS, -1>);
    }
    BQ_CUDA(le);
    sel ^= 1;
  }
  {
    ProfScope ps("sort.repair", al.s);
    BQ_CUDA(launch_pdl(k_sort_repair<KeyT>, dim3(num_sms()), dim3(256), 0, al.s, keys[sel], vals[sel], nMax, nDev,
                       (const uint32_t *)(ctl + statusWords + numPasses), (const uint32_t *)dErr));
  }
  BQ_CUDA(cudaGetLastError());
  *outSel = sel;
  return BQ_OK;
}

} // namespace

int onesweep_sort_u64(uint64_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al, uint32_t *ctlWs)
{
  return onesweep_impl<uint64_t>(keys, vals, nMax, nDev, beginBit, endBit, dHist, outSel, dErr, al, ctlWs);
}

int onesweep_sort_u32(uint32_t *keys[2], uint32_t *vals[2], uint32_t nMax, const uint32_t *nDev, int beginBit,
                      int endBit, const uint32_t *dHist, int *outSel, uint32_t *dErr, Alloc &al)
{
  return onesweep_impl<uint32_t>(keys, vals, nMax, nDev, beginBit, endBit, dHist, outSel, dErr, al, nullptr);
}

size_t onesweep_ctl_words(uint32_t nMax, int beginBit, int endBit)
{
  constexpr int TILE = SORT_BLOCK * SORT_ITEMS;
  const int numPasses = endBit > beginBit ? (endBit - beginBit + 7) / 8 : 0;
  return (size_t)numPasses * div_up(nMax, TILE) * 256 + numPasses + 1;
}

} // namespace bq

extern "C" int bq_debug_inject_sort_timeout(int count)
{
  if (count < 0) return bq::set_error(BQ_ERR_INVALID_ARGUMENT, "count must be >= 0");
  bq::g_injectSortTimeout.store(count);
  return BQ_OK;
}
