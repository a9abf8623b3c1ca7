// bq_query.cuh -- pieces shared by the binary and wide point queries:
// the closest-point leaf functor, the per-call scratch (query order,
// overflow list, deep stacks) and its host-side setup and check.
#pragma once

#include "bq_traverse.cuh"

namespace bq {

constexpr int DEEP_THREADS = 2048;  // threads of a deep-stack re-run kernel
constexpr int DEEP_STACK = 1024;    // entries of 8 bytes per deep stack

// ------------------------------------------------------------------
// closest point candidates
// ------------------------------------------------------------------
template <int TIE>
struct CPLeaf {
  const uint32_t *__restrict__ primIDs;
  const float *__restrict__ points;
  float qx, qy, qz;
  float best;
  int32_t id;
  int32_t skipId;  // blacklisted prim (findClosest_exludeID), -1: none
  int skipSelf;    // skip points equal to the query (findClosest_exludeSelf)
  __device__ __forceinline__ float operator()(uint64_t off, uint32_t cnt)
  {
    for (uint32_t j = 0; j < cnt; j++) {
      const uint32_t pid = __ldg(primIDs + off + j);
      const float *p = points + 3ull * pid;
      const float px = __ldg(p), py = __ldg(p + 1), pz = __ldg(p + 2);
      // blacklisted candidates are passed over (findClosest.h:200-203)
      if ((int32_t)pid == skipId || (skipSelf && px == qx && py == qy && pz == qz)) continue;
      const float d = sqr_pp(px, py, pz, qx, qy, qz);
      const bool take = (TIE == TIE_REFERENCE) ? (d < best)  // findClosest.h:211-218
                                               : (d < best || (d == best && id >= 0 && (int32_t)pid < id));
      if (take) {
        best = d;
        id = (int32_t)pid;
      }
    }
    return best;
  }
};

// blacklist of a closest-point call: per-query excluded ids, or points
// equal to the query
struct CpExclude {
  const int32_t *ids;
  int self;
};

struct QueryScratch {
  uint32_t *order = nullptr;
  uint32_t *ovfList = nullptr, *ovfCount = nullptr, *err = nullptr;
  StackEntry *deep = nullptr;
};

// Allocates the call's scratch from `tmp` and, with `reorder`, sorts the
// queries along a 30-bit Morton curve inside rootBox (6 device floats:
// lower xyz, upper xyz); qs.order is then the visiting order.
int prepare_queries(const float *rootBox, const float *queries, uint32_t nq, bool reorder, TempSet &tmp, Alloc &al,
                    QueryScratch &qs);
// Synchronises the stream and turns the device error word into a status.
int finish_queries(QueryScratch &qs, Alloc &al);
// ids = -1, d = +inf (and numFound = 0) for nq queries of k results
__global__ void k_fill_empty(uint32_t nq, int k, int32_t *ids, float *d, int32_t *numFound);

} // namespace bq
