// bq_tune.cu -- launch-shape autotuner for one tree's build + query
// (closest point or kNN).  No counterpart in the reference, whose leaf
// size comes from BuildConfig and whose query launch shape is the user's
// own kernel.  Every combination of leaf threshold, stack depth and block
// size is timed with CUDA events on the caller's inputs (a Morton build of
// the boxes, then one query batch; one warm-up each), and the fastest
// build + query is returned.  With the default tie rule the answers do not
// depend on these knobs, only the time.
#include <cmath>

#include "bq_internal.cuh"

namespace bq {
int build_morton63(bq_bvh3f *bvh, const bq_box3f *boxes, uint32_t n, const bq_build_config *cfg, Alloc &al);
int closest_point(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, float maxSqr,
                  const bq_query_config *qcfg, int32_t *ids, float *d, Alloc &al, const int32_t *excludeIds,
                  int excludeSelf);
int knn(const bq_bvh3f *bvh, const float *points, const float *queries, uint32_t nq, int k, float maxSqr,
        const bq_query_config *qcfg, int32_t *ids, float *d, int32_t *numFound, Alloc &al);

namespace {
// mean ms of `reps` runs of fn after one warm-up, CUDA events on the stream
template <typename Fn>
int time_ms(Fn fn, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int reps, float *ms)
{
  BQ_TRY(fn());
  BQ_CUDA(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; r++) BQ_TRY(fn());
  BQ_CUDA(cudaEventRecord(e1, s));
  BQ_CUDA(cudaEventSynchronize(e1));
  BQ_CUDA(cudaEventElapsedTime(ms, e0, e1));
  *ms /= reps;
  return BQ_OK;
}

int free_tree(bq_bvh3f *t, Alloc &al)
{
  const int s1 = al.free_bytes(t->primIDs), s2 = al.free_bytes(t->nodes);
  *t = bq_bvh3f{};
  return s1 != BQ_OK ? s1 : s2;
}

struct Events {
  cudaEvent_t e[2] = {nullptr, nullptr};
  ~Events()
  {
    for (auto x : e)
      if (x) cudaEventDestroy(x);
  }
};
} // namespace

int autotune_query(const bq_box3f *boxes, const float *points, uint32_t n, const float *queries, uint32_t nq, int k,
                   bq_tuning *best, Alloc &al)
{
  if (!best) return set_error(BQ_ERR_INVALID_ARGUMENT, "best is NULL");
  if (k < 0 || k > 64) return set_error(BQ_ERR_INVALID_ARGUMENT, "k must be 0 (closest point) or in [1, 64]");
  if (n == 0 || nq == 0) return set_error(BQ_ERR_INVALID_ARGUMENT, "nothing to tune on");
  TempSet tmp(al);
  int32_t *ids = nullptr;
  float *d = nullptr;
  const size_t slots = (size_t)nq * (k ? k : 1);
  BQ_TRY(tmp.get(&ids, slots));
  BQ_TRY(tmp.get(&d, slots));
  Events ev;
  BQ_CUDA(cudaEventCreate(&ev.e[0]));
  BQ_CUDA(cudaEventCreate(&ev.e[1]));
  const int leaves[] = {1, 2, 4, 8}, stacks[] = {32, 64, 128}, blocks[] = {64, 128};
  float bestMs = INFINITY;
  for (int lf : leaves) {
    const bq_build_config bc{1 << 15, lf, BQ_SPATIAL_MEDIAN};
    bq_bvh3f t{};
    float tb = 0.f;
    BQ_TRY(time_ms(
        [&]() -> int {
          if (t.nodes) BQ_TRY(free_tree(&t, al));
          return build_morton63(&t, boxes, n, &bc, al);
        },
        al.s, ev.e[0], ev.e[1], 1, &tb));
    int status = BQ_OK;
    for (int st : stacks)
      for (int bl : blocks) {
        if (status != BQ_OK) break;
        const bq_query_config qc{BQ_TIES_LOWEST_ID, st, bl, 1, 32};
        float tq = 0.f;
        status = time_ms(
            [&]() -> int {
              return k == 0 ? closest_point(&t, points, queries, nq, INFINITY, &qc, ids, d, al, nullptr, 0)
                            : knn(&t, points, queries, nq, k, INFINITY, &qc, ids, d, nullptr, al);
            },
            al.s, ev.e[0], ev.e[1], 2, &tq);
        if (status == BQ_OK && tb + tq < bestMs) {
          bestMs = tb + tq;
          *best = bq_tuning{lf, st, bl, 32, tb, tq};
        }
      }
    const int fs = free_tree(&t, al);
    BQ_TRY(status);
    BQ_TRY(fs);
  }
  return BQ_OK;
}

} // namespace bq
