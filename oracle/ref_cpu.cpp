// ref_cpu.cpp -- C entry points over the reference library's own HOST code.
//
// TEST / BASELINE INFRASTRUCTURE ONLY.  Compiled by oracle/build_ref.sh
// directly against the unmodified reference headers (never copied into
// this repository) into oracle/_ref/libref_cpu.so.  It is used to
//   * pin the C restatement in bq_oracle.c (golden fixtures),
//   * time the reference's CPU path for the benchmark's reference arm.
//
// Reference entry points wrapped here:
//   cuBQL::cpuBuilder            cuBQL/builder/cpu.h:76-84
//   cuBQL::points::findClosest   cuBQL/queries/points/findClosest.h:336-360
//   cuBQL::points::findKNN       cuBQL/queries/points/knn.h:75-116
//   cuBQL::triangles::findClosest cuBQL/queries/triangles/findClosest.h:132-152
//     (device-only in the reference; compiled for the host with an empty
//      __device__ macro, the only change needed)
#include "cuBQL/bvh.h"
#include "cuBQL/builder/cpu.h"
#include "cuBQL/queries/points/findClosest.h"
#include "cuBQL/queries/points/knn.h"
#ifndef __device__
#define __device__
#endif
#include "cuBQL/queries/triangles/findClosest.h"
#include "samples/common/IO.h"

#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

using namespace cuBQL;

namespace {
template <typename F>
void parallel_for(uint32_t n, int nthreads, F f)
{
  if (nthreads <= 1 || n < 1024) {
    for (uint32_t i = 0; i < n; i++) f(i);
    return;
  }
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; t++) {
    ts.emplace_back([=]() {
      uint64_t b = (uint64_t)n * t / nthreads, e = (uint64_t)n * (t + 1) / nthreads;
      for (uint64_t i = b; i < e; i++) f((uint32_t)i);
    });
  }
  for (auto &th : ts) th.join();
}

bvh3f view(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims)
{
  bvh3f b;
  b.nodes = (bvh3f::Node *)nodes;
  b.numNodes = numNodes;
  b.primIDs = (uint32_t *)primIDs;
  b.numPrims = numPrims;
  return b;
}
} // namespace

extern "C" {

int ref_cpu_node_size(void) { return (int)sizeof(bvh3f::Node); }

// cpuBuilder over n boxes (24 B each); nodesOut must hold 2n+2 nodes.
int ref_cpu_build(const float *boxes, uint32_t n, int makeLeafThreshold, void *nodesOut, uint32_t *primIDsOut,
                  uint32_t *numNodes, uint32_t *numPrims)
{
  bvh3f bvh;
  BuildConfig cfg;
  cfg.makeLeafThreshold = makeLeafThreshold;
  cpuBuilder(bvh, (const box3f *)boxes, n, cfg);
  std::memcpy(nodesOut, bvh.nodes, sizeof(bvh3f::Node) * bvh.numNodes);
  std::memcpy(primIDsOut, bvh.primIDs, sizeof(uint32_t) * bvh.numPrims);
  *numNodes = bvh.numNodes;
  *numPrims = bvh.numPrims;
  cpu::freeBVH(bvh);
  return 0;
}

// Throughput of the reference's host builder with `nthreads` independent
// builds of the same boxes running at once (cpuBuilder is single-threaded,
// cuBQL/builder/cpu/spatialMedian.h:32-33, and keeps no shared state, so
// concurrent builds are the most the reference's CPU path can do on a
// multi-core host).  Each thread builds `reps` times; returns wall seconds.
int ref_cpu_build_throughput(const float *boxes, uint32_t n, int makeLeafThreshold, int nthreads, int reps,
                             double *seconds)
{
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; t++) {
    ts.emplace_back([=]() {
      for (int r = 0; r < reps; r++) {
        bvh3f bvh;
        BuildConfig cfg;
        cfg.makeLeafThreshold = makeLeafThreshold;
        cpuBuilder(bvh, (const box3f *)boxes, n, cfg);
        cpu::freeBVH(bvh);
      }
    });
  }
  for (auto &th : ts) th.join();
  *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

// closest point per query; dist = fSqrDistance_rd(points[id], q), or +inf.
int ref_cpu_closest(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                    const float *points, const float *queries, uint32_t nq, float maxSqr, int32_t *ids,
                    float *dists, int nthreads)
{
  bvh3f bvh = view(nodes, numNodes, primIDs, numPrims);
  const vec3f *pts = (const vec3f *)points;
  const vec3f *qs = (const vec3f *)queries;
  parallel_for(nq, nthreads, [&](uint32_t i) {
    int id = points::findClosest(bvh, pts, qs[i], maxSqr);
    ids[i] = id;
    dists[i] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[i]);
  });
  return 0;
}

// closest point with the reference's blacklists: excludeIds != NULL ->
// points::findClosest_exludeID(excludeIds[i], ...), else
// points::findClosest_exludeSelf (findClosest.h:278-334)
int ref_cpu_closest_exclude(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                            const float *points, const float *queries, uint32_t nq, float maxSqr,
                            const int32_t *excludeIds, int32_t *ids, float *dists, int nthreads)
{
  bvh3f bvh = view(nodes, numNodes, primIDs, numPrims);
  const vec3f *pts = (const vec3f *)points;
  const vec3f *qs = (const vec3f *)queries;
  parallel_for(nq, nthreads, [&](uint32_t i) {
    const int id = excludeIds ? points::findClosest_exludeID(excludeIds[i], bvh, pts, qs[i], maxSqr)
                              : points::findClosest_exludeSelf(bvh, pts, qs[i], maxSqr);
    ids[i] = id;
    dists[i] = id < 0 ? INFINITY : fSqrDistance_rd(pts[id], qs[i]);
  });
  return 0;
}

// kNN per query (k <= 64): ids/dists nq*k (unfilled: -1/+inf), numFound nq.
int ref_cpu_knn(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                const float *points, const float *queries, uint32_t nq, int k, float maxSqr, int32_t *ids,
                float *dists, int32_t *numFound, int nthreads)
{
  if (k < 1 || k > 64) return -1;
  bvh3f bvh = view(nodes, numNodes, primIDs, numPrims);
  const vec3f *pts = (const vec3f *)points;
  const vec3f *qs = (const vec3f *)queries;
  parallel_for(nq, nthreads, [&](uint32_t i) {
    knn::Candidate c[64];
    knn::Result r = points::findKNN(c, k, bvh, pts, qs[i], maxSqr);
    for (int j = 0; j < k; j++) {
      ids[(size_t)i * k + j] = j < r.numFound ? c[j].primID : -1;
      dists[(size_t)i * k + j] = j < r.numFound ? c[j].sqrDist : INFINITY;
    }
    numFound[i] = r.numFound;
  });
  return 0;
}

// triangles given indexed (int3 into float3 vertices); converted to the
// reference's non-indexed Triangle array here.
int ref_cpu_tri_closest(const void *nodes, uint32_t numNodes, const uint32_t *primIDs, uint32_t numPrims,
                        const int32_t *tris, uint32_t nt, const float *verts, const float *queries, uint32_t nq,
                        float maxSqr, int32_t *ids, float *dists, float *P, int nthreads)
{
  bvh3f bvh = view(nodes, numNodes, primIDs, numPrims);
  std::vector<Triangle> T(nt);
  const vec3f *V = (const vec3f *)verts;
  for (uint32_t t = 0; t < nt; t++) {
    T[t].a = V[tris[3 * t + 0]];
    T[t].b = V[tris[3 * t + 1]];
    T[t].c = V[tris[3 * t + 2]];
  }
  const vec3f *qs = (const vec3f *)queries;
  parallel_for(nq, nthreads, [&](uint32_t i) {
    triangles::FCPResult r;
    r.clear(maxSqr);
    r.P = vec3f(0.f, 0.f, 0.f);
    triangles::findClosest(r, bvh, T.data(), qs[i]);
    ids[i] = r.primID;
    dists[i] = r.primID < 0 ? INFINITY : r.sqrDist;
    if (P) {
      P[3 * (size_t)i + 0] = r.P.x;
      P[3 * (size_t)i + 1] = r.P.y;
      P[3 * (size_t)i + 2] = r.P.z;
    }
  });
  return 0;
}

// samples/common/IO.h: saveBinary / loadBinary of vec3d points and the
// convert<float,3> the samples apply after loading
int ref_cpu_save_points_f64(const char *path, const double *pts, uint64_t n)
{
  std::vector<vec3d> v(n);
  for (uint64_t i = 0; i < n; i++) v[i] = vec3d(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
  cuBQL::samples::saveBinary(path, v);
  return 0;
}

int ref_cpu_load_points_f64_as_f32(const char *path, float *out, uint64_t capacity, uint64_t *n)
{
  try {
    std::vector<vec3d> v = cuBQL::samples::loadBinary<vec3d>(path);
    std::vector<vec3f> f = cuBQL::samples::convert<float, 3>(v);
    *n = f.size();
    if (f.size() > capacity) return -1;
    for (size_t i = 0; i < f.size(); i++) {
      out[3 * i] = f[i].x;
      out[3 * i + 1] = f[i].y;
      out[3 * i + 2] = f[i].z;
    }
  } catch (...) {
    return -1;
  }
  return 0;
}

} // extern "C"
