/*
 * bq_oracle.c -- CPU restatement of the cuBQL BVH build-and-query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it to
 * produce the answers the CUDA library must reproduce.  No product code
 * path links it, and nothing here is ever timed as the product.
 *
 * Every function restates one piece of the reference (Ssz990220/cuBQL),
 * cited as path:line inside the reference project.  Floating-point
 * expressions are written with explicit fmaf() where the reference's GPU
 * build contracts a multiply-add, selected by `fma_mode`:
 *   0 = no contraction (what g++ emits for the reference's host code
 *       on x86-64 without -mfma);
 *   1 = the shapes nvcc emits for the reference's device code, pinned
 *       against the reference kernels themselves on a B200 (see the
 *       pin tests): x*x+y*y+z*z  ->  fmaf(z,z,fmaf(x,x,y*y)) and
 *       dot(v,v) (accumulating loop) -> fmaf(z,z,fmaf(y,y,x*x)).
 *
 * Build: oracle/build_oracle.sh (gcc -O2 -ffp-contract=off).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>

typedef struct { float lo[3], hi[3]; } obox;                 /* box3f, 24 B */
typedef struct { float lo[3], hi[3]; uint64_t admin; } onode; /* BinaryBVH<float,3>::Node, 32 B */

#define ADMIN(off, cnt) ((uint64_t)(off) | ((uint64_t)(cnt) << 48))
#define ADMIN_OFF(a) ((a) & 0xFFFFFFFFFFFFull)
#define ADMIN_CNT(a) ((uint32_t)((a) >> 48))

/* ------------------------------------------------------------------ */
/* seeded generator: LCG<8> seeded by TEA (cuBQL/math/random.h:24-68), */
/* points as in samples/common/Generator.cpp:201-215                    */
/* ------------------------------------------------------------------ */
static uint32_t lcg_seed(uint32_t v0, uint32_t v1)
{
  uint32_t s0 = 0;
  for (int n = 0; n < 8; n++) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}

static float lcg_next(uint32_t *state)
{
  *state = 1664525u * *state + 1013904223u;
  return (float)(*state & 0x00FFFFFFu) / (float)0x01000000;
}

/* out[3*i+d] = (float)(lo + u*(hi-lo)), u from LCG<8>(seed, i) */
void orc_uniform_points(uint32_t n, uint32_t seed, double lo, double hi, float *out)
{
  for (uint32_t i = 0; i < n; i++) {
    uint32_t st = lcg_seed(seed, i);
    for (int d = 0; d < 3; d++) {
      float u = lcg_next(&st);
      out[3 * (size_t)i + d] = (float)(lo + (double)u * (hi - lo));
    }
  }
}

/* ------------------------------------------------------------------ */
/* order-preserving float <-> int32 used for atomic centroid bounds     */
/* (cuBQL/builder/cuda/builder_common.h:102-117)                        */
/* ------------------------------------------------------------------ */
static int32_t enc_f(float f)
{
  int32_t b;
  memcpy(&b, &f, 4);
  if (b & (int32_t)0x80000000) b ^= 0x7fffffff;
  return b;
}

static float dec_f(int32_t b)
{
  float f;
  if (b & (int32_t)0x80000000) b ^= 0x7fffffff;
  memcpy(&f, &b, 4);
  return f;
}

static int box_empty(const obox *b) { return b->lo[0] > b->hi[0]; } /* box.h:139 */

static void box_center(const obox *b, float c[3]) /* box.h:146-147 */
{
  for (int d = 0; d < 3; d++) c[d] = (b->lo[d] + b->hi[d]) / 2.0f;
}

/* ------------------------------------------------------------------ */
/* stable LSD sort of (u64 key, u32 value), 8-bit digits                */
/* (stands in for cub::DeviceRadixSort::SortPairs, radix.h:666-687)     */
/* ------------------------------------------------------------------ */
static void stable_sort_pairs(uint64_t *keys, uint32_t *vals, uint32_t n, int beginBit, int endBit)
{
  uint64_t *k2 = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint32_t *v2 = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (int shift = beginBit; shift < endBit; shift += 8) {
    uint32_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (uint32_t i = 0; i < n; i++) cnt[((keys[i] >> shift) & 0xff) + 1]++;
    for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
    for (uint32_t i = 0; i < n; i++) {
      uint32_t p = cnt[(keys[i] >> shift) & 0xff]++;
      k2[p] = keys[i];
      v2[p] = vals[i];
    }
    memcpy(keys, k2, sizeof(uint64_t) * n);
    memcpy(vals, v2, sizeof(uint32_t) * n);
  }
  free(k2);
  free(v2);
}

/* ------------------------------------------------------------------ */
/* refit (cuBQL/builder/cuda/sm_builder.h:616-675): leaf = union of its */
/* prim boxes in primIDs order, inner = union(left, right).  min/max of */
/* floats is exact, so processing children before parents in any order */
/* gives the same bits as the reference's atomic bottom-up climb.       */
/* ------------------------------------------------------------------ */
static void refit_tree(onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const obox *boxes)
{
  /* children always have larger indices than their parent in the trees
     built here (BFS or DFS allocation), so a reverse sweep suffices */
  for (int64_t i = (int64_t)numNodes - 1; i >= 0; i--) {
    if (i == 1) continue;
    onode *n = &nodes[i];
    uint64_t off = ADMIN_OFF(n->admin);
    uint32_t cnt = ADMIN_CNT(n->admin);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (cnt) {
      for (uint32_t j = 0; j < cnt; j++) {
        const obox *b = &boxes[primIDs[off + j]];
        for (int d = 0; d < 3; d++) { lo[d] = fminf(lo[d], b->lo[d]); hi[d] = fmaxf(hi[d], b->hi[d]); }
      }
    } else {
      const onode *l = &nodes[off], *r = &nodes[off + 1];
      for (int d = 0; d < 3; d++) { lo[d] = fminf(l->lo[d], r->lo[d]); hi[d] = fmaxf(l->hi[d], r->hi[d]); }
    }
    memcpy(n->lo, lo, sizeof(lo));
    memcpy(n->hi, hi, sizeof(hi));
  }
}

/* ------------------------------------------------------------------ */
/* Morton / radix builder (cuBQL/builder/cuda/radix.h)                  */
/* ------------------------------------------------------------------ */

/* 21 bits of x spread to every third bit (radix.h:340-354 computes the
   same with shift/mask stages; written here as a plain loop) */
static uint64_t spread3(uint32_t x)
{
  uint64_t r = 0;
  for (int i = 0; i < 21; i++) r |= (uint64_t)((x >> i) & 1u) << (3 * i);
  return r;
}

/* quantizer (radix.h:41-62): bias = centroid lower, scale =
   2^21 * (1/max(maxExtent, 1e-20)); cell = min(uint((c-bias)*scale), 2^21-1) */
typedef struct { float bias[3]; float scale; } oquant;

static void quant_init(oquant *q, const int32_t cbLo[3], const int32_t cbHi[3])
{
  float lo[3], sz[3];
  for (int d = 0; d < 3; d++) { lo[d] = dec_f(cbLo[d]); sz[d] = dec_f(cbHi[d]) - lo[d]; }
  float ext = fmaxf(fmaxf(sz[0], sz[1]), sz[2]);   /* reduce_max, vec.h:564 */
  float rc = 1.0f / fmaxf(ext, 1e-20f);            /* rcp, math.h:44 */
  for (int d = 0; d < 3; d++) q->bias[d] = lo[d];
  q->scale = 2097152.0f * rc;
}

static uint32_t quant_cell(float c, float bias, float scale)
{
  float f = (c - bias) * scale;
  uint32_t u;
  if (!(f > 0.0f)) u = 0;                     /* cvt.rzi.u32: negative / NaN -> 0 */
  else if (f >= 4294967296.0f) u = 0xFFFFFFFFu;
  else u = (uint32_t)f;
  return u < 2097151u ? u : 2097151u;
}

uint64_t orc_morton63(float cx, float cy, float cz, const float bias[3], float scale)
{
  return spread3(quant_cell(cx, bias[0], scale)) | (spread3(quant_cell(cy, bias[1], scale)) << 1)
       | (spread3(quant_cell(cz, bias[2], scale)) << 2);
}

/* findSplit (radix.h:446-482) */
static int find_split(int64_t *split, const uint64_t *keys, int64_t begin, int64_t end, int maxLeaf)
{
  uint64_t fk = keys[begin], lk = keys[end - 1];
  if (fk == lk) {
    if (end - begin > maxLeaf) { *split = (begin + end) / 2; return 1; }
    return 0;
  }
  int nm = __builtin_clzll(fk ^ lk);
  uint64_t sk = lk & (0xFFFFFFFFFFFFFFFFull << (63 - nm));
  while (end > begin) {
    int64_t mid = (begin + end) / 2;
    if (keys[mid] < sk) begin = mid + 1; else end = mid;
  }
  *split = begin;
  return 1;
}

/* Shared topology pass for the Morton builders: level-by-level
   createNodes (radix.h:501-570) with children allocated in index order,
   which yields canonical BFS numbering.  keys/ids are sorted; writes
   admin words into nodes[] and returns the node count. */
static uint32_t radix_topology(const uint64_t *keys, uint32_t nv, int leafThr, onode *nodes)
{
  typedef struct { uint32_t a, b; } tnode;
  uint64_t cap = 2ull * (nv ? nv : 1) + 2;
  tnode *t = (tnode *)calloc(cap, sizeof(tnode));
  uint8_t *fin = (uint8_t *)calloc(cap, 1);
  t[0].a = 0; t[0].b = nv;
  uint64_t devAlloc = 2, done = 0, alloc = 1;
  while (done < alloc) {
    for (uint64_t id = done; id < alloc; id++) {
      uint32_t a = t[id].a, b = t[id].b;
      int64_t size = (int64_t)b - (int64_t)a, split = -1;
      if (size <= leafThr || !find_split(&split, keys, a, b, leafThr)) {
        t[id].a = a; t[id].b = (uint32_t)size; fin[id] = 1;     /* leaf {offset,count} */
      } else {
        uint64_t c = devAlloc; devAlloc += 2;
        t[c].a = a; t[c].b = (uint32_t)split;
        t[c + 1].a = (uint32_t)split; t[c + 1].b = b;
        t[id].a = (uint32_t)c; t[id].b = 0; fin[id] = 1;        /* inner {childOffset,0} */
      }
    }
    done = alloc;
    alloc = devAlloc;
  }
  for (uint64_t i = 0; i < devAlloc; i++) {
    memset(&nodes[i], 0, sizeof(onode));
    nodes[i].admin = (i == 1) ? 0 : ADMIN(t[i].a, t[i].b);     /* writeFinalNodes, radix.h:572-589 */
  }
  free(t);
  free(fin);
  return (uint32_t)devAlloc;
}

/* cuda::radixBuilder (radix.h:591-771).  nodes needs room for 2*n+2,
   primIDs for n.  Empty boxes are dropped by a stable compaction.
   Returns 0 on success. */
int orc_radix_build(const obox *boxes, uint32_t n, int makeLeafThreshold, int maxAllowedLeafSize,
                    onode *nodes, uint32_t *primIDs, uint32_t *numNodes, uint32_t *numPrims,
                    uint64_t *keysOut)
{
  int thr = makeLeafThreshold > 0
              ? (makeLeafThreshold < maxAllowedLeafSize ? makeLeafThreshold : maxAllowedLeafSize)
              : 1;                                          /* radix.h:599-602 */
  int32_t cbLo[3], cbHi[3];
  for (int d = 0; d < 3; d++) { cbLo[d] = enc_f(FLT_MAX); cbHi[d] = enc_f(-FLT_MAX); }
  uint32_t nv = 0;
  for (uint32_t i = 0; i < n; i++) {                        /* fillBuildState, radix.h:199-227 */
    if (box_empty(&boxes[i])) continue;
    float c[3];
    box_center(&boxes[i], c);
    for (int d = 0; d < 3; d++) {
      int32_t e = enc_f(c[d]);
      if (e < cbLo[d]) cbLo[d] = e;
      if (e > cbHi[d]) cbHi[d] = e;
    }
    nv++;
  }
  oquant q;
  quant_init(&q, cbLo, cbHi);                              /* finishBuildState, radix.h:229-241 */
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (nv ? nv : 1));
  uint32_t j = 0;
  for (uint32_t i = 0; i < n; i++) {                        /* computeUnsortedKeysAndPrimIDs, radix.h:396-421 */
    if (box_empty(&boxes[i])) continue;
    float c[3];
    box_center(&boxes[i], c);
    keys[j] = orc_morton63(c[0], c[1], c[2], q.bias, q.scale);
    primIDs[j] = i;
    j++;
  }
  stable_sort_pairs(keys, primIDs, nv, 0, 64);
  if (nv == 0) {
    *numNodes = 0;
    *numPrims = 0;
    free(keys);
    return 0;
  }
  *numNodes = radix_topology(keys, nv, thr, nodes);
  *numPrims = nv;
  refit_tree(nodes, *numNodes, primIDs, boxes);
  if (keysOut) memcpy(keysOut, keys, sizeof(uint64_t) * nv);
  free(keys);
  return 0;
}

/* ------------------------------------------------------------------ */
/* spatial-median GPU builder (cuBQL/builder/cuda/sm_builder.h:147-614, */
/* dispatch gpu_builder.h:31-67), level-synchronous, BFS numbering.     */
/* The reference assigns sides for degenerate nodes (dim == -1) by an   */
/* atomic counter whose start value is the bit pattern of the encoded   */
/* centroid lower-z (the field aliases it in the TempNode union,        */
/* sm_builder.h:82-103); the k-th prim to arrive goes to side           */
/* (start + k) & 1.  Here "k-th" is the k-th prim of the node in primID */
/* order, which reproduces the reference's child counts exactly.        */
/* ------------------------------------------------------------------ */
typedef struct { uint32_t begin, end; int32_t cbLo[3], cbHi[3]; } sm_open;

static void sm_bounds(const obox *boxes, const uint32_t *ids, uint32_t b, uint32_t e, sm_open *o)
{
  for (int d = 0; d < 3; d++) { o->cbLo[d] = enc_f(FLT_MAX); o->cbHi[d] = enc_f(-FLT_MAX); }
  for (uint32_t i = b; i < e; i++) {
    float c[3];
    box_center(&boxes[ids[i]], c);
    for (int d = 0; d < 3; d++) {
      int32_t v = enc_f(c[d]);
      if (v < o->cbLo[d]) o->cbLo[d] = v;
      if (v > o->cbHi[d]) o->cbHi[d] = v;
    }
  }
}

int orc_sm_build(const obox *boxes, uint32_t n, int makeLeafThreshold, onode *nodes, uint32_t *primIDs,
                 uint32_t *numNodes, uint32_t *numPrims)
{
  if (n == 0) { *numNodes = 0; *numPrims = 0; return 0; }  /* gpu_builder.h:39 */
  int thr = makeLeafThreshold == 0 ? 1 : makeLeafThreshold;   /* gpu_builder.h:60-63 */
  uint32_t *cur = primIDs, *alt = (uint32_t *)malloc(sizeof(uint32_t) * n);
  uint32_t nv = 0, ninv = 0;
  for (uint32_t i = 0; i < n; i++)                     /* initPrims, sm_builder.h:121-145 */
    if (boxes[i].lo[0] <= boxes[i].hi[0]) cur[nv++] = i;
  for (uint32_t i = 0; i < n; i++)
    if (!(boxes[i].lo[0] <= boxes[i].hi[0])) { cur[nv + ninv] = i; ninv++; }
  uint64_t cap = 2ull * n + 2;
  sm_open *lvl = (sm_open *)malloc(sizeof(sm_open) * cap);
  uint32_t *lvlId = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  sm_open *nxt = (sm_open *)malloc(sizeof(sm_open) * cap);
  uint32_t *nxtId = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  memset(&nodes[0], 0, 2 * sizeof(onode));
  uint64_t alloc = 2, nl = 1;
  lvl[0].begin = 0; lvl[0].end = nv; lvlId[0] = 0;
  sm_bounds(boxes, cur, 0, nv, &lvl[0]);
  while (nl) {
    uint64_t nn = 0;
    for (uint64_t k = 0; k < nl; k++) {                  /* selectSplits, sm_builder.h:147-244 */
      sm_open *o = &lvl[k];
      uint32_t id = lvlId[k], count = o->end - o->begin;
      memset(&nodes[id], 0, sizeof(onode));
      if ((int64_t)count <= thr) { nodes[id].admin = ADMIN(o->begin, count); continue; }
      float widestWidth = 0.f, wLo = 0.f, wHi = 0.f, wCtr = 0.f;
      int widestDim = -1;
      for (int d = 0; d < 3; d++) {
        float lo = dec_f(o->cbLo[d]), hi = dec_f(o->cbHi[d]);
        float width = hi - lo;
        if (width <= widestWidth) continue;
        float ctr = 0.5f * (hi + lo);
        widestWidth = width; widestDim = d; wLo = lo; wHi = hi; wCtr = ctr;
      }
      int dim = (widestDim < 0 || wCtr == wLo || wCtr == wHi) ? -1 : widestDim;
      float pos = wCtr;
      uint32_t tb = (uint32_t)o->cbLo[2];
      /* stable partition (updatePrims_shm, sm_builder.h:317-393):
         left side in order, then right side in order */
      uint32_t nLeft = 0;
      for (uint32_t i = o->begin; i < o->end; i++) {
        uint32_t pid = cur[i];
        int side = dim < 0 ? (int)((tb + (i - o->begin)) & 1u)
                           : (0.5f * (boxes[pid].lo[dim] + boxes[pid].hi[dim])) >= pos;
        if (!side) nLeft++;
      }
      uint32_t wl = o->begin, wr = o->begin + nLeft;
      for (uint32_t i = o->begin; i < o->end; i++) {
        uint32_t pid = cur[i];
        int side = dim < 0 ? (int)((tb + (i - o->begin)) & 1u)
                           : (0.5f * (boxes[pid].lo[dim] + boxes[pid].hi[dim])) >= pos;
        if (!side) alt[wl++] = pid; else alt[wr++] = pid;
      }
      memcpy(cur + o->begin, alt + o->begin, sizeof(uint32_t) * count);
      uint64_t c = alloc; alloc += 2;
      nodes[id].admin = ADMIN(c, 0);
      nxt[nn].begin = o->begin; nxt[nn].end = o->begin + nLeft; nxtId[nn] = (uint32_t)c;
      sm_bounds(boxes, cur, nxt[nn].begin, nxt[nn].end, &nxt[nn]); nn++;
      nxt[nn].begin = o->begin + nLeft; nxt[nn].end = o->end; nxtId[nn] = (uint32_t)c + 1;
      sm_bounds(boxes, cur, nxt[nn].begin, nxt[nn].end, &nxt[nn]); nn++;
    }
    sm_open *t = lvl; lvl = nxt; nxt = t;
    uint32_t *ti = lvlId; lvlId = nxtId; nxtId = ti;
    nl = nn;
  }
  *numNodes = (uint32_t)alloc;
  *numPrims = n;                                         /* sm_builder.h:584 keeps invalid prims at the end */
  refit_tree(nodes, *numNodes, cur, boxes);
  free(alt); free(lvl); free(lvlId); free(nxt); free(nxtId);
  return 0;
}

/* ------------------------------------------------------------------ */
/* binned SAH GPU builder (cuBQL/builder/cuda/sah_builder.h:22-538,    */
/* dispatch gpu_builder.h:41-53) and its edge-length sibling, the ELH  */
/* builder (cuBQL/builder/cuda/elh_builder.h:22-556, dispatch           */
/* gpu_builder.h:54-59).  heur 0 = SAH: 16 bins per axis, bin          */
/* denominator hi - lo + 1e-20, cost measure surfaceArea; heur 1 = ELH: */
/* 8 bins, denominator hi - lo, measure edgeLengths (sx + sy + sz).     */
/* Bin boxes are the union of the prim boxes, AtomicBox-encoded          */
/* (builder_common.h:38-167, empty = +-FLT_MAX).                        */
/* ------------------------------------------------------------------ */
#define SAH_BINS 16
typedef struct { int32_t lo[3], hi[3]; int32_t count, pad; } osah_bin; /* 32 B, as SAHBins::bins[] */
typedef struct { osah_bin b[3][SAH_BINS]; } osah_bins;                /* ELH uses b[d][0..7] */
static int heur_bins(int heur) { return heur ? 8 : SAH_BINS; }

/* edgeLengths(box) (elh_builder.h:66-76): sum += upper - lower, from 0 */
static float elh_len(const float *lo, const float *hi)
{
  float sum = 0.f;
  for (int k = 0; k < 3; k++) sum += hi[k] - lo[k];
  return sum;
}

/* surfaceArea(box3f) (cuBQL/math/box.h:198-205): sx*sy + sx*sz + sy*sz */
static float sah_area(const float *lo, const float *hi, int fma_mode)
{
  float sx = hi[0] - lo[0], sy = hi[1] - lo[1], sz = hi[2] - lo[2];
  if (fma_mode) return fmaf(sy, sz, fmaf(sx, sy, sx * sz));
  return (sx * sy + sx * sz) + sy * sz;
}

float orc_sah_area(const float *lo, const float *hi, int fma_mode) { return sah_area(lo, hi, fma_mode); }

static float heur_measure(const float *lo, const float *hi, int fma_mode, int heur)
{
  return heur ? elh_len(lo, hi) : sah_area(lo, hi, fma_mode);
}

/* evaluateSAH (sah_builder.h:61-104) / evaluateELH (elh_builder.h:93-133):
   returns the split dim (-1: leaf) and *splitBin; costs
   lMeasure*lCount + rMeasure*rCount */
int orc_heur_evaluate(const osah_bins *s, int fma_mode, int heur, int *splitBin)
{
  const int NB = heur_bins(heur);
  float bestCost = INFINITY;
  int splitDim = -1;
  float rAreas[SAH_BINS];
  for (int d = 0; d < 3; d++) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int rCount = 0;
    for (int b = NB - 1; b >= 0; --b) {
      const osah_bin *bin = &s->b[d][b];
      for (int k = 0; k < 3; k++) {
        float bl = dec_f(bin->lo[k]), bh = dec_f(bin->hi[k]);
        if (bl < lo[k]) lo[k] = bl;
        if (bh > hi[k]) hi[k] = bh;
      }
      rCount += bin->count;
      rAreas[b] = heur_measure(lo, hi, fma_mode, heur);
    }
    float leafCost = rAreas[0] * (float)rCount;
    if (leafCost < bestCost) { bestCost = leafCost; splitDim = -1; }
    lo[0] = lo[1] = lo[2] = INFINITY;
    hi[0] = hi[1] = hi[2] = -INFINITY;
    int lCount = 0;
    for (int b = 0; b < NB; b++) {
      float rArea = rAreas[b];
      float lArea = heur_measure(lo, hi, fma_mode, heur);
      if (lCount > 0 && rCount > 0) {
        float cost = fma_mode ? fmaf(lArea, (float)lCount, rArea * (float)rCount)
                              : lArea * (float)lCount + rArea * (float)rCount;
        if (cost < bestCost) { bestCost = cost; splitDim = d; *splitBin = b; }
      }
      const osah_bin *bin = &s->b[d][b];
      for (int k = 0; k < 3; k++) {
        float bl = dec_f(bin->lo[k]), bh = dec_f(bin->hi[k]);
        if (bl < lo[k]) lo[k] = bl;
        if (bh > hi[k]) hi[k] = bh;
      }
      lCount += bin->count;
      rCount -= bin->count;
    }
  }
  return splitDim;
}

int orc_sah_evaluate(const osah_bins *s, int fma_mode, int *splitBin)
{
  return orc_heur_evaluate(s, fma_mode, 0, splitBin);
}

/* bin of a centroid coordinate (SAH binPrims :170-180, updatePrims
   :300-306; ELH :205-217, :343-351 divide by hi - lo alone) */
static int sah_bin_of(float c, float lo, float hi, int heur)
{
  if (!(hi > lo)) return 0;
  const int NB = heur_bins(heur);
  float rel = heur ? (c - lo) / (hi - lo) : (c - lo) / ((hi - lo) + 1e-20f);
  float f = rel * (float)NB;
  int bin = (f != f) ? 0 : (f >= 2147483647.f ? 2147483647 : (f <= -2147483648.f ? (-2147483647 - 1) : (int)f));
  return bin < 0 ? 0 : (bin > NB - 1 ? NB - 1 : bin);
}

static void sah_center(const obox *b, int d, float *c) { *c = 0.5f * (b->lo[d] + b->hi[d]); }

/* Level-synchronous, BFS numbering; partitions stable, so leaves list
   their prims in ascending primID order (the reference's final
   (nodeID, primID) sort, :446-473).  A node the heuristic would make a
   leaf of more than 65535 prims (the 16-bit count) is split in halves
   by position instead (the reference writes a truncated count). */
int orc_heur_build(const obox *boxes, uint32_t n, int makeLeafThreshold, int fma_mode, int heur, onode *nodes,
                   uint32_t *primIDs, uint32_t *numNodes, uint32_t *numPrims)
{
  const int NB = heur_bins(heur);
  if (n == 0) { *numNodes = 0; *numPrims = 0; return 0; }
  int thr = makeLeafThreshold;
  uint32_t *cur = primIDs, *alt = (uint32_t *)malloc(sizeof(uint32_t) * n);
  uint32_t nv = 0, ninv = 0;
  for (uint32_t i = 0; i < n; i++)                     /* initPrims :124-146 */
    if (boxes[i].lo[0] <= boxes[i].hi[0]) cur[nv++] = i;
  for (uint32_t i = 0; i < n; i++)
    if (!(boxes[i].lo[0] <= boxes[i].hi[0])) { cur[nv + ninv] = i; ninv++; }
  uint64_t cap = 2ull * n + 2;
  sm_open *lvl = (sm_open *)malloc(sizeof(sm_open) * cap);
  uint32_t *lvlId = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  sm_open *nxt = (sm_open *)malloc(sizeof(sm_open) * cap);
  uint32_t *nxtId = (uint32_t *)malloc(sizeof(uint32_t) * cap);
  osah_bins *bins = (osah_bins *)malloc(sizeof(osah_bins));
  memset(&nodes[0], 0, 2 * sizeof(onode));
  uint64_t alloc = 2, nl = 1;
  lvl[0].begin = 0; lvl[0].end = nv; lvlId[0] = 0;
  sm_bounds(boxes, cur, 0, nv, &lvl[0]);
  while (nl) {
    uint64_t nn = 0;
    for (uint64_t k = 0; k < nl; k++) {
      sm_open *o = &lvl[k];
      uint32_t id = lvlId[k], count = o->end - o->begin;
      memset(&nodes[id], 0, sizeof(onode));
      int dim = -1, sbin = 0;
      float clo[3], chi[3];
      for (int d = 0; d < 3; d++) { clo[d] = dec_f(o->cbLo[d]); chi[d] = dec_f(o->cbHi[d]); }
      if ((int64_t)count > thr) {                       /* selectSplits :220-263 */
        for (int d = 0; d < 3; d++)
          for (int b = 0; b < NB; b++) {
            osah_bin *x = &bins->b[d][b];
            for (int k = 0; k < 3; k++) { x->lo[k] = enc_f(FLT_MAX); x->hi[k] = enc_f(-FLT_MAX); }
            x->count = 0;
          }
        for (uint32_t i = o->begin; i < o->end; i++) {  /* binPrims :148-197 */
          const obox *pb = &boxes[cur[i]];
          for (int d = 0; d < 3; d++) {
            float c;
            sah_center(pb, d, &c);
            osah_bin *x = &bins->b[d][sah_bin_of(c, clo[d], chi[d], heur)];
            for (int k = 0; k < 3; k++) {
              int32_t el = enc_f(pb->lo[k]), eh = enc_f(pb->hi[k]);
              if (el < x->lo[k]) x->lo[k] = el;
              if (eh > x->hi[k]) x->hi[k] = eh;
            }
            x->count++;
          }
        }
        dim = orc_heur_evaluate(bins, fma_mode, heur, &sbin);
      }
      int halves = dim < 0 && count > 65535u;
      if (dim < 0 && !halves) { nodes[id].admin = ADMIN(o->begin, count); continue; }
      /* updatePrims :266-310: side = (bin along dim >= split bin), stable */
      uint32_t nLeft = 0;
      for (uint32_t i = o->begin; i < o->end; i++) {
        float c = 0.f;
        if (!halves) sah_center(&boxes[cur[i]], dim, &c);
        int side = halves ? (i - o->begin) >= count / 2 : sah_bin_of(c, clo[dim], chi[dim], heur) >= sbin;
        if (!side) nLeft++;
      }
      uint32_t wl = o->begin, wr = o->begin + nLeft;
      for (uint32_t i = o->begin; i < o->end; i++) {
        float c = 0.f;
        if (!halves) sah_center(&boxes[cur[i]], dim, &c);
        int side = halves ? (i - o->begin) >= count / 2 : sah_bin_of(c, clo[dim], chi[dim], heur) >= sbin;
        if (!side) alt[wl++] = cur[i]; else alt[wr++] = cur[i];
      }
      memcpy(cur + o->begin, alt + o->begin, sizeof(uint32_t) * count);
      if (nLeft == 0 || nLeft == count) {             /* cannot happen: the split had both sides */
        free(alt); free(lvl); free(lvlId); free(nxt); free(nxtId); free(bins);
        return -1;
      }
      uint64_t c = alloc; alloc += 2;
      nodes[id].admin = ADMIN(c, 0);
      nxt[nn].begin = o->begin; nxt[nn].end = o->begin + nLeft; nxtId[nn] = (uint32_t)c;
      sm_bounds(boxes, cur, nxt[nn].begin, nxt[nn].end, &nxt[nn]); nn++;
      nxt[nn].begin = o->begin + nLeft; nxt[nn].end = o->end; nxtId[nn] = (uint32_t)c + 1;
      sm_bounds(boxes, cur, nxt[nn].begin, nxt[nn].end, &nxt[nn]); nn++;
    }
    sm_open *t = lvl; lvl = nxt; nxt = t;
    uint32_t *ti = lvlId; lvlId = nxtId; nxtId = ti;
    nl = nn;
  }
  *numNodes = (uint32_t)alloc;
  *numPrims = n;
  refit_tree(nodes, *numNodes, cur, boxes);
  free(alt); free(lvl); free(lvlId); free(nxt); free(nxtId); free(bins);
  return 0;
}

int orc_sah_build(const obox *boxes, uint32_t n, int makeLeafThreshold, int fma_mode, onode *nodes,
                  uint32_t *primIDs, uint32_t *numNodes, uint32_t *numPrims)
{
  return orc_heur_build(boxes, n, makeLeafThreshold, fma_mode, 0, nodes, primIDs, numNodes, numPrims);
}

/* ------------------------------------------------------------------ */
/* host spatial-median builder cpuBuilder (cuBQL/builder/cpu/           */
/* spatialMedian.h:45-180): recursive, DFS numbering, right side filled */
/* from the end backwards.                                              */
/* ------------------------------------------------------------------ */
typedef struct { onode *nodes; uint64_t count; uint32_t *ids, *alt; const obox *boxes; int thr; } cpu_ctx;

static void cpu_rec(cpu_ctx *c, uint64_t nodeID, uint32_t begin, uint32_t end)
{
  if ((int64_t)(end - begin) <= c->thr) { c->nodes[nodeID].admin = ADMIN(begin, end - begin); return; }
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = begin; i < end; i++) {
    float ct[3];
    box_center(&c->boxes[c->ids[i]], ct);
    for (int d = 0; d < 3; d++) {                       /* std::min / std::max */
      lo[d] = ct[d] < lo[d] ? ct[d] : lo[d];
      hi[d] = hi[d] < ct[d] ? ct[d] : hi[d];
    }
  }
  float sz[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  float mxy = sz[0] < sz[1] ? sz[1] : sz[0];
  int dim = sz[2] > mxy ? 2 : (sz[1] > sz[0] ? 1 : 0);  /* arg_max, vec.h:640-643 */
  float pos = (lo[dim] + hi[dim]) / 2.0f;
  uint32_t Nl = 0, Nr = 0;
  for (uint32_t i = begin; i < end; i++) {
    uint32_t pid = c->ids[i];
    float ct[3];
    box_center(&c->boxes[pid], ct);
    if (ct[dim] < pos) c->alt[begin + Nl++] = pid;
    else c->alt[end - ++Nr] = pid;
  }
  uint32_t mid;
  int mx = c->thr > 1 ? c->thr : 1;
  if (Nl && Nr) mid = begin + Nl;
  else if ((int64_t)(end - begin) <= mx) { c->nodes[nodeID].admin = ADMIN(begin, end - begin); return; }
  else mid = (begin + end) / 2;
  for (uint32_t i = begin; i < end; i++) c->ids[i] = c->alt[i];
  uint64_t child = c->count;
  c->count += 2;
  c->nodes[nodeID].admin = ADMIN(child, 0);
  cpu_rec(c, child + 0, begin, mid);
  cpu_rec(c, child + 1, mid, end);
}

int orc_cpu_build(const obox *boxes, uint32_t n, int makeLeafThreshold, onode *nodes, uint32_t *primIDs,
                  uint32_t *numNodes, uint32_t *numPrims)
{
  cpu_ctx c;
  uint32_t nv = 0;
  for (uint32_t i = 0; i < n; i++)
    if (!box_empty(&boxes[i])) primIDs[nv++] = i;
  c.nodes = nodes; c.count = 1; c.ids = primIDs; c.boxes = boxes; c.thr = makeLeafThreshold;
  c.alt = (uint32_t *)malloc(sizeof(uint32_t) * (nv ? nv : 1));
  memset(nodes, 0, sizeof(onode));
  cpu_rec(&c, 0, 0, nv);
  free(c.alt);
  *numNodes = (uint32_t)c.count;
  *numPrims = nv;
  /* DFS allocation also puts children after parents */
  for (uint64_t i = c.count; i-- > 0;) {
    onode *nd = &nodes[i];
    uint64_t off = ADMIN_OFF(nd->admin);
    uint32_t cnt = ADMIN_CNT(nd->admin);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (cnt) {
      for (uint32_t j = 0; j < cnt; j++) {
        const obox *b = &boxes[primIDs[off + j]];
        for (int d = 0; d < 3; d++) {
          lo[d] = b->lo[d] < lo[d] ? b->lo[d] : lo[d];
          hi[d] = hi[d] < b->hi[d] ? b->hi[d] : hi[d];
        }
      }
    } else {
      for (int k = 0; k < 2; k++) {
        const onode *ch = &nodes[off + k];
        for (int d = 0; d < 3; d++) {
          lo[d] = ch->lo[d] < lo[d] ? ch->lo[d] : lo[d];
          hi[d] = hi[d] < ch->hi[d] ? ch->hi[d] : hi[d];
        }
      }
    }
    memcpy(nd->lo, lo, sizeof(lo));
    memcpy(nd->hi, hi, sizeof(hi));
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* canonical renumbering: BFS from node 0, children visited (offset,   */
/* offset+1), node 1 left zero, leaves' prims laid out in BFS order.    */
/* Two builds of the same topology then compare byte for byte.          */
/* ------------------------------------------------------------------ */
int orc_canonicalize(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, onode *outNodes,
                     uint32_t *outPrimIDs, uint32_t *outNumPrims)
{
  if (numNodes == 0) { *outNumPrims = 0; return 0; }
  uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * numNodes);
  uint64_t head = 0, tail = 0, nextPair = 2, primPos = 0;
  q[tail++] = 0;
  memset(&outNodes[0], 0, sizeof(onode) * (numNodes < 2 ? numNodes : 2));
  /* outIdx of queue entry k: 0 for the root, then 2,3,4,... */
  uint32_t *outIdx = (uint32_t *)malloc(sizeof(uint32_t) * numNodes);
  outIdx[0] = 0;
  while (head < tail) {
    uint32_t src = q[head];
    uint32_t dst = outIdx[head];
    head++;
    const onode *s = &nodes[src];
    onode *d = &outNodes[dst];
    memcpy(d->lo, s->lo, sizeof(d->lo));
    memcpy(d->hi, s->hi, sizeof(d->hi));
    uint64_t off = ADMIN_OFF(s->admin);
    uint32_t cnt = ADMIN_CNT(s->admin);
    if (cnt) {
      for (uint32_t j = 0; j < cnt; j++) outPrimIDs[primPos + j] = primIDs[off + j];
      d->admin = ADMIN(primPos, cnt);
      primPos += cnt;
    } else {
      if (off + 1 >= numNodes || tail + 2 > numNodes) { free(q); free(outIdx); return -1; }
      d->admin = ADMIN(nextPair, 0);
      q[tail] = (uint32_t)off; outIdx[tail] = (uint32_t)nextPair; tail++;
      q[tail] = (uint32_t)off + 1; outIdx[tail] = (uint32_t)nextPair + 1; tail++;
      nextPair += 2;
    }
  }
  free(q);
  free(outIdx);
  *outNumPrims = (uint32_t)primPos;
  return (int)(nextPair == numNodes ? 0 : -2);
}

/* ------------------------------------------------------------------ */
/* distances                                                            */
/* ------------------------------------------------------------------ */
/* fSqrDistance_rd(vec3f,vec3f) = fSqrLength_rd(a-b)
   (cuBQL/math/conservativeDistances.h:60-100) */
static float sqr_pp(const float *p, const float *q, int fma_mode)
{
  float x = p[0] - q[0], y = p[1] - q[1], z = p[2] - q[2];
  if (fma_mode) return fmaf(z, z, fmaf(x, x, y * y));
  return (x * x + y * y) + z * z;
}

/* shrinkingRadiusQuery::fSqrDistance_rd(vec3f, box3f)
   (cuBQL/traversal/shrinkingRadiusQuery.h:253-259) with dot() as the
   accumulating loop of cuBQL/math/vec.h:459-466 */
static float sqr_pbox(const float *q, const float *lo, const float *hi, int fma_mode)
{
  float v[3];
  for (int d = 0; d < 3; d++) {
    float pr = fminf(fmaxf(q[d], lo[d]), hi[d]);
    v[d] = pr - q[d];
  }
  if (fma_mode) return fmaf(v[2], v[2], fmaf(v[1], v[1], v[0] * v[0]));
  return ((0.0f + v[0] * v[0]) + v[1] * v[1]) + v[2] * v[2];
}

float orc_sqr_pp(const float *p, const float *q, int fma_mode) { return sqr_pp(p, q, fma_mode); }
float orc_sqr_pbox(const float *q, const float *lo, const float *hi, int fma_mode)
{
  return sqr_pbox(q, lo, hi, fma_mode);
}

/* ------------------------------------------------------------------ */
/* shrinking-radius traversal (shrinkingRadiusQuery.h:409-508) driving  */
/* the closest-point and kNN candidate logic.                           */
/*   (numbering as BQ_TIES_* in include/bq.h)                          */
/*   tie_mode 1: the reference's rules -- accept strictly closer       */
/*     (findClosest.h:211-213), cull children at >= (:456), ties in    */
/*     descent go to child 1 (:463-471), pop at <= (:494-506); kNN     */
/*     candidates inserted by insert_linear (common/knn.h:57-78).      */
/*   tie_mode 0: results independent of tree shape -- candidates are   */
/*     ordered by (sqrDist, primID); nodes are culled only when        */
/*     strictly farther than the current bound.                        */
/* The stack is unbounded here; *overflow reports whether a stack of   */
/* `stackLimit` entries would have overflowed (the reference then      */
/* returns early, :475-478).                                           */
/* ------------------------------------------------------------------ */
typedef struct {
  int k, tie_mode, fma_mode;
  int numFound;
  float sqrDistMax;   /* knn::Result.sqrDistMax */
  int32_t *ids;
  float *dists;
  const float *points;
  const float *q;
} knn_state;

/* returns the new cull radius proposal for this prim */
static float knn_visit(knn_state *s, uint32_t pid)
{
  float d = sqr_pp(s->points + 3 * (size_t)pid, s->q, s->fma_mode);
  int k = s->k;
  if (s->tie_mode == 1) {
    int ins;
    if (s->numFound < k) ins = s->numFound++;
    else {
      if (d >= s->sqrDistMax) return s->sqrDistMax;
      ins = k - 1;
    }
    while (ins > 0 && s->dists[ins - 1] > d) {
      s->dists[ins] = s->dists[ins - 1];
      s->ids[ins] = s->ids[ins - 1];
      --ins;
    }
    s->dists[ins] = d;
    s->ids[ins] = (int32_t)pid;
    if (s->numFound == k) s->sqrDistMax = s->dists[k - 1];
    return s->sqrDistMax;
  }
  /* tie_mode 0: keep the k smallest (d, id) with d < initial radius */
  int ins;
  if (s->numFound < k) {
    if (!(d < s->sqrDistMax)) return s->sqrDistMax;
    ins = s->numFound++;
  } else {
    float ld = s->dists[k - 1];
    int32_t li = s->ids[k - 1];
    if (d > ld || (d == ld && (int32_t)pid >= li)) return s->sqrDistMax;
    ins = k - 1;
  }
  while (ins > 0 && (s->dists[ins - 1] > d || (s->dists[ins - 1] == d && s->ids[ins - 1] > (int32_t)pid))) {
    s->dists[ins] = s->dists[ins - 1];
    s->ids[ins] = s->ids[ins - 1];
    --ins;
  }
  s->dists[ins] = d;
  s->ids[ins] = (int32_t)pid;
  if (s->numFound == k) s->sqrDistMax = s->dists[k - 1];
  return s->sqrDistMax;
}

typedef struct { uint32_t idx; float dist; } stk_e;

/* tie_mode 0 compares node distances against the radius widened by 2^-20
   relative (node-box and point distances round differently); only the
   set of visited nodes changes, never the answer */
static float lowest_slack(float c) { return fmaf(c, 0x1p-20f, c); }

static void traverse(const onode *nodes, const uint32_t *primIDs, const float *q, float maxSqr,
                     knn_state *s, int stackLimit, int *overflow, uint32_t *visitedNodes)
{
  int tie = s->tie_mode;
  float cull = maxSqr;
  size_t cap = 256, sp = 0, maxsp = 0;
  stk_e *stack = (stk_e *)malloc(sizeof(stk_e) * cap);
  uint64_t admin = nodes[0].admin;
  *overflow = 0;
  for (;;) {
    for (;;) {
      if (ADMIN_CNT(admin) != 0) break;
      uint32_t i0 = (uint32_t)ADMIN_OFF(admin), i1 = i0 + 1;
      const onode *n0 = &nodes[i0], *n1 = &nodes[i1];
      if (visitedNodes) *visitedNodes += 2;
      float d0 = sqr_pbox(q, n0->lo, n0->hi, s->fma_mode);
      float d1 = sqr_pbox(q, n1->lo, n1->hi, s->fma_mode);
      float dmin = fminf(d0, d1), dmax = fmaxf(d0, d1);
      float cs = tie == 1 ? cull : lowest_slack(cull);
      int dead = tie == 1 ? (dmin >= cull) : (dmin > cs);
      if (dead) { admin = 0; break; }
      uint32_t farID;
      if (d0 < d1) { admin = n0->admin; farID = i1; }
      else { admin = n1->admin; farID = i0; }
      int both = tie == 1 ? (dmax < cull) : (dmax <= cs);
      if (both) {
        if (sp >= (size_t)stackLimit && !*overflow) *overflow = 1;
        if (sp == cap) { cap *= 2; stack = (stk_e *)realloc(stack, sizeof(stk_e) * cap); }
        stack[sp].idx = farID; stack[sp].dist = dmax; sp++;
        if (sp > maxsp) maxsp = sp;
      }
    }
    if (ADMIN_CNT(admin) != 0) {
      uint64_t off = ADMIN_OFF(admin);
      uint32_t cnt = ADMIN_CNT(admin);
      float leaf = INFINITY;
      for (uint32_t j = 0; j < cnt; j++) {
        float r = knn_visit(s, primIDs[off + j]);
        leaf = fminf(leaf, r);
      }
      cull = fminf(cull, leaf);
    }
    for (;;) {
      if (sp == 0) { free(stack); return; }
      stk_e e = stack[--sp];
      if (e.dist <= (tie == 1 ? cull : lowest_slack(cull))) { admin = nodes[e.idx].admin; break; }
    }
  }
}

/* kNN over nq queries: ids/dists are nq*k (unfilled slots: -1 / +inf),
   numFound nq.  k == 1 with tie_mode 1 is NOT findClosest (which rejects
   at >= the running best and never inserts beyond the radius); use
   orc_closest_point for that. */
int orc_knn(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const float *points,
            const float *queries, uint32_t nq, int k, float maxSqr, int fma_mode, int tie_mode,
            int stackLimit, int32_t *ids, float *dists, int32_t *numFound, uint8_t *overflowed)
{
  for (uint32_t i = 0; i < nq; i++) {
    knn_state s;
    s.k = k; s.tie_mode = tie_mode; s.fma_mode = fma_mode; s.numFound = 0; s.sqrDistMax = maxSqr;
    s.ids = ids + (size_t)i * k; s.dists = dists + (size_t)i * k;
    s.points = points; s.q = queries + 3 * (size_t)i;
    for (int j = 0; j < k; j++) { s.ids[j] = -1; s.dists[j] = INFINITY; }
    int of = 0;
    if (numNodes) traverse(nodes, primIDs, s.q, maxSqr, &s, stackLimit, &of, NULL);
    numFound[i] = s.numFound;
    if (overflowed) overflowed[i] = (uint8_t)of;
  }
  return 0;
}

/* closest point (findClosest.h:181-226, 336-360).  tie_mode 1 accepts a
   candidate only when strictly closer; tie_mode 0 also takes an equally
   close candidate with a lower primID.  Not found: id -1, dist +inf.
   Blacklists (findClosest_withBlackList, findClosest.h:181-226): with
   excludeIds, query i skips prim excludeIds[i] (when >= 0;
   findClosest_exludeID, :278-305); with excludeSelf, every query skips the
   points equal to itself (findClosest_exludeSelf, :307-334). */
static int closest_impl(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const float *points,
                        const float *queries, uint32_t nq, float maxSqr, int fma_mode, int tie_mode,
                        int stackLimit, const int32_t *excludeIds, int excludeSelf, int32_t *ids, float *dists,
                        uint8_t *overflowed, uint32_t *visits)
{
  for (uint32_t i = 0; i < nq; i++) {
    const float *q = queries + 3 * (size_t)i;
    int32_t best = -1;
    float bestD = maxSqr;
    int of = 0;
    uint32_t nvis = 0;
    if (numNodes) {
      float cull = maxSqr;
      size_t cap = 256, sp = 0;
      stk_e *stack = (stk_e *)malloc(sizeof(stk_e) * cap);
      uint64_t admin = nodes[0].admin;
      for (;;) {
        for (;;) {
          if (ADMIN_CNT(admin) != 0) break;
          uint32_t i0 = (uint32_t)ADMIN_OFF(admin), i1 = i0 + 1;
          const onode *n0 = &nodes[i0], *n1 = &nodes[i1];
          nvis += 2;
          float d0 = sqr_pbox(q, n0->lo, n0->hi, fma_mode);
          float d1 = sqr_pbox(q, n1->lo, n1->hi, fma_mode);
          float dmin = fminf(d0, d1), dmax = fmaxf(d0, d1);
          float cs = tie_mode == 1 ? cull : lowest_slack(cull);
          int dead = tie_mode == 1 ? (dmin >= cull) : (dmin > cs);
          if (dead) { admin = 0; break; }
          uint32_t farID;
          if (d0 < d1) { admin = n0->admin; farID = i1; }
          else { admin = n1->admin; farID = i0; }
          int both = tie_mode == 1 ? (dmax < cull) : (dmax <= cs);
          if (both) {
            if (sp >= (size_t)stackLimit) of = 1;
            if (sp == cap) { cap *= 2; stack = (stk_e *)realloc(stack, sizeof(stk_e) * cap); }
            stack[sp].idx = farID; stack[sp].dist = dmax; sp++;
          }
        }
        if (ADMIN_CNT(admin) != 0) {
          uint64_t off = ADMIN_OFF(admin);
          uint32_t cnt = ADMIN_CNT(admin);
          float leaf = INFINITY;
          for (uint32_t j = 0; j < cnt; j++) {
            uint32_t pid = primIDs[off + j];
            const float *pp = points + 3 * (size_t)pid;
            if (excludeIds && excludeIds[i] >= 0 && (int32_t)pid == excludeIds[i]) continue;
            if (excludeSelf && pp[0] == q[0] && pp[1] == q[1] && pp[2] == q[2]) continue;
            float d = sqr_pp(pp, q, fma_mode);
            int take = tie_mode == 1 ? (d < bestD)
                                     : (d < bestD || (best >= 0 && d == bestD && (int32_t)pid < best));
            if (take) { bestD = d; best = (int32_t)pid; }
            leaf = fminf(leaf, bestD);
          }
          cull = fminf(cull, leaf);
        }
        int popped = 0;
        while (sp) {
          stk_e e = stack[--sp];
          if (e.dist <= (tie_mode == 1 ? cull : lowest_slack(cull))) { admin = nodes[e.idx].admin; popped = 1; break; }
        }
        if (!popped) break;
      }
      free(stack);
    }
    ids[i] = best;
    dists[i] = best >= 0 ? bestD : INFINITY;
    if (overflowed) overflowed[i] = (uint8_t)of;
    if (visits) visits[i] = nvis;
  }
  return 0;
}

int orc_closest_point(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const float *points,
                      const float *queries, uint32_t nq, float maxSqr, int fma_mode, int tie_mode,
                      int stackLimit, int32_t *ids, float *dists, uint8_t *overflowed, uint32_t *visits)
{
  return closest_impl(nodes, numNodes, primIDs, points, queries, nq, maxSqr, fma_mode, tie_mode, stackLimit, NULL, 0,
                      ids, dists, overflowed, visits);
}

int orc_closest_point_exclude(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const float *points,
                              const float *queries, uint32_t nq, float maxSqr, int fma_mode, int tie_mode,
                              const int32_t *excludeIds, int excludeSelf, int32_t *ids, float *dists)
{
  return closest_impl(nodes, numNodes, primIDs, points, queries, nq, maxSqr, fma_mode, tie_mode, 1 << 30,
                      excludeIds, excludeSelf, ids, dists, NULL, NULL);
}

/* ------------------------------------------------------------------ */
/* fixed-box query: fixedBoxQuery::forEachLeaf over a BinaryBVH         */
/* (cuBQL/traversal/fixedBoxQuery.h:73-137) with forEachPrim's per-prim */
/* loop (:139-156), the lambda keeping prims whose own box overlaps the */
/* query box; overlap is box_t::overlaps (cuBQL/math/box.h:208-212).    */
/* ------------------------------------------------------------------ */
static int box_ov(const float *qlo, const float *qhi, const float *lo, const float *hi)
{
  return !(qhi[0] < lo[0] || qhi[1] < lo[1] || qhi[2] < lo[2] || hi[0] < qlo[0] || hi[1] < qlo[1] ||
           hi[2] < qlo[2]);
}

/* For query q the overlapping prims go to ids[offsets[q] ..] in visiting
   order (pass ids = NULL to count only); counts[q] gets their number.
   Returns 0, or -1 when a traversal needs more than stackLimit entries. */
int orc_box_query(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const obox *boxes,
                  const obox *queryBoxes, uint32_t nq, int stackLimit, uint32_t *counts, const uint64_t *offsets,
                  int32_t *ids)
{
  uint64_t *stack = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(stackLimit > 0 ? stackLimit : 1));
  int rc = 0;
  if (!stack) return -1;
  for (uint32_t q = 0; q < nq; q++) {
    const float *qlo = queryBoxes[q].lo, *qhi = queryBoxes[q].hi;
    uint32_t c = 0;
    int sp = 0;
    if (numNodes == 0) { counts[q] = 0; continue; }
    uint64_t node = nodes[0].admin;
    for (;;) {
      int leaf = 1;
      while (ADMIN_CNT(node) == 0) {
        const onode *n0 = &nodes[ADMIN_OFF(node)], *n1 = n0 + 1;
        int o0 = box_ov(qlo, qhi, n0->lo, n0->hi), o1 = box_ov(qlo, qhi, n1->lo, n1->hi);
        if (o0) {
          if (o1) {
            if (sp >= stackLimit) { rc = -1; goto next; }
            stack[sp++] = n1->admin;
          }
          node = n0->admin;
        } else if (o1) {
          node = n1->admin;
        } else {
          leaf = 0;
          break;
        }
      }
      if (leaf) {
        for (uint32_t j = 0; j < ADMIN_CNT(node); j++) {
          uint32_t pid = primIDs[ADMIN_OFF(node) + j];
          if (box_ov(qlo, qhi, boxes[pid].lo, boxes[pid].hi)) {
            if (ids) ids[offsets[q] + c] = (int32_t)pid;
            c++;
          }
        }
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
  next:
    counts[q] = c;
  }
  free(stack);
  return rc;
}

/* ------------------------------------------------------------------ */
/* wide BVHs: WideBVH<float,3,W> (cuBQL/bvh.h:113-141).  A slot is an   */
/* onode whose word holds valid (bit 0), offset (bits 1-45), count      */
/* (bits 46-61).                                                        */
/* ------------------------------------------------------------------ */
#define WS_MASK45 ((1ull << 45) - 1)
#define WS_MAKE(off, cnt) (1ull | (((uint64_t)(off) & WS_MASK45) << 1) | ((uint64_t)((cnt) & 0xFFFFu) << 46))
#define WS_VALID(w) ((w) & 1ull)
#define WS_OFF(w) (((w) >> 1) & WS_MASK45)
#define WS_CNT(w) ((uint32_t)((w) >> 46) & 0xFFFFu)
#define WS_UNUSED ((0xFFFFFFFFull << 1) | (0xFFFFull << 46))
#define WS_BITS(w) ((w) & ((1ull << 62) - 1)) /* the bit field's 62 bits */

static int log2w(int W) { return W == 2 ? 1 : (W == 4 ? 2 : (W == 8 ? 3 : -1)); }

/* Binary -> wide collapse, wide_gpu_builder.h:40-158: inner nodes at a
   depth that is a multiple of log2(W) (and the root) root wide nodes,
   numbered by increasing binary index; each wide node's slots are its
   treelet's frontier in collapseExecute's stack order (:131-149).  Node 1
   is skipped.  outSlots holds up to numNodes*W slots.  Returns the wide
   node count, or -1 on a malformed tree. */
int orc_wide_collapse(const onode *nodes, uint32_t numNodes, int W, onode *outSlots)
{
  int lg = log2w(W);
  if (lg < 0) return -1;
  if (numNodes == 0) return 0;
  uint32_t *parent = (uint32_t *)malloc(sizeof(uint32_t) * numNodes);
  uint32_t *wid = (uint32_t *)malloc(sizeof(uint32_t) * numNodes);
  uint8_t *flag = (uint8_t *)calloc(numNodes, 1);
  int rc = 0;
  for (uint32_t i = 0; i < numNodes; i++) parent[i] = 0xFFFFFFFFu;
  for (uint32_t i = 0; i < numNodes; i++) {
    if (i == 1 || ADMIN_CNT(nodes[i].admin)) continue;
    uint64_t off = ADMIN_OFF(nodes[i].admin);
    if (off < 2 || off + 1 >= numNodes) { rc = -1; goto done; }
    parent[off] = parent[off + 1] = i;
  }
  flag[0] = 1;
  for (uint32_t i = 2; i < numNodes; i++) {
    if (ADMIN_CNT(nodes[i].admin)) continue;
    uint32_t n = i, depth = 0;
    while (n != 0 && n < numNodes && depth <= numNodes) { n = parent[n]; depth++; }
    if (n == 0 && depth % (uint32_t)lg == 0) flag[i] = 1;
  }
  uint32_t nw = 0;
  for (uint32_t i = 0; i < numNodes; i++) { wid[i] = nw; nw += flag[i]; }
  for (uint32_t i = 0; i < numNodes; i++) {
    if (!flag[i]) continue;
    onode *out = outSlots + (size_t)wid[i] * W;
    uint32_t stack[8];
    int sp = 0, written = 0;
    stack[sp++] = i;
    while (sp) {
      uint32_t n = stack[--sp];
      const onode *nd = &nodes[n];
      uint32_t cnt = ADMIN_CNT(nd->admin);
      if (cnt || (n != i && flag[n])) {
        if (written >= W) { rc = -1; goto done; }
        onode *o = &out[written++];
        memcpy(o->lo, nd->lo, sizeof(o->lo));
        memcpy(o->hi, nd->hi, sizeof(o->hi));
        o->admin = cnt ? WS_MAKE(ADMIN_OFF(nd->admin), cnt) : WS_MAKE(wid[n], 0);
      } else {
        uint64_t off = ADMIN_OFF(nd->admin);
        if (off + 1 >= numNodes || sp + 2 > 8) { rc = -1; goto done; }
        stack[sp++] = (uint32_t)off;
        stack[sp++] = (uint32_t)off + 1;
      }
    }
    for (; written < W; written++) {
      onode *o = &out[written];
      o->lo[0] = o->lo[1] = o->lo[2] = INFINITY;
      o->hi[0] = o->hi[1] = o->hi[2] = -INFINITY;
      o->admin = WS_UNUSED;
    }
  }
  rc = (int)nw;
done:
  free(parent); free(wid); free(flag);
  return rc;
}

/* Canonical form of a wide tree: BFS from node 0, slots kept in order,
   inner slots renumbered in BFS order, leaf prims laid out in BFS order,
   bits 62-63 of every word cleared (the reference leaves them as they
   were in memory).  Returns 0, or -1 on a malformed tree. */
int orc_wide_canonicalize(const onode *slots, uint32_t numWide, int W, const uint32_t *primIDs, onode *outSlots,
                          uint32_t *outPrimIDs, uint32_t *outNumPrims)
{
  if (numWide == 0) { *outNumPrims = 0; return 0; }
  uint32_t *q = (uint32_t *)malloc(sizeof(uint32_t) * numWide);
  uint32_t head = 0, tail = 0, primPos = 0;
  q[tail++] = 0;
  while (head < tail) {
    uint32_t src = q[head], dst = head;
    head++;
    for (int c = 0; c < W; c++) {
      const onode *s = &slots[(size_t)src * W + c];
      onode *d = &outSlots[(size_t)dst * W + c];
      *d = *s;
      uint64_t w = WS_BITS(s->admin);
      d->admin = w;
      if (!WS_VALID(w)) continue;
      if (WS_CNT(w)) {
        uint64_t off = WS_OFF(w);
        for (uint32_t j = 0; j < WS_CNT(w); j++) outPrimIDs[primPos + j] = primIDs[off + j];
        d->admin = WS_MAKE(primPos, WS_CNT(w));
        primPos += WS_CNT(w);
      } else {
        if (WS_OFF(w) >= numWide || tail >= numWide) { free(q); return -1; }
        q[tail] = (uint32_t)WS_OFF(w);
        d->admin = WS_MAKE(tail, 0);
        tail++;
      }
    }
  }
  free(q);
  *outNumPrims = primPos;
  return tail == numWide ? 0 : -2;
}

/* Closest point over a wide tree (findClosest.h:228-270 and
   shrinkingRadiusQuery.h:553-636); tie modes as orc_closest_point.
   Unbounded stack. */
int orc_wide_closest(const onode *slots, uint32_t numWide, int W, const uint32_t *primIDs, const float *points,
                     const float *queries, uint32_t nq, float maxSqr, int fma_mode, int tie_mode, int32_t *ids,
                     float *dists)
{
  int lg = log2w(W);
  if (lg < 0) return -1;
  for (uint32_t i = 0; i < nq; i++) {
    const float *q = queries + 3 * (size_t)i;
    int32_t best = -1;
    float bestD = maxSqr, cull = maxSqr;
    if (numWide) {
      size_t cap = 256, sp = 0;
      uint64_t *stack = (uint64_t *)malloc(sizeof(uint64_t) * cap);
      uint32_t nodeID = 0;
      for (;;) {
        int done = 0;
        for (;;) {
          while (nodeID == 0xFFFFFFFFu) {
            if (sp == 0) { done = 1; break; }
            uint64_t tos = stack[--sp];
            uint32_t db = (uint32_t)(tos >> 32);
            float d;
            memcpy(&d, &db, 4);
            if (d > (tie_mode == 1 ? cull : lowest_slack(cull))) continue;
            nodeID = (uint32_t)tos;
          }
          if (done || (nodeID & 0x80000000u)) break;
          float cs = tie_mode == 1 ? cull : lowest_slack(cull);
          uint64_t v[8];
          for (int c = 0; c < W; c++) {
            const onode *sl = &slots[(size_t)nodeID * W + c];
            v[c] = ~0ull;
            if (!WS_VALID(sl->admin)) continue;
            float d = sqr_pbox(q, sl->lo, sl->hi, fma_mode);
            if (d > cs) continue;
            uint32_t payload = WS_CNT(sl->admin) ? (0x80000000u | (nodeID << lg) | (uint32_t)c)
                                                  : (uint32_t)WS_OFF(sl->admin);
            uint32_t db;
            memcpy(&db, &d, 4);
            v[c] = ((uint64_t)db << 32) | payload;
          }
          for (int a = W - 1; a > 0; --a)
            for (int b = 0; b < a; b++) {
              uint64_t c0 = v[b], c1 = v[b + 1];
              v[b] = c0 < c1 ? c0 : c1;
              v[b + 1] = c0 < c1 ? c1 : c0;
            }
          for (int c = W - 1; c > 0; --c) {
            if (v[c] == ~0ull) continue;
            if (sp == cap) { cap *= 2; stack = (uint64_t *)realloc(stack, sizeof(uint64_t) * cap); }
            stack[sp++] = v[c];
          }
          nodeID = v[0] == ~0ull ? 0xFFFFFFFFu : (uint32_t)v[0];
        }
        if (done) break;
        uint32_t c = nodeID & (uint32_t)(W - 1);
        uint32_t n = (nodeID & 0x7fffffffu) >> lg;
        uint64_t w = slots[(size_t)n * W + c].admin;
        uint64_t off = WS_OFF(w);
        float leaf = INFINITY;
        for (uint32_t j = 0; j < WS_CNT(w); j++) {
          uint32_t pid = primIDs[off + j];
          float d = sqr_pp(points + 3 * (size_t)pid, q, fma_mode);
          int take = tie_mode == 1 ? (d < bestD) : (d < bestD || (best >= 0 && d == bestD && (int32_t)pid < best));
          if (take) { bestD = d; best = (int32_t)pid; }
          leaf = fminf(leaf, bestD);
        }
        cull = fminf(cull, leaf);
        nodeID = 0xFFFFFFFFu;
      }
      free(stack);
    }
    ids[i] = best;
    dists[i] = best >= 0 ? bestD : INFINITY;
  }
  return 0;
}

/* fixedBoxQuery over a wide tree (fixedBoxQuery.h:161-277): depth first,
   slots in order, per-prim box test as orc_box_query. */
int orc_wide_box_query(const onode *slots, uint32_t numWide, int W, const uint32_t *primIDs, const obox *boxes,
                       const obox *queryBoxes, uint32_t nq, uint32_t *counts, const uint64_t *offsets, int32_t *ids)
{
  size_t cap = 256;
  uint64_t *stack = (uint64_t *)malloc(sizeof(uint64_t) * cap);
  for (uint32_t qi = 0; qi < nq; qi++) {
    const float *qlo = queryBoxes[qi].lo, *qhi = queryBoxes[qi].hi;
    uint32_t cnt = 0;
    size_t sp = 0;
    uint64_t node = 0;
    uint32_t c = 0;
    while (numWide) {
      const onode *sl = &slots[node * W + c];
      if (WS_VALID(sl->admin) && box_ov(qlo, qhi, sl->lo, sl->hi)) {
        if (WS_CNT(sl->admin) == 0) {
          if (c + 1 < (uint32_t)W) {
            if (sp == cap) { cap *= 2; stack = (uint64_t *)realloc(stack, sizeof(uint64_t) * cap); }
            stack[sp++] = (node << 8) | (c + 1);
          }
          node = WS_OFF(sl->admin);
          c = 0;
          continue;
        }
        uint64_t off = WS_OFF(sl->admin);
        for (uint32_t j = 0; j < WS_CNT(sl->admin); j++) {
          uint32_t pid = primIDs[off + j];
          if (box_ov(qlo, qhi, boxes[pid].lo, boxes[pid].hi)) {
            if (ids) ids[offsets[qi] + cnt] = (int32_t)pid;
            cnt++;
          }
        }
      }
      if (c + 1 < (uint32_t)W) c++;
      else if (sp) { uint64_t e = stack[--sp]; node = e >> 8; c = (uint32_t)(e & 0xFF); }
      else break;
    }
    counts[qi] = cnt;
  }
  free(stack);
  return 0;
}

/* ------------------------------------------------------------------ */
/* point-to-triangle closest point, FP32, as the reference computes it  */
/* (cuBQL/queries/triangles/findClosest.h:56-152), without contraction. */
/* Only compared at a tolerance.                                        */
/* ------------------------------------------------------------------ */
typedef struct { int32_t primID; float sqrDist; float P[3]; } ofcp;

static float dot3f(const float *a, const float *b) { return ((0.0f + a[0] * b[0]) + a[1] * b[1]) + a[2] * b[2]; }
static void sub3f(const float *a, const float *b, float *r) { r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2]; }
static void cross3f(const float *a, const float *b, float *r)
{
  r[0] = a[1] * b[2] - b[1] * a[2];
  r[1] = a[2] * b[0] - b[2] * a[0];
  r[2] = a[0] * b[1] - b[0] * a[1];
}

static int edge_cp(ofcp *res, const float *a, const float *b, const float *p)
{
  float pa[3], ba[3], cp[3], d[3];
  sub3f(p, a, pa);
  sub3f(b, a, ba);
  float t = dot3f(pa, ba) / dot3f(ba, ba);
  t = fminf(fmaxf(t, 0.0f), 1.0f);
  for (int i = 0; i < 3; i++) cp[i] = a[i] + t * ba[i];
  sub3f(cp, p, d);
  float sd = dot3f(d, d);
  if (sd >= res->sqrDist) return 0;
  res->sqrDist = sd;
  memcpy(res->P, cp, sizeof(cp));
  return 1;
}

static int tri_cp(ofcp *res, const float *a, const float *b, const float *c, const float *qp)
{
  float ba[3], ca[3], N[3], t0[3], t1[3], e[3], w[3];
  sub3f(b, a, ba);
  sub3f(c, a, ca);
  cross3f(ba, ca, N);
  int outside = (N[0] == 0.f && N[1] == 0.f && N[2] == 0.f);
  if (!outside) { sub3f(qp, a, t0); cross3f(ba, N, t1); outside = dot3f(t0, t1) >= 0.f; }
  if (!outside) { sub3f(qp, b, t0); sub3f(c, b, e); cross3f(e, N, t1); outside = dot3f(t0, t1) >= 0.f; }
  if (!outside) { sub3f(qp, c, t0); sub3f(a, c, e); cross3f(e, N, t1); outside = dot3f(t0, t1) >= 0.f; }
  if (outside) {
    int r = edge_cp(res, a, b, qp);
    r |= edge_cp(res, b, c, qp);
    r |= edge_cp(res, c, a, qp);
    return r;
  }
  float inv = 1.0f / sqrtf(dot3f(N, N));
  for (int i = 0; i < 3; i++) w[i] = N[i] * inv;
  sub3f(qp, a, t0);
  float sd = dot3f(t0, w);
  float d2 = sd * sd;
  if (d2 >= res->sqrDist) return 0;
  res->sqrDist = d2;
  for (int i = 0; i < 3; i++) res->P[i] = qp[i] - sd * w[i];
  return 1;
}

/* tris: int32 triples into verts (float3).  Not found: id -1, +inf. */
int orc_tri_closest(const onode *nodes, uint32_t numNodes, const uint32_t *primIDs, const int32_t *tris,
                    const float *verts, const float *queries, uint32_t nq, float maxSqr, int32_t *ids,
                    float *dists, float *P)
{
  for (uint32_t qi = 0; qi < nq; qi++) {
    const float *q = queries + 3 * (size_t)qi;
    ofcp res;
    res.primID = -1; res.sqrDist = maxSqr; res.P[0] = res.P[1] = res.P[2] = 0.f;
    if (numNodes) {
      float cull = maxSqr;
      size_t cap = 256, sp = 0;
      stk_e *stack = (stk_e *)malloc(sizeof(stk_e) * cap);
      uint64_t admin = nodes[0].admin;
      for (;;) {
        for (;;) {
          if (ADMIN_CNT(admin) != 0) break;
          uint32_t i0 = (uint32_t)ADMIN_OFF(admin), i1 = i0 + 1;
          float d0 = sqr_pbox(q, nodes[i0].lo, nodes[i0].hi, 0);
          float d1 = sqr_pbox(q, nodes[i1].lo, nodes[i1].hi, 0);
          if (fminf(d0, d1) >= cull) { admin = 0; break; }
          uint32_t farID;
          if (d0 < d1) { admin = nodes[i0].admin; farID = i1; }
          else { admin = nodes[i1].admin; farID = i0; }
          if (fmaxf(d0, d1) < cull) {
            if (sp == cap) { cap *= 2; stack = (stk_e *)realloc(stack, sizeof(stk_e) * cap); }
            stack[sp].idx = farID; stack[sp].dist = fmaxf(d0, d1); sp++;
          }
        }
        if (ADMIN_CNT(admin) != 0) {
          uint64_t off = ADMIN_OFF(admin);
          uint32_t cnt = ADMIN_CNT(admin);
          float leaf = INFINITY;
          for (uint32_t j = 0; j < cnt; j++) {
            uint32_t pid = primIDs[off + j];
            const int32_t *t = tris + 3 * (size_t)pid;
            if (tri_cp(&res, verts + 3 * (size_t)t[0], verts + 3 * (size_t)t[1], verts + 3 * (size_t)t[2], q))
              res.primID = (int32_t)pid;
            leaf = fminf(leaf, res.sqrDist);
          }
          cull = fminf(cull, leaf);
        }
        int popped = 0;
        while (sp) {
          stk_e e = stack[--sp];
          if (e.dist <= cull) { admin = nodes[e.idx].admin; popped = 1; break; }
        }
        if (!popped) break;
      }
      free(stack);
    }
    ids[qi] = res.primID;
    dists[qi] = res.primID >= 0 ? res.sqrDist : INFINITY;
    if (P) memcpy(P + 3 * (size_t)qi, res.P, sizeof(res.P));
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* FP64 closest point on a triangle with barycentric weights            */
/* (region classification of Ericson, Real-Time Collision Detection,    */
/* sec. 5.1.5); degenerate triangles fall back to the three edges.      */
/* ------------------------------------------------------------------ */
static double dot3d(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void seg_cp_d(const double *a, const double *b, const double *p, double *t_out, double *d2_out)
{
  double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, ap[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
  double L = dot3d(ab, ab), t = L > 0 ? dot3d(ap, ab) / L : 0.0;
  if (t < 0) t = 0; if (t > 1) t = 1;
  double d[3] = {a[0] + t * ab[0] - p[0], a[1] + t * ab[1] - p[1], a[2] + t * ab[2] - p[2]};
  *t_out = t;
  *d2_out = dot3d(d, d);
}

/* returns squared distance; w[3] barycentric weights of the closest point */
double orc_tri_cp_f64(const double *a, const double *b, const double *c, const double *p, double *w)
{
  double ab[3], ac[3], ap[3], bp[3], cp[3];
  for (int i = 0; i < 3; i++) {
    ab[i] = b[i] - a[i]; ac[i] = c[i] - a[i]; ap[i] = p[i] - a[i]; bp[i] = p[i] - b[i]; cp[i] = p[i] - c[i];
  }
  double d1 = dot3d(ab, ap), d2 = dot3d(ac, ap), d3 = dot3d(ab, bp), d4 = dot3d(ac, bp);
  double d5 = dot3d(ab, cp), d6 = dot3d(ac, cp);
  double vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
  double wa, wb, wc;
  if (d1 <= 0 && d2 <= 0) { wa = 1; wb = 0; wc = 0; }
  else if (d3 >= 0 && d4 <= d3) { wa = 0; wb = 1; wc = 0; }
  else if (vc <= 0 && d1 >= 0 && d3 <= 0) { double v = d1 / (d1 - d3); wa = 1 - v; wb = v; wc = 0; }
  else if (d6 >= 0 && d5 <= d6) { wa = 0; wb = 0; wc = 1; }
  else if (vb <= 0 && d2 >= 0 && d6 <= 0) { double t = d2 / (d2 - d6); wa = 1 - t; wb = 0; wc = t; }
  else if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    double t = (d4 - d3) / ((d4 - d3) + (d5 - d6)); wa = 0; wb = 1 - t; wc = t;
  } else if (va + vb + vc != 0.0) {
    double den = 1.0 / (va + vb + vc); wb = vb * den; wc = vc * den; wa = 1 - wb - wc;
  } else {
    double t, dd, best = INFINITY;
    wa = 1; wb = 0; wc = 0;
    seg_cp_d(a, b, p, &t, &dd); if (dd < best) { best = dd; wa = 1 - t; wb = t; wc = 0; }
    seg_cp_d(b, c, p, &t, &dd); if (dd < best) { best = dd; wa = 0; wb = 1 - t; wc = t; }
    seg_cp_d(c, a, p, &t, &dd); if (dd < best) { best = dd; wa = t; wb = 0; wc = 1 - t; }
  }
  double X[3], d[3];
  for (int i = 0; i < 3; i++) { X[i] = wa * a[i] + wb * b[i] + wc * c[i]; d[i] = p[i] - X[i]; }
  if (w) { w[0] = wa; w[1] = wb; w[2] = wc; }
  return dot3d(d, d);
}

/* FP64 brute force over all triangles: sqr distance and the lowest
   triangle id attaining it */
int orc_tri_brute_f64(const int32_t *tris, const float *verts, uint32_t nt, const float *queries,
                      uint32_t nq, double *d2, int32_t *ids)
{
  for (uint32_t qi = 0; qi < nq; qi++) {
    double p[3] = {queries[3 * (size_t)qi], queries[3 * (size_t)qi + 1], queries[3 * (size_t)qi + 2]};
    double best = INFINITY;
    int32_t bid = -1;
    for (uint32_t t = 0; t < nt; t++) {
      double v[3][3];
      for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++) v[k][i] = verts[3 * (size_t)tris[3 * (size_t)t + k] + i];
      double dd = orc_tri_cp_f64(v[0], v[1], v[2], p, NULL);
      if (dd < best) { best = dd; bid = (int32_t)t; }
    }
    d2[qi] = best;
    ids[qi] = bid;
  }
  return 0;
}

/* FP64 analytic adjoint of sqrDist(q, tri[primID]) for each query:
   d/dq = 2 (q - X), d/dv_k = -2 w_k (q - X), X = sum_k w_k v_k the
   closest point (envelope theorem: the optimal barycentric weights are
   constrained to a fixed simplex).  gradV accumulates per vertex. */
int orc_tri_grad_f64(const int32_t *tris, const float *verts, const float *queries, uint32_t nq,
                     const int32_t *primIDs, const float *gradSqr, double *gradQ, double *gradV)
{
  for (uint32_t qi = 0; qi < nq; qi++) {
    int32_t t = primIDs[qi];
    double *gq = gradQ + 3 * (size_t)qi;
    gq[0] = gq[1] = gq[2] = 0;
    if (t < 0) continue;
    double p[3] = {queries[3 * (size_t)qi], queries[3 * (size_t)qi + 1], queries[3 * (size_t)qi + 2]};
    double v[3][3], w[3];
    for (int k = 0; k < 3; k++)
      for (int i = 0; i < 3; i++) v[k][i] = verts[3 * (size_t)tris[3 * (size_t)t + k] + i];
    orc_tri_cp_f64(v[0], v[1], v[2], p, w);
    double g = gradSqr[qi];
    for (int i = 0; i < 3; i++) {
      double X = w[0] * v[0][i] + w[1] * v[1][i] + w[2] * v[2][i];
      double r = 2.0 * (p[i] - X) * g;
      gq[i] = r;
      for (int k = 0; k < 3; k++) gradV[3 * (size_t)tris[3 * (size_t)t + k] + i] -= w[k] * r;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* rebinning Morton builder, 30-bit keys (cuBQL/builder/cuda/          */
/* rebinMortonBuilder.h:1161-1488), restated level-synchronously with   */
/* children allocated in node order (canonical BFS-like numbering).     */
/* ------------------------------------------------------------------ */
static uint32_t spread3_10(uint32_t x)
{
  uint32_t r = 0;
  for (int i = 0; i < 10; i++) r |= ((x >> i) & 1u) << (3 * i);
  return r;
}

/* Quantizer<float,3> with 10 bits (rebinMortonBuilder.h:33-61) over a
   centroid domain lo/hi */
static uint32_t morton30(const float c[3], const float lo[3], const float hi[3])
{
  float sz[3];
  for (int d = 0; d < 3; d++) sz[d] = hi[d] - lo[d];
  float ext = fmaxf(fmaxf(sz[0], sz[1]), sz[2]);
  float scale = 1024.0f * (1.0f / fmaxf(ext, 1e-20f));
  uint32_t cell[3];
  for (int d = 0; d < 3; d++) {
    float f = (c[d] - lo[d]) * scale;
    uint32_t u = !(f > 0.0f) ? 0u : (f >= 4294967296.0f ? 0xFFFFFFFFu : (uint32_t)f);
    cell[d] = u < 1023u ? u : 1023u;
  }
  return spread3_10(cell[0]) | (spread3_10(cell[1]) << 1) | (spread3_10(cell[2]) << 2);
}

/* findSplit on 32-bit keys (rebinMortonBuilder.h:566-590) */
static int find_split32(int64_t *split, const uint32_t *keys, int64_t begin, int64_t end)
{
  uint32_t fk = keys[begin], lk = keys[end - 1];
  if (fk == lk) return 0;
  int nm = __builtin_clz(fk ^ lk);
  uint32_t sk = (uint32_t)(lk & (0xFFFFFFFFull << (31 - nm)));
  while (end > begin) {
    int64_t mid = (begin + end) / 2;
    if (keys[mid] < sk) begin = mid + 1; else end = mid;
  }
  *split = begin;
  return 1;
}

/* centroid domain of prims[b..e) */
static void range_domain(const obox *boxes, const uint32_t *ids, uint64_t b, uint64_t e, float lo[3], float hi[3])
{
  for (int d = 0; d < 3; d++) { lo[d] = INFINITY; hi[d] = -INFINITY; }
  for (uint64_t i = b; i < e; i++) {
    float c[3];
    box_center(&boxes[ids[i]], c);
    for (int d = 0; d < 3; d++) { lo[d] = fminf(lo[d], c[d]); hi[d] = fmaxf(hi[d], c[d]); }
  }
}

typedef struct { uint32_t a, b; uint8_t open; } rnode; /* open: [a,b); done: {offset a, count b} */

int orc_rebin_build(const obox *boxes, uint32_t n, int makeLeafThreshold, int maxAllowedLeafSize, onode *nodes,
                    uint32_t *primIDs, uint32_t *numNodes, uint32_t *numPrims)
{
  int thr = makeLeafThreshold > 0
              ? (makeLeafThreshold < maxAllowedLeafSize ? makeLeafThreshold : maxAllowedLeafSize)
              : 1;
  int32_t cbLo[3], cbHi[3];
  for (int d = 0; d < 3; d++) { cbLo[d] = enc_f(FLT_MAX); cbHi[d] = enc_f(-FLT_MAX); }
  uint32_t nv = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (box_empty(&boxes[i])) continue;
    float c[3];
    box_center(&boxes[i], c);
    for (int d = 0; d < 3; d++) {
      int32_t e = enc_f(c[d]);
      if (e < cbLo[d]) cbLo[d] = e;
      if (e > cbHi[d]) cbHi[d] = e;
    }
    nv++;
  }
  if (nv == 0) { *numNodes = 0; *numPrims = 0; return 0; }
  float glo[3], ghi[3];
  for (int d = 0; d < 3; d++) { glo[d] = dec_f(cbLo[d]); ghi[d] = dec_f(cbHi[d]); }
  uint64_t *k64 = (uint64_t *)malloc(sizeof(uint64_t) * nv);
  uint32_t *keys = (uint32_t *)malloc(sizeof(uint32_t) * nv);
  uint32_t j = 0;
  for (uint32_t i = 0; i < n; i++) {               /* computeUnsortedKeysAndPrimIDs (:503-533) */
    if (box_empty(&boxes[i])) continue;
    float c[3];
    box_center(&boxes[i], c);
    k64[j] = morton30(c, glo, ghi);
    primIDs[j] = i;
    j++;
  }
  stable_sort_pairs(k64, primIDs, nv, 0, 32);      /* SortPairs bits [0,32) (:1235-1257) */
  for (uint32_t i = 0; i < nv; i++) keys[i] = (uint32_t)k64[i];
  uint64_t cap = 2ull * nv + 2;
  rnode *t = (rnode *)calloc(cap, sizeof(rnode));
  t[0].a = 0; t[0].b = nv; t[0].open = 1;          /* initNodes (:674-687) */
  uint64_t alloc = 2;
  /* broad phase with rebinning restarts (:1283-1393); the first pass
     sees the root only, a restart sees every node allocated so far */
  uint64_t done = 0, upTo = 1;
  int restart = 0;
  for (;;) {
    while (done < upTo) {
      uint64_t end = upTo;
      for (uint64_t id = done; id < end; id++) {
        if (id == 1 || !t[id].open) continue;
        uint32_t b = t[id].a, e = t[id].b, size = e - b;
        int64_t split;
        if ((int64_t)size <= thr) { t[id].a = b; t[id].b = size; t[id].open = 0; }
        else if (size <= 32) { /* leaves broad phase, stays open */ }
        else if (!find_split32(&split, keys, b, e)) { /* rebin job, stays open */ }
        else {
          uint64_t c = alloc; alloc += 2;
          t[c].a = b; t[c].b = (uint32_t)split; t[c].open = 1;
          t[c + 1].a = (uint32_t)split; t[c + 1].b = e; t[c + 1].open = 1;
          t[id].a = (uint32_t)c; t[id].b = 0; t[id].open = 0;
        }
      }
      done = end;
      upTo = alloc;
    }
    /* rebin every still-open node larger than the broad-phase limit; the
       reference would restart forever on a run whose centroid bounds are
       narrower than 1e-20 but not a point: from depth 40 on, runs are
       keyed by position (the library's documented cap) */
    int jobs = 0;
    restart++;
    const int atCap = restart >= 40;
    for (uint64_t id = 0; id < alloc; id++) {
      if (id == 1 || !t[id].open) continue;
      uint32_t b = t[id].a, e = t[id].b;
      if (e - b <= 32) continue;
      jobs++;
      float lo[3], hi[3];
      range_domain(boxes, primIDs, b, e, lo, hi);
      int degenerate = lo[0] == hi[0] && lo[1] == hi[1] && lo[2] == hi[2];
      uint64_t *nk = (uint64_t *)malloc(sizeof(uint64_t) * (e - b));
      uint32_t *nid = (uint32_t *)malloc(sizeof(uint32_t) * (e - b));
      for (uint32_t i = b; i < e; i++) {           /* rebinCreateNewKeysAndPrimIDs (:1022-1063) */
        float c[3];
        box_center(&boxes[primIDs[i]], c);
        nk[i - b] = (degenerate || atCap) ? (i - b) : morton30(c, lo, hi);
        nid[i - b] = primIDs[i];
      }
      stable_sort_pairs(nk, nid, e - b, 0, 32);    /* sort by (range, morton), stable */
      for (uint32_t i = b; i < e; i++) { keys[i] = (uint32_t)nk[i - b]; primIDs[i] = nid[i - b]; }
      free(nk);
      free(nid);
    }
    if (!jobs) break;
    done = 0;
    upTo = alloc;
  }
  /* thread phase (:766-872, :1413-1426) */
  {
    done = 0;
    while (done < alloc) {
      uint64_t end = alloc;
      for (uint64_t id = done; id < end; id++) {
        if (id == 1 || !t[id].open) continue;
        uint32_t b = t[id].a, e = t[id].b, size = e - b;
        int64_t split;
        int doSplit = 0;
        if ((int64_t)size <= thr) { t[id].a = b; t[id].b = size; t[id].open = 0; continue; }
        if (find_split32(&split, keys, b, e)) doSplit = 1;
        else {
          float lo[3], hi[3];
          range_domain(boxes, primIDs, b, e, lo, hi);
          int degenerate = lo[0] == hi[0] && lo[1] == hi[1] && lo[2] == hi[2];
          for (uint32_t i = b; i < e; i++) {
            float c[3];
            box_center(&boxes[primIDs[i]], c);
            keys[i] = degenerate ? (i - b) : morton30(c, lo, hi);
          }
          for (uint32_t x = b; x < e; x++)         /* bubbleSort (:756-764), not stable */
            for (uint32_t y = x + 1; y < e; y++)
              if (keys[y] < keys[x]) {
                uint32_t tk = keys[x]; keys[x] = keys[y]; keys[y] = tk;
                uint32_t ti = primIDs[x]; primIDs[x] = primIDs[y]; primIDs[y] = ti;
              }
          if (find_split32(&split, keys, b, e)) doSplit = 1;
          else { t[id].a = b; t[id].b = size; t[id].open = 0; continue; }
        }
        if (doSplit) {
          uint64_t c = alloc; alloc += 2;
          t[c].a = b; t[c].b = (uint32_t)split; t[c].open = 1;
          t[c + 1].a = (uint32_t)split; t[c + 1].b = e; t[c + 1].open = 1;
          t[id].a = (uint32_t)c; t[id].b = 0; t[id].open = 0;
        }
      }
      done = end;
    }
  }
  for (uint64_t i = 0; i < alloc; i++) {
    memset(&nodes[i], 0, sizeof(onode));
    nodes[i].admin = (i == 1) ? 0 : ADMIN(t[i].a, t[i].b);
  }
  *numNodes = (uint32_t)alloc;
  *numPrims = nv;
  refit_tree(nodes, *numNodes, primIDs, boxes);
  free(t);
  free(keys);
  free(k64);
  return 0;
}
