#!/usr/bin/env python
"""Benchmark of the BVH build-and-query path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (the 10M-point configuration): a step is one BVH build,
leaf threshold 1, over 10,000,000 uniformly distributed points (seeded,
U[0,1]^3), inputs already in HBM.  Ours is the Morton (radix, 63-bit)
builder; `value` is build throughput in Mprims/s summed over ranks (each
rank builds its own 10M-point set: weak scaling, no data-path collective).
The line also carries, measured in the same run:
  * e2e        the same build through the public API from pinned host
               boxes, the tree copied back to host every step;
  * roofline   for the dominant kernel (CUDA events on the library's own
               stream via the libbq phase profiler), against the measured
               HBM copy bandwidth, and for every component below;
  * components spatial-median build, 10M closest-point and 10M kNN(k=16)
               queries on uniform and Gaussian-mixture points,
               triangle-mesh distance forward+adjoint, the batched
               configurations; the reference's own GPU kernels compiled
               for sm_100a are timed on the same inputs by the reference arm;
  * cpu_baseline the reference's host builder (cpuBuilder) on the same 10M
               points, one core.
Inputs (240 MB of boxes) are larger than the 126 MB L2, so no flush is
needed between steps.

--impl reference times the reference's own CPU build path (cpuBuilder,
compiled from the reference's sources into oracle/_ref) on this host with
all cores: every step runs one concurrent 10M-point build per host thread.
It prints the same metric and config, and never loads this repository's
library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "build Mprims/s + kNN/closest-pt Mqueries/s @10M pts; batched fwd+bwd queries/s"
N_POINTS = 10_000_000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_POINTS)
    ap.add_argument("--no-components", action="store_true")
    ap.add_argument("--only-queries", action="store_true",
                    help="build one tree, then time closest-point and kNN(16) queries only (the short program "
                         "the query ncu captures run)")
    ap.add_argument("--queries", type=int, default=N_POINTS, help="query count for --only-queries/-tri/-wide")
    ap.add_argument("--only-tri", action="store_true",
                    help="triangle forward only: icosphere of --mesh-level over --queries queries in [-1.5,1.5]^3 "
                         "(the short program the triangle ncu captures run)")
    ap.add_argument("--mesh-level", type=int, default=8)
    ap.add_argument("--only-wide", action="store_true",
                    help="build one 4-wide tree, then time wide closest-point queries only")
    ap.add_argument("--only-build", action="store_true",
                    help="time the build loop only (no profile pass, e2e, components or CPU leg): "
                         "the short program the ncu captures run")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(", ") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        mine = [r for r in rows if self.uuid and r[0].strip() in self.uuid] or rows
        sm = [float(r[1].split()[0]) for r in mine if len(r) > 2 and r[1].split()[0].replace(".", "").isdigit()]
        mx = [float(r[2].split()[0]) for r in mine if len(r) > 2 and r[2].split()[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in mine:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(mine)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(units_per_rank, ms_max, world):
    """Whole-job throughput in M units/s: every rank processes the same
    number of units; the job takes as long as its slowest rank."""
    return world * units_per_rank / ms_max / 1e3


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def workloads():
    """cubql_b200/workloads.py loaded by path: the seeded generators, without
    the package (whose import loads libbq.so)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bq_workloads", os.path.join(ROOT, "cubql_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def bench_config(n, seed):
    """The workload both arms run (identical in both lines)."""
    return {"workload": f"BVH build, leaf threshold 1, over {n} uniform points U[0,1]^3 (seeded)",
            "points_per_gpu": n, "seed": seed,
            "l2": "inputs (240 MB boxes per GPU) larger than the 126 MB L2; no flush"}


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    W = workloads()
    from oracle.oracle import RefCPU, have_ref_cpu, Oracle
    n = args.n
    boxes = W.point_boxes(W.uniform_points(n, W.SEED_DATA))
    threads = max(1, min(os.cpu_count() or 1, 16))
    if have_ref_cpu():
        r = RefCPU()
        kind = "reference"
        run = lambda: r.build_throughput(boxes, 0, threads, 1)  # noqa: E731
    else:
        o = Oracle()
        kind = "port"
        threads = 1
        run = lambda: _timed(lambda: o.cpu_build(boxes, 0))  # noqa: E731
    for _ in range(args.warmup):
        run()
    secs = [run() for _ in range(args.steps)]
    t = sum(secs) / len(secs)
    value = threads * n / t / 1e6
    sample = f"{threads} concurrent cpuBuilder builds (spatial median, leaf 1) of all {n} points per step"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mprims/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(n, W.SEED_DATA),
            "impl_detail": {"builder": "reference cpuBuilder (host, single-threaded by design), one build per "
                                       "host thread", "threads": threads},
            "cpu_baseline": {"value": value, "unit": "Mprims/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Mprims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_components:
        line["reference_components"] = reference_components(W, n)
    print(json.dumps(line))


def reference_components(W, n):
    """The reference's own GPU code (compiled for sm_100a from its sources
    into oracle/_ref) and host code on the workloads of our arm's
    components: the same seeds and sizes."""
    import numpy as np
    from oracle.oracle import RefGPU, have_ref_gpu
    comp = {}
    pts_np = W.uniform_points(n, W.SEED_DATA)
    reference_gpu(comp, pts_np, W)
    comp["c1_reference"] = c1_reference(W, pts_np)
    if have_ref_gpu():
        r = RefGPU()
        verts, tris = W.icosphere(8)
        tv = verts[tris]
        tbox = np.concatenate([tv.min(1), tv.max(1)], 1).astype(np.float32)
        comp["sah_build_triangles"] = {"triangles": int(len(tris)),
                                       "reference_sahBuilder_ms": r.time_build_boxes(RefGPU.SAH, tbox, 0, reps=2),
                                       "reference_gpuBuilder_elh_ms": r.time_build_boxes(RefGPU.ELH, tbox, 0,
                                                                                        reps=2)}
        tq = W.uniform_points(4_000_000, W.SEED_QUERIES, -1.5, 1.5)
        comp["triangle_distance"] = {"triangles": int(len(tris)), "queries": int(len(tq)),
                                     "reference_findClosest_ms": r.time_tri(RefGPU.RADIX, tris, verts, tq, reps=2),
                                     "note": "reference triangles::findClosest kernel, one thread per query, over "
                                             "its radixBuilder tree of the triangle boxes (build not timed)"}
        del tq
        g = W.gmm_points(n)
        gq = W.gmm_points(n, sample_seed=W.SEED_GMM_QUERIES)
        pb, ob, qb, qob = W.cloud_batch()
        comp["batched_knn_512_clouds"] = {"clouds": len(ob) - 1, "points": int(len(pb)), "queries": int(len(qb)),
                                          "k": 16,
                                          "reference_per_cloud_loop_ms": r.time_batched_knn(pb, ob, qb, qob, 16),
                                          "note": "for every cloud: the reference's radixBuilder, its findKNN "
                                                  "kernel over the cloud's queries, cuda::free"}
        del pb, qb
        comp["gmm10m"] = {"points": n, "queries": n,
                          "reference_radixBuilder_ms": r.time_build(RefGPU.RADIX, g, 0, reps=2),
                          "reference_gpuBuilder_leaf8_ms": r.time_build(RefGPU.SPATIAL_MEDIAN, g, 8, reps=2),
                          "reference_findClosest_ms": r.time_query(RefGPU.RADIX, g, gq, 0, reps=2),
                          "reference_findKNN16_ms": r.time_query(RefGPU.RADIX, g, gq, 16, reps=2)}
    return comp


def _timed(fn):
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
HBM_FALLBACK = 6650.0


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/ncu_summary.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_summary.json")) as f:
            return json.load(f).get(kernel, {}).get("dram_bytes_per_launch_scaled")
    except Exception:
        return None


class CBuild:
    """Direct C-ABI build loop with the library's own stream-ordered
    allocator (no Python in the way between steps)."""

    def __init__(self, bq, boxes, n):
        import ctypes
        self.bq, self.ctypes = bq, ctypes
        self.boxes, self.n = boxes, n
        self.cfg = bq.bq_build_config(1 << 15, 0, 0)

    def step(self, stream):
        c = self.bq.bq_bvh3f()
        rc = self.bq._lib.bq_build_morton63_f3(self.ctypes.byref(c), self.ctypes.c_void_p(self.boxes.data_ptr()),
                                               self.n, self.ctypes.byref(self.cfg), None, stream)
        self.bq._check(rc)
        self.bq._check(self.bq._lib.bq_free_f3(self.ctypes.byref(c), None, stream))


def time_loop(fn, steps, warmup, world):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    return e0.elapsed_time(e1) / steps


# algorithmic bytes per element of each libbq phase (Morton build)
PHASE_BYTES = {
    "morton.bounds": 24,            # box read
    "morton.keygen": 24 + 12,       # box read, key + id written
    "sort.onesweep64": 24,          # per pass: key+id read, key+id written
    "morton.runs": 8 + 1,           # keys read, split level written (+ rewrites inside runs)
    "morton.agg_local": 4 + 24 + 1 + 64 + 32,  # id, box gather, level, 2N nodes written, siblings read
    # morton.agg_global: the few chunk-crossing nodes, negligible bytes
}


def hbm_frac(nbytes, ms, peak):
    gbs = nbytes / ms / 1e6
    return {"bound": "hbm", "alg_bytes": int(nbytes), "achieved": gbs, "peak": peak, "unit": "GB/s",
            "frac": gbs / peak}


def query_roofline(counts, nq, out_bytes, prim_bytes, ms, peak, compulsory):
    """Touched bytes of a traversal batch from its visit counts: 64 B per
    inner node expanded (both 32-byte children), 16 B per admin load,
    prim_bytes per prim tested, and each query's input (12 B) and output;
    beside it the compulsory bytes (every input and the tree read once)."""
    touched = 64 * counts["inner_nodes"] + 16 * counts["admin_loads"] + prim_bytes * counts["prims"] + \
        nq * (12 + out_bytes)
    r = hbm_frac(touched, ms, peak)
    r.update({"model": "touched bytes B_t (mostly served from L1/L2, so frac may exceed 1)",
              "visit_counts": counts, "compulsory_bytes": int(compulsory),
              "compulsory_frac": compulsory / ms / 1e6 / peak})
    return r


def morton_build_bytes(n, num_nodes):
    """The fixed accounting model of a Morton build: 288 B per prim + 64 B per node."""
    return 288 * n + 64 * num_nodes


def open_prim_levels(nodes_f32):
    """Sum over levels of the prims still in open (inner) nodes: the sum of
    the prim counts of all inner nodes, from the tree's admin words."""
    import numpy as np
    adm = nodes_f32.view(np.uint64).reshape(-1, 4)[:, 3]
    cnt = (adm >> np.uint64(48)).astype(np.int64)
    off = (adm & np.uint64(0xFFFFFFFFFFFF)).astype(np.int64)
    size = np.where(cnt > 0, cnt, 0)
    # parents before children is not guaranteed: iterate until sizes settle (depth passes)
    inner = np.nonzero(cnt == 0)[0]
    inner = inner[inner != 1]
    for _ in range(200):
        new = size.copy()
        new[inner] = size[off[inner]] + size[off[inner] + 1]
        if np.array_equal(new, size):
            break
        size = new
    return int(size[inner].sum())


def components(bq, W, torch, pts_np, tp, boxes_t, comp):
    import numpy as np
    n = len(pts_np)
    stream = torch.cuda.current_stream()

    def ev_time(fn, reps=3, warm=1):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    # spatial-median build, leaf 8
    def smb():
        bq.gpuBuilder(boxes_t, bq.BuildConfig(makeLeafThreshold=8)).free()
    ms = ev_time(smb)
    peak, _ = hbm_peak()
    smt = bq.gpuBuilder(boxes_t, bq.BuildConfig(makeLeafThreshold=8))
    sm_nodes = smt.nodes_tensor().cpu().numpy()
    smt.free()
    a_sum = open_prim_levels(sm_nodes)
    comp["spatial_median_build"] = {"ms": ms, "Mprims_s": n / ms / 1e3, "leaf": 8,
                                    "vs_published_reference_13ms": 13.0 / ms,
                                    "roofline": dict(hbm_frac(n * (24 + 28) + 40 * a_sum + 64 * len(sm_nodes), ms, peak),
                                                     model="N*(24+28) + sum_levels A_l*(24+8+8) + 64*M",
                                                     sum_levels_open_prims=a_sum, nodes=len(sm_nodes))}
    with bq.profile() as prof:
        smb()
    comp["spatial_median_build"]["phases_ms"] = {k: round(v[1], 4) for k, v in prof.table.items()}

    def smb1():
        bq.gpuBuilder(boxes_t, bq.BuildConfig(makeLeafThreshold=1)).free()
    ms = ev_time(smb1)
    comp["spatial_median_build_leaf1"] = {"ms": ms, "Mprims_s": n / ms / 1e3, "leaf": 1}

    # rebinning Morton-30 build, leaf 1
    def rbb():
        bq.cuda.rebinRadixBuilder(boxes_t).free()
    ms = ev_time(rbb)
    comp["rebin_morton30_build"] = {"ms": ms, "Mprims_s": n / ms / 1e3, "leaf": 1}
    with bq.profile() as prof:
        rbb()
    comp["rebin_morton30_build"]["phases_ms"] = {k: round(v[1], 4) for k, v in prof.table.items()}
    # queries on the Morton tree (leaf 1)
    bvh = bq.cuda.radixBuilder(boxes_t)
    qs = torch.from_numpy(W.uniform_points(n, W.SEED_QUERIES)).cuda()
    ms = ev_time(lambda: bq.points.findClosest(bvh, tp, qs))
    nn = bvh.numNodes
    cpc = bq.points.visitCounts(bvh, tp, qs, 0)
    comp["closest_point"] = {"ms": ms, "Mqueries_s": n / ms / 1e3, "queries": n,
                             "roofline": query_roofline(cpc, n, 8, 16, ms, peak, n * 20 + 32 * nn + 16 * n)}
    ms = ev_time(lambda: bq.points.findKNN(bvh, tp, qs, 16))
    knc = bq.points.visitCounts(bvh, tp, qs, 16)
    # the warp-cooperative form: a group of lanes per query, the top-k list one candidate per lane
    lane_ms = {g: ev_time(lambda: bq.points.findKNN(bvh, tp, qs, 16, qcfg=bq.query_config(lanesPerQuery=g)))
               for g in (16, 32)}
    comp["knn16"] = {"ms": ms, "Mqueries_s": n / ms / 1e3, "queries": n, "k": 16,
                     "roofline": query_roofline(knc, n, 8 * 16 + 4, 16, ms, peak, n * (12 + 132) + 32 * nn + 16 * n),
                     "lane_group_ms": {f"lanesPerQuery={g}": v for g, v in lane_ms.items()}}
    with bq.profile() as prof:
        bq.points.findClosest(bvh, tp, qs)
        bq.points.findKNN(bvh, tp, qs, 16)
    comp["query_phases_ms"] = {k: round(v[1], 4) for k, v in prof.table.items()}
    # the single-tree autotuner's launch shape for the same workloads (build + query)
    from cubql_b200 import tuning
    for name, kk in (("closest_point", 0), ("knn16", 16)):
        t = tuning.tuned_query(boxes_t, tp, qs, kk)
        tcfg = bq.BuildConfig(makeLeafThreshold=t["makeLeafThreshold"])
        tt = bq.cuda.radixBuilder(boxes_t, tcfg)
        qc = tuning.query_config_of(t)
        run = (lambda: bq.points.findClosest(tt, tp, qs, qcfg=qc)) if kk == 0 else \
            (lambda: bq.points.findKNN(tt, tp, qs, kk, qcfg=qc))
        ms_t = ev_time(run)
        tt.free()
        comp[name]["tuned"] = {k: v for k, v in t.items() if k != "key"}
        comp[name]["tuned_query_ms"] = ms_t
    # wide trees: gpuBuilder(WideBVH<float,3,W>) with the default config (leaf 1) and closest point
    for width in (4, 8):
        ms_b = ev_time(lambda: bq.gpuBuilderWide(boxes_t, width).free())
        wb = bq.gpuBuilderWide(boxes_t, width)
        ms_q = ev_time(lambda: bq.points.findClosest(wb, tp, qs))
        with bq.profile() as prof:
            bq.gpuBuilderWide(boxes_t, width).free()
            bq.points.findClosest(wb, tp, qs)
        comp[f"wide{width}"] = {"build_ms": ms_b, "build_Mprims_s": n / ms_b / 1e3, "wide_nodes": wb.numNodes,
                                "closest_point_ms": ms_q, "Mqueries_s": n / ms_q / 1e3, "queries": n,
                                "phases_ms": {k: round(v[1], 4) for k, v in prof.table.items()}}
        wb.free()
    del qs
    # nearest other point of every data point (findClosest_exludeSelf)
    ms = ev_time(lambda: bq.points.findClosest_exludeSelf(bvh, tp, tp))
    comp["closest_point_exclude_self"] = {"ms": ms, "Mqueries_s": n / ms / 1e3, "queries": n}
    # fixed-box queries: 1M boxes of half size 0.00585 (about 16 points each): one traversal into
    # slab rows + scan + gather, and the two-pass form (count + scan + fill) beside it
    qb = box_queries(W, 1_000_000)
    qbt = torch.from_numpy(qb).cuda()
    ms = ev_time(lambda: bq.fixedBoxQuery.findPrims(bvh, boxes_t, qbt))
    ms2 = ev_time(lambda: bq.fixedBoxQuery.findPrims(bvh, boxes_t, qbt, slabCap=0))
    off, _ = bq.fixedBoxQuery.findPrims(bvh, boxes_t, qbt)
    comp["box_query"] = {"ms": ms, "Mqueries_s": len(qb) / ms / 1e3, "queries": len(qb),
                         "results": int(off[-1]), "half_size": BOX_HALF, "two_pass_ms": ms2,
                         "path": "fixedBoxQuery.findPrims: slab kernel (one traversal, 64 ids per query kept), "
                                 "cumsum, host read of the total, gather kernel (longer queries traversed again)"}
    del qbt, off
    bvh.free()
    # triangle-mesh distance forward + adjoint (icosphere, 1,310,720 triangles, 4M queries)
    verts, tris = W.icosphere(8)
    tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    tq = torch.from_numpy(W.uniform_points(4_000_000, W.SEED_QUERIES, -1.5, 1.5)).cuda()
    g1 = torch.ones(len(tq), device="cuda")

    def fwd():
        b = bq.cuda.radixBuilder(bq.triangles.boxes(tt, tv))
        out = bq.triangles.findClosest(b, tt, tv, tq)
        b.free()
        return out

    def fwdbwd():
        ids, d, _ = fwd()
        bq.triangles.distanceBackward(tt, tv, tq, ids, g1)

    # SAH and spatial-median builds over the triangle boxes (the SAH builder's use case)
    tbox = bq.triangles.boxes(tt, tv)
    ms_sah = ev_time(lambda: bq.cuda.sahBuilder(tbox).free())
    ms_elh = ev_time(lambda: bq.gpuBuilder(tbox, bq.BuildConfig().enableELH()).free())
    ms_smt = ev_time(lambda: bq.gpuBuilder(tbox).free())
    with bq.profile() as prof:
        bq.cuda.sahBuilder(tbox).free()
    comp["sah_build_triangles"] = {"triangles": int(len(tris)), "ms": ms_sah, "Mprims_s": len(tris) / ms_sah / 1e3,
                                   "spatial_median_ms": ms_smt, "elh_ms": ms_elh,
                                   "phases_ms": {k: round(v[1], 4) for k, v in prof.table.items()}}
    tb = bq.cuda.radixBuilder(tbox)
    ms_f = ev_time(lambda: bq.triangles.findClosest(tb, tt, tv, tq))
    ids, dsq, _ = bq.triangles.findClosest(tb, tt, tv, tq)
    ms_b = ev_time(lambda: bq.triangles.distanceBackward(tt, tv, tq, ids, g1))
    other_trees = tri_forward_other_trees(bq, torch, tbox, tt, tv, tq, ids, dsq, ev_time)
    h = 1e-3

    def fd():  # forward + central differences for the query gradient: 7 forwards
        bq.triangles.findClosest(tb, tt, tv, tq)
        for a in range(3):
            for s in (h, -h):
                qq = tq.clone()
                qq[:, a] += s
                bq.triangles.findClosest(tb, tt, tv, qq)
    ms_fd = ev_time(fd, reps=2)
    nq, nv, nt = len(tq), len(verts), len(tris)
    trc = bq.triangles.visitCounts(tb, tt, tv, tq)
    # forward: per triangle tested its id (4), index triple (12) and 3 vertices (36); output id, sqrDist, P
    fwd_roof = query_roofline(trc, nq, 20, 52, ms_f, peak, nq * 32 + 32 * tb.numNodes + 52 * nt)
    # adjoint: pairs kernel (q, id, g, triangle, vertices read; gradQ, 3 keys, 3 values, 3 contributions written),
    # 3 sort passes of the 3Q (u32, u32) pairs + histogram, the reduce (sorted pairs, contributions) and gradV
    bwd_bytes = nq * (12 + 4 + 4 + 12 + 36 + 12 + 12 + 12 + 36) + 3 * nq * (3 * 16 + 4) + 3 * nq * (8 + 12) + 12 * nv
    comp["triangle_distance"] = {"triangles": int(nt), "queries": int(nq), "forward_ms": ms_f,
                                 "backward_ms": ms_b, "fwd_bwd_queries_s": nq / (ms_f + ms_b) * 1e3,
                                 "forward_plus_fd_ms": ms_fd, "speedup_vs_forward_plus_fd": ms_fd / (ms_f + ms_b),
                                 "fd_baseline": "forward + central differences of the query coordinates only "
                                                "(7 forwards); a vertex-gradient FD would need 6 forwards per "
                                                "vertex, so the ratio is against the cheaper baseline",
                                 "forward_roofline": fwd_roof, **other_trees,
                                 "backward_roofline": dict(hbm_frac(bwd_bytes, ms_b, peak),
                                                           model="pairs kernel 140 B/query + 3 sort passes and a "
                                                                 "histogram of 3Q pairs + reduce 60 B/query + 12 B/vertex")}
    tb.free()


def _ev_time(torch, fn, reps=3, warm=1):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def gmm_component(bq, W, torch, comp, n):
    """The 10M-point Gaussian-mixture configuration (64 components, sigma
    log-uniform in [1e-4, 1e-1], coordinates offset by 1e5: many exact
    duplicates and long runs of equal Morton keys): Morton and
    spatial-median (leaf 8) builds, then 10M closest-point and 10M kNN(16)
    queries drawn from the same mixture."""
    peak, _ = hbm_peak()
    pts = torch.from_numpy(W.gmm_points(n)).cuda()
    qs = torch.from_numpy(W.gmm_points(n, sample_seed=W.SEED_GMM_QUERIES)).cuda()
    boxes = bq.points_to_boxes(pts)
    ms_m = _ev_time(torch, lambda: bq.cuda.radixBuilder(boxes).free())
    with bq.profile() as prof:
        bq.cuda.radixBuilder(boxes).free()
    ms_s = _ev_time(torch, lambda: bq.gpuBuilder(boxes, bq.BuildConfig(makeLeafThreshold=8)).free())
    bvh = bq.cuda.radixBuilder(boxes)
    nn = bvh.numNodes
    # Queries under the reference's tie rule (answers bit-identical to the reference's kernels).  The
    # lowest-id rule has to look at every point at the tied distance, and here tight clusters collapse
    # into ~1e5 identical points, so it is timed on a 100k-query sample only.
    ref = bq.query_config(tieMode=bq.TIES_REFERENCE)
    ms_cp = _ev_time(torch, lambda: bq.points.findClosest(bvh, pts, qs, qcfg=ref), reps=2)
    ms_knn = _ev_time(torch, lambda: bq.points.findKNN(bvh, pts, qs, 16, qcfg=ref), reps=2)
    cpc = bq.points.visitCounts(bvh, pts, qs, 0, qcfg=ref)
    knc = bq.points.visitCounts(bvh, pts, qs, 16, qcfg=ref)
    qsam = qs[:100_000]
    ms_cp_low = _ev_time(torch, lambda: bq.points.findClosest(bvh, pts, qsam), reps=1)
    ms_knn_low = _ev_time(torch, lambda: bq.points.findKNN(bvh, pts, qsam, 16), reps=1)
    low = bq.points.visitCounts(bvh, pts, qsam, 0)
    bvh.free()
    comp["gmm10m"] = {
        "points": n, "queries": n,
        "morton_build_ms": ms_m, "morton_build_Mprims_s": n / ms_m / 1e3,
        "morton_build_roofline": dict(hbm_frac(morton_build_bytes(n, nn), ms_m, peak), model="288 N + 64 M"),
        "morton_phases_ms": {k: round(v[1], 4) for k, v in prof.table.items()},
        "spatial_median_leaf8_ms": ms_s, "spatial_median_Mprims_s": n / ms_s / 1e3,
        "query_tie_rule": "reference (BQ_TIES_REFERENCE)",
        "closest_point_ms": ms_cp, "closest_point_Mqueries_s": n / ms_cp / 1e3,
        "closest_point_roofline": query_roofline(cpc, n, 8, 16, ms_cp, peak, n * 20 + 32 * nn + 16 * n),
        "knn16_ms": ms_knn, "knn16_Mqueries_s": n / ms_knn / 1e3,
        "knn16_roofline": query_roofline(knc, n, 132, 16, ms_knn, peak, n * 144 + 32 * nn + 16 * n),
        "lowest_id_rule_100k_sample": {"closest_point_ms": ms_cp_low, "knn16_ms": ms_knn_low,
                                       "prims_tested_per_query": low["prims"] / len(qsam)}}
    del pts, qs, boxes


def c1_component(bq, W, torch, comp, pts_np, tp, boxes_t):
    """The 1M-point configuration: spatial-median build (leaf 8) and 1M
    closest-point queries (the reference's numbers for the same workload
    are in the reference arm's line, c1_reference)."""
    n1 = 1_000_000
    b1, tp1 = boxes_t[:n1], tp[:n1]
    q1 = W.uniform_points(n1, W.SEED_QUERIES, -0.1, 1.1)
    tq1 = torch.from_numpy(q1).cuda()
    cfg = bq.BuildConfig(makeLeafThreshold=8)
    ms_b = _ev_time(torch, lambda: bq.gpuBuilder(b1, cfg).free())
    t = bq.gpuBuilder(b1, cfg)
    ms_q = _ev_time(torch, lambda: bq.points.findClosest(t, tp1, tq1))
    t.free()
    comp["c1_1M_points_leaf8"] = {"points": n1, "queries": n1, "leaf": 8, "build_ms": ms_b, "closest_point_ms": ms_q,
                                  "build_Mprims_s": n1 / ms_b / 1e3, "Mqueries_s": n1 / ms_q / 1e3}


def c1_reference(W, pts_np):
    """The reference's GPU builder and kernel (sm_100a) and its host builder
    and query (one core, and all cores for the query) on the 1M-point
    configuration."""
    n1 = 1_000_000
    q1 = W.uniform_points(n1, W.SEED_QUERIES, -0.1, 1.1)
    out = {}
    from oracle.oracle import RefCPU, RefGPU, have_ref_cpu, have_ref_gpu
    if have_ref_gpu():
        r = RefGPU()
        out["reference_gpu_build_ms"] = r.time_build(RefGPU.SPATIAL_MEDIAN, pts_np[:n1], 8, reps=3)
        out["reference_gpu_closest_point_ms"] = r.time_query(RefGPU.SPATIAL_MEDIAN, pts_np[:n1], q1, 0, 8, reps=3)
    if have_ref_cpu():
        rc = RefCPU()
        bx = W.point_boxes(pts_np[:n1])
        t0 = time.perf_counter()
        nodes, prims = rc.build(bx, 8)
        out["reference_cpu_build_ms"] = (time.perf_counter() - t0) * 1e3
        sample = 100_000
        t0 = time.perf_counter()
        rc.closest_point(nodes, prims, pts_np[:n1], q1[:sample], threads=1)
        out["reference_cpu_closest_point_ms_1core"] = (time.perf_counter() - t0) * 1e3 * n1 / sample
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        rc.closest_point(nodes, prims, pts_np[:n1], q1, threads=threads)
        out["reference_cpu_closest_point_ms_allcores"] = (time.perf_counter() - t0) * 1e3
        out["host_threads"] = threads
    return out


def tri_forward_other_trees(bq, torch, tbox, tt, tv, tq, ids, d, timer):
    """The triangle forward over SAH and spatial-median trees of the same
    triangle boxes (the benchmark's own tree is the Morton one, as in the
    reference's timing): time, and whether the answers equal the Morton
    tree's (under the default lowest-id tie rule they do not depend on the
    tree)."""
    out = {}
    for name, build in (("sah", lambda: bq.cuda.sahBuilder(tbox)), ("spatial_median", lambda: bq.gpuBuilder(tbox))):
        t = build()
        out[f"forward_{name}_tree_ms"] = timer(lambda: bq.triangles.findClosest(t, tt, tv, tq))
        i2, d2, _ = bq.triangles.findClosest(t, tt, tv, tq)
        out[f"forward_{name}_tree_same_answers"] = bool(torch.equal(i2, ids) and torch.equal(d2, d))
        t.free()
    return out


def batched_components(bq, W, torch, comp):
    """The two batched workloads: 512 point clouds (about 19M points, 25.6M
    kNN(16) queries; one segmented build + one query launch replayed from a
    CUDA graph, against a per-cloud loop of single builds and queries), and
    a 100-step fitting loop over 128 triangle meshes (6.4M queries per step:
    triangle boxes, batched refit, batched closest triangle, adjoint,
    vertex update)."""
    import numpy as np
    pts, off, qs, qoff = W.cloud_batch()
    n, nq = len(pts), len(qs)
    b = torch.from_numpy(W.point_boxes(pts)).cuda()
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    toff, tqoff = torch.from_numpy(off).cuda().int(), torch.from_numpy(qoff).cuda().int()
    # launch shape from the autotuner (JSON cache; tuned here on a cache miss, untimed)
    from cubql_b200 import tuning
    tuned = tuning.tuned_batched_knn(b, tp, toff, tq, tqoff, 16)
    bcfg = bq.BuildConfig(makeLeafThreshold=tuned["makeLeafThreshold"])
    qcfg = tuning.query_config_of(tuned)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # first use of the stream-ordered pool, outside the capture
        bq.batched_knn(bq.Batch(b, toff, bcfg, stream_alloc_null=True), tp, toff, tq, tqoff, 16, qcfg=qcfg,
                       stream_alloc_null=True)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        gbatch = bq.Batch(b, toff, bcfg, stream_alloc_null=True)
        gout = bq.batched_knn(gbatch, tp, toff, tq, tqoff, 16, qcfg=qcfg, stream_alloc_null=True)
    ms_graph = _ev_time(torch, graph.replay)
    ms_build = _ev_time(torch, lambda: bq.Batch(b, toff, bcfg))
    bat = bq.Batch(b, toff, bcfg)
    ms_query = _ev_time(torch, lambda: bq.batched_knn(bat, tp, toff, tq, tqoff, 16, qcfg=qcfg))

    def loop():
        for c in range(len(off) - 1):
            sl, ql = slice(int(off[c]), int(off[c + 1])), slice(int(qoff[c]), int(qoff[c + 1]))
            t = bq.cuda.radixBuilder(b[sl])
            bq.points.findKNN(t, tp[sl], tq[ql], 16)
            t.free()
    ms_loop = _ev_time(torch, loop, reps=1, warm=1)
    same = True
    graph.replay()
    torch.cuda.synchronize()
    for c in range(len(off) - 1):  # every cloud: batched answers == per-cloud answers
        sl, ql = slice(int(off[c]), int(off[c + 1])), slice(int(qoff[c]), int(qoff[c + 1]))
        t = bq.cuda.radixBuilder(b[sl])
        si, sd, _ = bq.points.findKNN(t, tp[sl], tq[ql], 16)
        same &= bool(torch.equal(si, gout[0][ql]) and torch.equal(sd, gout[1][ql]))
        t.free()
    del graph
    comp["batched_knn_512_clouds"] = {
        "clouds": len(off) - 1, "points": n, "queries": nq, "k": 16,
        "graph_ms": ms_graph, "build_ms": ms_build, "query_ms": ms_query,
        "Mqueries_s": nq / ms_graph / 1e3, "build_Mprims_s": n / ms_build / 1e3,
        "per_cloud_loop_ms": ms_loop, "speedup_vs_per_cloud_loop": ms_loop / ms_graph,
        "matches_per_cloud_answers": same, "clouds_compared": len(off) - 1,
        "tuned": {k: v for k, v in tuned.items() if k != "key"}, "tuning_key": tuned["key"]}
    del b, tp, tq, bat, gbatch, gout

    verts, tris, toffm, qsm, qoffm = W.mesh_batch()
    tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    tqm = torch.from_numpy(qsm).cuda()
    toff_t, qoff_t = torch.from_numpy(toffm).cuda().int(), torch.from_numpy(qoffm).cuda().int()
    batch = bq.Batch(bq.triangles.boxes(tt, tv), toff_t)
    g = torch.full((len(qsm),), 1.0 / len(qsm), device="cuda")
    state = {"v": tv}

    def step(check=False):
        v = state["v"]
        boxes = bq.triangles.boxes(tt, v)
        bq.batched_refit(batch, boxes)
        ids, d, _ = bq.batched_tri_closest(batch, tt, v, tqm, qoff_t)
        ok = True
        if check:  # the refitted trees' forward against trees rebuilt from scratch
            fresh = bq.Batch(boxes, toff_t)
            fi, fd, _ = bq.batched_tri_closest(fresh, tt, v, tqm, qoff_t)
            ok = bool(torch.equal(ids, fi) and torch.equal(d, fd))
            del fresh
        _, gv = bq.triangles.distanceBackward(tt, v, tqm, ids, g)
        state["v"] = v - 0.5 * gv
        return ok

    steps = 100
    # untimed run: every step's forward checked against a rebuild
    all_equal = all([step(check=True) for _ in range(steps)])
    state["v"] = tv  # the timed run repeats the same 100 steps from the same vertices
    ms_step = _ev_time(torch, step, reps=steps, warm=0)
    comp["fit_loop_128_meshes"] = {
        "meshes": len(toffm) - 1, "triangles": int(len(tris)), "queries_per_step": int(len(qsm)), "steps": steps,
        "ms_per_step": ms_step, "fwd_bwd_queries_s": len(qsm) / ms_step * 1e3,
        "refit_forward_equals_rebuild": all_equal, "steps_checked": steps}


BOX_HALF = 0.00585


def box_queries(W, nq):
    """nq query boxes of half size BOX_HALF around uniform centres."""
    import numpy as np
    c = W.uniform_points(nq, W.SEED_QUERIES)
    return np.concatenate([c - BOX_HALF, c + BOX_HALF], 1).astype(np.float32)


def reference_gpu(comp, pts_np, W):
    from oracle.oracle import RefGPU, have_ref_gpu
    if not have_ref_gpu():
        comp["reference_gpu"] = {"unavailable": "oracle/_ref/libref_gpu.so not built"}
        return
    r = RefGPU()
    n = len(pts_np)
    out = {}
    out["radixBuilder_ms"] = r.time_build(RefGPU.RADIX, pts_np, 0, reps=3)
    out["gpuBuilder_leaf8_ms"] = r.time_build(RefGPU.SPATIAL_MEDIAN, pts_np, 8, reps=3)
    out["gpuBuilder_leaf1_ms"] = r.time_build(RefGPU.SPATIAL_MEDIAN, pts_np, 0, reps=3)
    out["rebinRadixBuilder_ms"] = r.time_build(RefGPU.REBIN, pts_np, 0, reps=3)
    qs = W.uniform_points(n, W.SEED_QUERIES)
    out["findClosest_ms"] = r.time_query(RefGPU.RADIX, pts_np, qs, 0, reps=2)
    out["findKNN16_ms"] = r.time_query(RefGPU.RADIX, pts_np, qs, 16, reps=2)
    out["findClosest_exludeSelf_ms"] = r.time_query(RefGPU.RADIX, pts_np, pts_np, -1, reps=2)
    out["gpuBuilder_wide4_ms"] = r.time_build(RefGPU.WIDE4, pts_np, 0, reps=2)
    out["gpuBuilder_wide8_ms"] = r.time_build(RefGPU.WIDE8, pts_np, 0, reps=2)
    out["findClosest_wide4_ms"] = r.time_wide_query(4, pts_np, qs, 0, reps=2)
    out["findClosest_wide8_ms"] = r.time_wide_query(8, pts_np, qs, 0, reps=2)
    out["fixedBoxQuery_count_fill_ms"], out["fixedBoxQuery_results"] = r.time_box_query(
        RefGPU.RADIX, pts_np, box_queries(W, 1_000_000), reps=2)
    out["note"] = "reference kernels compiled for sm_100a, same points, one thread per query <<<ceil(Q/128),128>>>"
    comp["reference_gpu"] = out


def run_ours(args):
    import ctypes

    import numpy as np
    import torch

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    import cubql_b200 as bq
    from cubql_b200 import workloads as W

    n = args.n
    pts_np = W.uniform_points(n, W.SEED_DATA + rank)
    boxes_np = W.point_boxes(pts_np)
    tp = torch.from_numpy(pts_np).cuda()
    boxes_t = torch.from_numpy(boxes_np).cuda()
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    cb = CBuild(bq, boxes_t, n)

    if args.only_tri:
        verts, tris = W.icosphere(args.mesh_level)
        tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
        tq = torch.from_numpy(W.uniform_points(args.queries, W.SEED_QUERIES, -1.5, 1.5)).cuda()
        tbox = bq.triangles.boxes(tt, tv)
        tb = bq.cuda.radixBuilder(tbox)
        ms_t = time_loop(lambda: bq.triangles.findClosest(tb, tt, tv, tq), args.steps, args.warmup, world)
        ids, dsq, _ = bq.triangles.findClosest(tb, tt, tv, tq)
        other = tri_forward_other_trees(bq, torch, tbox, tt, tv, tq, ids, dsq,
                                        lambda fn: time_loop(fn, args.steps, args.warmup, world))
        if rank == 0:
            print(json.dumps({"only_tri": True, "triangles": len(tris), "queries": args.queries, "forward_ms": ms_t,
                              **other}))
        tb.free()
        return
    if args.only_wide:
        wb = bq.gpuBuilderWide(boxes_t, 4)
        qs = torch.from_numpy(W.uniform_points(args.queries, W.SEED_QUERIES)).cuda()
        ms_w = time_loop(lambda: bq.points.findClosest(wb, tp, qs), args.steps, args.warmup, world)
        if rank == 0:
            print(json.dumps({"only_wide": True, "points": n, "queries": args.queries, "wide4_closest_point_ms": ms_w}))
        wb.free()
        return
    if args.only_queries:
        bvh = bq.cuda.radixBuilder(boxes_t)
        qs = torch.from_numpy(W.uniform_points(args.queries, W.SEED_QUERIES)).cuda()
        ms_cp = time_loop(lambda: bq.points.findClosest(bvh, tp, qs), args.steps, args.warmup, world)
        ms_knn = time_loop(lambda: bq.points.findKNN(bvh, tp, qs, 16), args.steps, args.warmup, world)
        if rank == 0:
            print(json.dumps({"only_queries": True, "points": n, "queries": args.queries, "closest_point_ms": ms_cp,
                              "knn16_ms": ms_knn}))
        bvh.free()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    props = torch.cuda.get_device_properties(local)
    uuid = str(getattr(props, "uuid", ""))
    clocks = ClockSampler(uuid)
    clocks.start()
    ms = time_loop(lambda: cb.step(sptr), args.steps, args.warmup, world)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world)
    value = weak_value(n, ms_max, world)
    if args.only_build:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "Mprims/s", "ms_per_step": ms_max,
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "only_build": True}))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    # per-phase breakdown of the same step (library events on its stream)
    with bq.profile() as prof:
        for _ in range(max(3, min(args.steps, 10))):
            cb.step(sptr)
    steps_prof = max(3, min(args.steps, 10))
    table = prof.table
    launches_per_step = sum(v[0] for v in table.values()) / steps_prof
    peak, peak_kind = hbm_peak()
    kernels = {}
    for name, (launches, tms) in table.items():
        per = tms / launches
        bytes_per = PHASE_BYTES.get(name, 0) * n
        kernels[name] = {"launches_per_step": launches / steps_prof, "ms_per_launch": per,
                         "share": tms / sum(v[1] for v in table.values()),
                         "alg_bytes_per_launch": bytes_per,
                         "GB_s": bytes_per / per / 1e6 if bytes_per else None,
                         "frac_of_measured_hbm": (bytes_per / per / 1e6 / peak) if bytes_per else None}
    dom = max(table.items(), key=lambda kv: kv[1][1])[0]
    dk = kernels[dom]
    build_bytes = 288 * n + 64 * 2 * n  # the fixed accounting model: 288 N + 64 M, M = 2N
    roofline = {"kernel": dom, "bound": "hbm", "achieved": dk["GB_s"], "peak": peak, "unit": "GB/s",
                "frac": dk["frac_of_measured_hbm"], "traffic": ncu_traffic(dom), "peak_source": peak_kind,
                "whole_build": {"alg_bytes": build_bytes, "GB_s": build_bytes / ms / 1e6,
                                "frac": build_bytes / ms / 1e6 / peak}}

    # end to end through the public API: pinned host boxes -> tree on host
    e2e = e2e_pipelined(bq, torch, boxes_np, n, max(4, args.steps // 2), 2, world)

    comp = {}
    cpu_baseline = None
    if rank == 0 and not args.no_components:
        components(bq, W, torch, pts_np, tp, boxes_t, comp)
        c1_component(bq, W, torch, comp, pts_np, tp, boxes_t)
        gmm_component(bq, W, torch, comp, n)
        batched_components(bq, W, torch, comp)
    if rank == 0:
        cpu_baseline = cpu_leg(W, pts_np)
    barrier(world)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mprims/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": bench_config(n, W.SEED_DATA),
                "impl_detail": {"builder": "Morton (radix, 63-bit) builder, C ABI bq_build_morton63_f3",
                                "parallelism": f"{world} independent builds, one per GPU"},
                "e2e": e2e, "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu_baseline,
                "gpu_launches": int(round(launches_per_step * args.steps)), "clocks": clk, "components": comp}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def e2e_pipelined(bq, torch, boxes_np, n, steps, warmup, world):
    """The build through the public API (cubql_b200.cuda.radixBuilder) with
    host buffers: every step copies its boxes host->device, builds, and
    copies the whole tree (nodes + primIDs) device->host.  Consecutive steps
    alternate between two streams, so one step's tree download overlaps the
    next step's upload and build (separate copy engines per direction).
    Timed with CUDA events around all steps, on the device."""
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    host_boxes = [torch.from_numpy(boxes_np).pin_memory() for _ in range(2)]
    dev_boxes = [torch.empty((n, 6), dtype=torch.float32, device="cuda") for _ in range(2)]
    host_nodes = [torch.empty((2 * n, 8), dtype=torch.float32).pin_memory() for _ in range(2)]
    host_prims = [torch.empty(n, dtype=torch.int32).pin_memory() for _ in range(2)]
    trees = [None, None]

    def step(i):
        k = i % 2
        with torch.cuda.stream(streams[k]):
            if trees[k] is not None:
                trees[k].free()  # stream-ordered: after that tree's download
            dev_boxes[k].copy_(host_boxes[k], non_blocking=True)
            b = bq.cuda.radixBuilder(dev_boxes[k])
            host_nodes[k][: b.numNodes].copy_(b.nodes_tensor(), non_blocking=True)
            host_prims[k][: b.numPrims].copy_(b.primids_tensor(), non_blocking=True)
            trees[k] = b

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    barrier(world)
    cur = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    for s in streams:
        s.wait_event(e0)
    for i in range(steps):
        step(i)
    for s in streams:
        cur.wait_stream(s)
    e1.record(cur)
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
    for b in trees:
        if b is not None:
            b.free()
    torch.cuda.synchronize()
    return {"value": weak_value(n, ms, world), "unit": "Mprims/s", "h2d_bytes_per_step": 24 * n,
            "d2h_bytes_per_step": 32 * 2 * n + 4 * n, "ms_per_step": ms, "steps": steps,
            "path": "cubql_b200.cuda.radixBuilder (C ABI bq_build_morton63_f3) from pinned host boxes, whole tree "
                    "copied back every step; consecutive steps on two streams (upload/build/download overlap)"}


def cpu_leg(W, pts_np):
    """The reference's host builder on the benchmark's own points (all of
    them), one core: the median of 3 builds."""
    from oracle.oracle import Oracle, RefCPU, have_ref_cpu
    boxes = W.point_boxes(pts_np)
    if have_ref_cpu():
        r = RefCPU()
        kind = "reference"
        fn = lambda: r.build(boxes, 0)  # noqa: E731
    else:
        o = Oracle()
        kind = "port"
        fn = lambda: o.cpu_build(boxes, 0)  # noqa: E731
    secs = [_timed(fn) for _ in range(3)]
    t = statistics.median(secs)
    return {"value": len(pts_np) / t / 1e6, "unit": "Mprims/s", "cores": 1, "kind": kind,
            "sample": f"cpuBuilder (spatial median, leaf 1) over all {len(pts_np)} benchmark points, "
                      f"median of 3 builds, {t:.3f} s each"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
