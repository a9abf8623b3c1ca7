"""ctypes bindings of the CPU oracle and of the compiled reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference legs, never by the product package.

  liboracle.so  C restatement of the reference algorithms (bq_oracle.c)
  libref_cpu.so the reference's host code, compiled from its sources
  libref_gpu.so the reference's GPU builders and query device functions,
                compiled for sm_100a from its sources (needs a GPU to run)
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_gpu.so")

NODE = np.dtype([("lower", "<f4", 3), ("upper", "<f4", 3), ("admin", "<u8")])
assert NODE.itemsize == 32
# one SAH bin (sah_builder.h:53-60): AtomicBox-encoded bounds + count, 32 B
SAH_BIN = np.dtype([("lo", "<i4", 3), ("hi", "<i4", 3), ("count", "<i4"), ("pad", "<i4")])
SAH_BINS = np.dtype([("b", SAH_BIN, (3, 16))])
assert SAH_BINS.itemsize == 1536


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def build(reference_dir=None):
    """Compile the oracle (always) and the reference libraries from the
    reference source tree `reference_dir` (when given and present)."""
    import subprocess
    subprocess.run(["sh", os.path.join(HERE, "build_oracle.sh")], check=True)
    if reference_dir and os.path.isdir(os.path.join(reference_dir, "cuBQL")):
        subprocess.run(["sh", os.path.join(HERE, "build_ref.sh"), reference_dir], check=True)


_libs = {}


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run oracle/build_oracle.sh / build_ref.sh)")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def have_ref_cpu():
    return os.path.exists(REF_CPU_SO)


def have_ref_gpu():
    return os.path.exists(REF_GPU_SO)


def offsets(nodes):
    return (nodes["admin"] & np.uint64(0xFFFFFFFFFFFF)).astype(np.int64)


def counts(nodes):
    return (nodes["admin"] >> np.uint64(48)).astype(np.int64)


# ---------------------------------------------------------------------------
# C restatement
# ---------------------------------------------------------------------------
class Oracle:
    def __init__(self):
        self.lib = _load(ORACLE_SO)

    def uniform_points(self, n, seed, lo=0.0, hi=1.0):
        out = np.empty((n, 3), dtype=np.float32)
        self.lib.orc_uniform_points(ctypes.c_uint32(n), ctypes.c_uint32(seed), ctypes.c_double(lo),
                                    ctypes.c_double(hi), _p(out))
        return out

    def _tree(self, fn, boxes, *args):
        boxes = _f32(boxes).reshape(-1, 6)
        n = boxes.shape[0]
        nodes = np.zeros(2 * n + 2, dtype=NODE)
        prims = np.zeros(max(n, 1), dtype=np.uint32)
        nn, npr = ctypes.c_uint32(), ctypes.c_uint32()
        rc = fn(_p(boxes), ctypes.c_uint32(n), *args, _p(nodes), _p(prims), ctypes.byref(nn), ctypes.byref(npr))
        assert rc == 0
        return nodes[: nn.value].copy(), prims[: npr.value].copy()

    def radix_build(self, boxes, makeLeafThreshold=0, maxAllowedLeafSize=1 << 15, keys=False):
        boxes = _f32(boxes).reshape(-1, 6)
        n = boxes.shape[0]
        nodes = np.zeros(2 * n + 2, dtype=NODE)
        prims = np.zeros(max(n, 1), dtype=np.uint32)
        k = np.zeros(max(n, 1), dtype=np.uint64)
        nn, npr = ctypes.c_uint32(), ctypes.c_uint32()
        rc = self.lib.orc_radix_build(_p(boxes), ctypes.c_uint32(n), ctypes.c_int(makeLeafThreshold),
                                      ctypes.c_int(maxAllowedLeafSize), _p(nodes), _p(prims), ctypes.byref(nn),
                                      ctypes.byref(npr), _p(k))
        assert rc == 0
        out = (nodes[: nn.value].copy(), prims[: npr.value].copy())
        return out + (k[: npr.value].copy(),) if keys else out

    def rebin_build(self, boxes, makeLeafThreshold=0, maxAllowedLeafSize=1 << 15):
        return self._tree(self.lib.orc_rebin_build, boxes, ctypes.c_int(makeLeafThreshold),
                          ctypes.c_int(maxAllowedLeafSize))

    def sm_build(self, boxes, makeLeafThreshold=0):
        return self._tree(self.lib.orc_sm_build, boxes, ctypes.c_int(makeLeafThreshold))

    def sah_build(self, boxes, makeLeafThreshold=0, fma_mode=1, heur=0):
        """heur 0: SAH builder; 1: ELH builder (8 bins, edge lengths)."""
        return self._tree(self.lib.orc_heur_build, boxes, ctypes.c_int(makeLeafThreshold), ctypes.c_int(fma_mode),
                          ctypes.c_int(heur))

    def sah_evaluate(self, bins, fma_mode=1, heur=0):
        """evaluateSAH (heur 0) / evaluateELH (heur 1, bins b[:, :8]) per
        SAH_BINS record: (dims (-1 leaf), bins)."""
        bins = np.ascontiguousarray(bins, dtype=SAH_BINS)
        dims = np.zeros(len(bins), dtype=np.int32)
        sb = np.zeros(len(bins), dtype=np.int32)
        for i in range(len(bins)):
            b = ctypes.c_int(0)
            dims[i] = self.lib.orc_heur_evaluate(bins[i:i + 1].ctypes.data_as(ctypes.c_void_p),
                                                 ctypes.c_int(fma_mode), ctypes.c_int(heur), ctypes.byref(b))
            sb[i] = b.value
        return dims, sb

    def sah_area(self, boxes, fma_mode=1):
        f = self.lib.orc_sah_area
        f.restype = ctypes.c_float
        boxes = _f32(boxes).reshape(-1, 6)
        return np.array([f(_p(boxes[i, :3].copy()), _p(boxes[i, 3:].copy()), ctypes.c_int(fma_mode))
                         for i in range(len(boxes))], dtype=np.float32)

    def cpu_build(self, boxes, makeLeafThreshold=0):
        return self._tree(self.lib.orc_cpu_build, boxes, ctypes.c_int(makeLeafThreshold))

    def canonicalize(self, nodes, prims):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        out = np.zeros(len(nodes), dtype=NODE)
        outp = np.zeros(max(len(prims), 1), dtype=np.uint32)
        npr = ctypes.c_uint32()
        rc = self.lib.orc_canonicalize(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(out), _p(outp),
                                       ctypes.byref(npr))
        if rc != 0:
            raise ValueError(f"tree is not a valid BinaryBVH (canonicalize rc={rc})")
        return out, outp[: npr.value].copy()

    def closest_point(self, nodes, prims, points, queries, maxSqr=np.inf, fma_mode=1, tie_mode=0, stack=64):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        ovf = np.zeros(nq, dtype=np.uint8)
        vis = np.zeros(nq, dtype=np.uint32)
        self.lib.orc_closest_point(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(points), _p(queries),
                                   ctypes.c_uint32(nq), ctypes.c_float(maxSqr), ctypes.c_int(fma_mode),
                                   ctypes.c_int(tie_mode), ctypes.c_int(stack), _p(ids), _p(d), _p(ovf), _p(vis))
        return ids, d, ovf.astype(bool), vis

    def closest_point_exclude(self, nodes, prims, points, queries, exclude_ids=None, exclude_self=False,
                              maxSqr=np.inf, fma_mode=1, tie_mode=0):
        """findClosest_exludeID (one prim id per query, -1: none) or
        findClosest_exludeSelf (points equal to the query), findClosest.h:278-334."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        ex = None if exclude_ids is None else np.ascontiguousarray(exclude_ids, dtype=np.int32)
        self.lib.orc_closest_point_exclude(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(points), _p(queries),
                                           ctypes.c_uint32(nq), ctypes.c_float(maxSqr), ctypes.c_int(fma_mode),
                                           ctypes.c_int(tie_mode), _p(ex) if ex is not None else None,
                                           ctypes.c_int(1 if exclude_self else 0), _p(ids), _p(d))
        return ids, d

    def box_query(self, nodes, prims, boxes, query_boxes, stack=1 << 20):
        """fixedBoxQuery::forEachPrim with a per-prim box test
        (fixedBoxQuery.h:73-156): returns (offsets int64 (nq+1,), ids int32)
        in visiting order; raises on a traversal deeper than `stack`."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        boxes, qb = _f32(boxes).reshape(-1, 6), _f32(query_boxes).reshape(-1, 6)
        nq = qb.shape[0]
        counts = np.zeros(nq, dtype=np.uint32)
        args = (_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(boxes), _p(qb), ctypes.c_uint32(nq),
                ctypes.c_int(stack))
        if self.lib.orc_box_query(*args, _p(counts), None, None) != 0:
            raise RuntimeError("box query traversal stack exceeded")
        offsets = np.zeros(nq + 1, dtype=np.uint64)
        np.cumsum(counts, out=offsets[1:])
        ids = np.zeros(max(int(offsets[-1]), 1), dtype=np.int32)
        self.lib.orc_box_query(*args, _p(counts), _p(offsets), _p(ids))
        return offsets.astype(np.int64), ids[:int(offsets[-1])]

    # ---- wide trees (slots are NODE records whose admin word holds the
    # valid/offset/count bit field of WideBVH::Node::Child) ----
    def wide_collapse(self, nodes, width):
        """Binary -> width-wide collapse; returns the slots (numWide*width)."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        out = np.zeros(max(len(nodes), 1) * width, dtype=NODE)
        nw = self.lib.orc_wide_collapse(_p(nodes), ctypes.c_uint32(len(nodes)), ctypes.c_int(width), _p(out))
        if nw < 0:
            raise ValueError("binary tree is not valid for the collapse")
        return out[: nw * width].copy()

    def wide_canonicalize(self, slots, width, prims):
        slots = np.ascontiguousarray(slots, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        out = np.zeros(len(slots), dtype=NODE)
        outp = np.zeros(max(len(prims), 1), dtype=np.uint32)
        npr = ctypes.c_uint32()
        rc = self.lib.orc_wide_canonicalize(_p(slots), ctypes.c_uint32(len(slots) // width), ctypes.c_int(width),
                                            _p(prims), _p(out), _p(outp), ctypes.byref(npr))
        if rc != 0:
            raise ValueError(f"not a valid wide tree (rc={rc})")
        return out, outp[: npr.value].copy()

    def wide_closest(self, slots, width, prims, points, queries, maxSqr=np.inf, fma_mode=1, tie_mode=0):
        slots = np.ascontiguousarray(slots, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        rc = self.lib.orc_wide_closest(_p(slots), ctypes.c_uint32(len(slots) // width), ctypes.c_int(width),
                                       _p(prims), _p(points), _p(queries), ctypes.c_uint32(nq),
                                       ctypes.c_float(maxSqr), ctypes.c_int(fma_mode), ctypes.c_int(tie_mode),
                                       _p(ids), _p(d))
        assert rc == 0
        return ids, d

    def wide_box_query(self, slots, width, prims, boxes, query_boxes):
        slots = np.ascontiguousarray(slots, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        boxes, qb = _f32(boxes).reshape(-1, 6), _f32(query_boxes).reshape(-1, 6)
        nq = qb.shape[0]
        counts = np.zeros(nq, dtype=np.uint32)
        args = (_p(slots), ctypes.c_uint32(len(slots) // width), ctypes.c_int(width), _p(prims), _p(boxes), _p(qb),
                ctypes.c_uint32(nq), _p(counts))
        self.lib.orc_wide_box_query(*args, None, None)
        offsets = np.zeros(nq + 1, dtype=np.uint64)
        np.cumsum(counts, out=offsets[1:])
        ids = np.zeros(max(int(offsets[-1]), 1), dtype=np.int32)
        self.lib.orc_wide_box_query(*args, _p(offsets), _p(ids))
        return offsets.astype(np.int64), ids[:int(offsets[-1])]

    def knn(self, nodes, prims, points, queries, k, maxSqr=np.inf, fma_mode=1, tie_mode=0, stack=64):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), dtype=np.int32)
        d = np.zeros((nq, k), dtype=np.float32)
        nf = np.zeros(nq, dtype=np.int32)
        ovf = np.zeros(nq, dtype=np.uint8)
        self.lib.orc_knn(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(points), _p(queries),
                         ctypes.c_uint32(nq), ctypes.c_int(k), ctypes.c_float(maxSqr), ctypes.c_int(fma_mode),
                         ctypes.c_int(tie_mode), ctypes.c_int(stack), _p(ids), _p(d), _p(nf), _p(ovf))
        return ids, d, nf, ovf.astype(bool)

    def sqr_pp(self, p, q, fma_mode):
        f = self.lib.orc_sqr_pp
        f.restype = ctypes.c_float
        p, q = _f32(p), _f32(q)
        return np.array([f(_p(p[i]), _p(q[i]), ctypes.c_int(fma_mode)) for i in range(len(p))], dtype=np.float32)

    def sqr_pbox(self, q, boxes, fma_mode):
        f = self.lib.orc_sqr_pbox
        f.restype = ctypes.c_float
        q, boxes = _f32(q), _f32(boxes)
        return np.array([f(_p(q[i]), _p(boxes[i, :3].copy()), _p(boxes[i, 3:].copy()), ctypes.c_int(fma_mode))
                         for i in range(len(q))], dtype=np.float32)

    def tri_closest(self, nodes, prims, tris, verts, queries, maxSqr=np.inf):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        P = np.zeros((nq, 3), dtype=np.float32)
        self.lib.orc_tri_closest(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), _p(tris), _p(verts),
                                 _p(queries), ctypes.c_uint32(nq), ctypes.c_float(maxSqr), _p(ids), _p(d), _p(P))
        return ids, d, P

    def tri_brute_f64(self, tris, verts, queries):
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        nq = queries.shape[0]
        d = np.zeros(nq, dtype=np.float64)
        ids = np.zeros(nq, dtype=np.int32)
        self.lib.orc_tri_brute_f64(_p(tris), _p(verts), ctypes.c_uint32(len(tris)), _p(queries), ctypes.c_uint32(nq),
                                   _p(d), _p(ids))
        return d, ids

    def tri_grad_f64(self, tris, verts, queries, ids, grad_sqr):
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        g = _f32(grad_sqr)
        nq = queries.shape[0]
        gq = np.zeros((nq, 3), dtype=np.float64)
        gv = np.zeros((verts.shape[0], 3), dtype=np.float64)
        self.lib.orc_tri_grad_f64(_p(tris), _p(verts), _p(queries), ctypes.c_uint32(nq), _p(ids), _p(g), _p(gq),
                                  _p(gv))
        return gq, gv

    def tri_cp_f64(self, a, b, c, p):
        f = self.lib.orc_tri_cp_f64
        f.restype = ctypes.c_double
        arr = [np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c, p)]
        w = np.zeros(3, dtype=np.float64)
        d = f(*[_p(x) for x in arr], _p(w))
        return d, w


# ---------------------------------------------------------------------------
# the reference itself
# ---------------------------------------------------------------------------
class RefCPU:
    def __init__(self):
        self.lib = _load(REF_CPU_SO)

    def build(self, boxes, makeLeafThreshold=0):
        boxes = _f32(boxes).reshape(-1, 6)
        n = boxes.shape[0]
        nodes = np.zeros(2 * n + 2, dtype=NODE)
        prims = np.zeros(max(n, 1), dtype=np.uint32)
        nn, npr = ctypes.c_uint32(), ctypes.c_uint32()
        self.lib.ref_cpu_build(_p(boxes), ctypes.c_uint32(n), ctypes.c_int(makeLeafThreshold), _p(nodes), _p(prims),
                               ctypes.byref(nn), ctypes.byref(npr))
        return nodes[: nn.value].copy(), prims[: npr.value].copy()

    def build_throughput(self, boxes, makeLeafThreshold, threads, reps):
        """Wall seconds for `threads` concurrent builds, `reps` each."""
        boxes = _f32(boxes).reshape(-1, 6)
        sec = ctypes.c_double()
        self.lib.ref_cpu_build_throughput(_p(boxes), ctypes.c_uint32(boxes.shape[0]), ctypes.c_int(makeLeafThreshold),
                                          ctypes.c_int(threads), ctypes.c_int(reps), ctypes.byref(sec))
        return sec.value

    def closest_point(self, nodes, prims, points, queries, maxSqr=np.inf, threads=1):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        self.lib.ref_cpu_closest(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                                 _p(points), _p(queries), ctypes.c_uint32(nq), ctypes.c_float(maxSqr), _p(ids), _p(d),
                                 ctypes.c_int(threads))
        return ids, d

    def closest_point_exclude(self, nodes, prims, points, queries, exclude_ids=None, maxSqr=np.inf, threads=1):
        """points::findClosest_exludeID (exclude_ids given) or
        points::findClosest_exludeSelf (exclude_ids None)."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        ex = None if exclude_ids is None else np.ascontiguousarray(exclude_ids, dtype=np.int32)
        self.lib.ref_cpu_closest_exclude(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                                         _p(points), _p(queries), ctypes.c_uint32(nq), ctypes.c_float(maxSqr),
                                         _p(ex) if ex is not None else None, _p(ids), _p(d), ctypes.c_int(threads))
        return ids, d

    def save_points_f64(self, path, pts):
        """samples::saveBinary of vec3d points."""
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        assert self.lib.ref_cpu_save_points_f64(os.fsencode(path), _p(pts), ctypes.c_uint64(len(pts))) == 0

    def load_points_f64_as_f32(self, path, capacity):
        """samples::loadBinary<vec3d> then convert<float,3>."""
        out = np.zeros((max(capacity, 1), 3), dtype=np.float32)
        n = ctypes.c_uint64()
        rc = self.lib.ref_cpu_load_points_f64_as_f32(os.fsencode(path), _p(out), ctypes.c_uint64(capacity),
                                                    ctypes.byref(n))
        assert rc == 0
        return out[: n.value].copy()

    def knn(self, nodes, prims, points, queries, k, maxSqr=np.inf, threads=1):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), dtype=np.int32)
        d = np.zeros((nq, k), dtype=np.float32)
        nf = np.zeros(nq, dtype=np.int32)
        self.lib.ref_cpu_knn(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                             _p(points), _p(queries), ctypes.c_uint32(nq), ctypes.c_int(k), ctypes.c_float(maxSqr),
                             _p(ids), _p(d), _p(nf), ctypes.c_int(threads))
        return ids, d, nf

    def tri_closest(self, nodes, prims, tris, verts, queries, maxSqr=np.inf, threads=1):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        P = np.zeros((nq, 3), dtype=np.float32)
        self.lib.ref_cpu_tri_closest(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                                     _p(tris), ctypes.c_uint32(len(tris)), _p(verts), _p(queries), ctypes.c_uint32(nq),
                                     ctypes.c_float(maxSqr), _p(ids), _p(d), _p(P), ctypes.c_int(threads))
        return ids, d, P


class RefGPU:
    """The reference's GPU code (runs only where a GPU is present)."""
    RADIX, SPATIAL_MEDIAN, REBIN, WIDE4, WIDE8, SAH, ELH = 0, 1, 2, 3, 4, 5, 6

    def __init__(self):
        self.lib = _load(REF_GPU_SO)

    def build(self, method, boxes, makeLeafThreshold=0):
        boxes = _f32(boxes).reshape(-1, 6)
        n = boxes.shape[0]
        nodes = np.zeros(2 * n + 2, dtype=NODE)
        prims = np.zeros(max(n, 1), dtype=np.uint32)
        nn, npr = ctypes.c_uint32(), ctypes.c_uint32()
        rc = self.lib.ref_gpu_build(ctypes.c_int(method), _p(boxes), ctypes.c_uint32(n),
                                    ctypes.c_int(makeLeafThreshold), _p(nodes), _p(prims), ctypes.byref(nn),
                                    ctypes.byref(npr))
        assert rc == 0, "reference GPU build failed"
        return nodes[: nn.value].copy(), prims[: npr.value].copy()

    def closest_point(self, nodes, prims, points, queries, maxSqr=np.inf):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        rc = self.lib.ref_gpu_closest(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                                      _p(points), ctypes.c_uint32(len(points)), _p(queries), ctypes.c_uint32(nq),
                                      ctypes.c_float(maxSqr), _p(ids), _p(d))
        assert rc == 0
        return ids, d

    def closest_point_exclude(self, nodes, prims, points, queries, exclude_ids=None, maxSqr=np.inf):
        """The reference's findClosest_exludeID (exclude_ids given) or
        findClosest_exludeSelf kernel, one thread per query."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        ex = None if exclude_ids is None else np.ascontiguousarray(exclude_ids, dtype=np.int32)
        rc = self.lib.ref_gpu_closest_exclude(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims),
                                              ctypes.c_uint32(len(prims)), _p(points), ctypes.c_uint32(len(points)),
                                              _p(queries), ctypes.c_uint32(nq), ctypes.c_float(maxSqr),
                                              _p(ex) if ex is not None else None, _p(ids), _p(d))
        assert rc == 0
        return ids, d

    def elh_pin(self, bins):
        """The reference's evaluateELH on each record's first 8 bins per
        axis: (dims, splitBins)."""
        bins = np.ascontiguousarray(bins, dtype=SAH_BINS)
        packed = np.ascontiguousarray(bins["b"][:, :, :8])  # ELHBins<float,3>: 3 x 8 bins of 32 B
        dims = np.zeros(len(bins), dtype=np.int32)
        sb = np.zeros(len(bins), dtype=np.int32)
        rc = self.lib.ref_gpu_elh_pin(_p(packed), ctypes.c_int(len(bins)), _p(dims), _p(sb))
        assert rc == 0
        return dims, sb

    def sah_pin(self, bins, boxes):
        """The reference's evaluateSAH on each SAH_BINS record and its
        surfaceArea on each box: (dims, splitBins, areas)."""
        bins = np.ascontiguousarray(bins, dtype=SAH_BINS)
        boxes = _f32(boxes).reshape(-1, 6)
        dims = np.zeros(len(bins), dtype=np.int32)
        sb = np.zeros(len(bins), dtype=np.int32)
        areas = np.zeros(len(boxes), dtype=np.float32)
        rc = self.lib.ref_gpu_sah_pin(_p(bins), ctypes.c_int(len(bins)), _p(dims), _p(sb), _p(boxes),
                                      ctypes.c_int(len(boxes)), _p(areas))
        assert rc == 0
        return dims, sb, areas

    def build_wide(self, width, boxes, makeLeafThreshold=0):
        """The reference's gpuBuilder into a WideBVH<float,3,width>:
        (slots as NODE records, numWide*width of them; primIDs)."""
        boxes = _f32(boxes).reshape(-1, 6)
        n = boxes.shape[0]
        slots = np.zeros((2 * n + 2) * width, dtype=NODE)
        prims = np.zeros(max(n, 1), dtype=np.uint32)
        nw, npr = ctypes.c_uint32(), ctypes.c_uint32()
        rc = self.lib.ref_gpu_build_wide(ctypes.c_int(width), _p(boxes), ctypes.c_uint32(n),
                                         ctypes.c_int(makeLeafThreshold), _p(slots), _p(prims), ctypes.byref(nw),
                                         ctypes.byref(npr))
        assert rc == 0, "reference wide build failed"
        return slots[: nw.value * width].copy(), prims[: npr.value].copy()

    def wide_closest(self, width, slots, prims, points, queries, maxSqr=np.inf):
        slots = np.ascontiguousarray(slots, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        rc = self.lib.ref_gpu_wide_closest(ctypes.c_int(width), _p(slots), ctypes.c_uint32(len(slots) // width),
                                           _p(prims), ctypes.c_uint32(len(prims)), _p(points),
                                           ctypes.c_uint32(len(points)), _p(queries), ctypes.c_uint32(nq),
                                           ctypes.c_float(maxSqr), _p(ids), _p(d))
        assert rc == 0
        return ids, d

    def wide_box_query(self, width, slots, prims, boxes, query_boxes):
        slots = np.ascontiguousarray(slots, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        boxes, qb = _f32(boxes).reshape(-1, 6), _f32(query_boxes).reshape(-1, 6)
        nq = qb.shape[0]
        counts = np.zeros(nq, dtype=np.uint32)
        args = (ctypes.c_int(width), _p(slots), ctypes.c_uint32(len(slots) // width), _p(prims),
                ctypes.c_uint32(len(prims)), _p(boxes), ctypes.c_uint32(len(boxes)), _p(qb), ctypes.c_uint32(nq),
                _p(counts))
        assert self.lib.ref_gpu_wide_box_query(*args, None, None) == 0
        offsets = np.zeros(nq + 1, dtype=np.uint64)
        np.cumsum(counts, out=offsets[1:])
        ids = np.zeros(max(int(offsets[-1]), 1), dtype=np.int32)
        assert self.lib.ref_gpu_wide_box_query(*args, _p(offsets), _p(ids)) == 0
        return offsets.astype(np.int64), ids[:int(offsets[-1])]

    def time_wide_query(self, width, points, queries, makeLeafThreshold=0, reps=5):
        points, queries = _f32(points), _f32(queries)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_wide_query(ctypes.c_int(width), _p(points), ctypes.c_uint32(len(points)),
                                              ctypes.c_int(makeLeafThreshold), _p(queries),
                                              ctypes.c_uint32(len(queries)), ctypes.c_int(reps), ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def box_query(self, nodes, prims, boxes, query_boxes):
        """The reference's fixedBoxQuery::forEachPrim in a kernel, one thread
        per query box, keeping prims whose box overlaps: (offsets, ids)."""
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        boxes, qb = _f32(boxes).reshape(-1, 6), _f32(query_boxes).reshape(-1, 6)
        nq = qb.shape[0]
        counts = np.zeros(nq, dtype=np.uint32)
        args = (_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)), _p(boxes),
                ctypes.c_uint32(len(boxes)), _p(qb), ctypes.c_uint32(nq), _p(counts))
        assert self.lib.ref_gpu_box_query(*args, None, None) == 0
        offsets = np.zeros(nq + 1, dtype=np.uint64)
        np.cumsum(counts, out=offsets[1:])
        ids = np.zeros(max(int(offsets[-1]), 1), dtype=np.int32)
        assert self.lib.ref_gpu_box_query(*args, _p(offsets), _p(ids)) == 0
        return offsets.astype(np.int64), ids[:int(offsets[-1])]

    def knn(self, nodes, prims, points, queries, k, maxSqr=np.inf):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        points, queries = _f32(points), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros((nq, k), dtype=np.int32)
        d = np.zeros((nq, k), dtype=np.float32)
        nf = np.zeros(nq, dtype=np.int32)
        rc = self.lib.ref_gpu_knn(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims), ctypes.c_uint32(len(prims)),
                                  _p(points), ctypes.c_uint32(len(points)), _p(queries), ctypes.c_uint32(nq),
                                  ctypes.c_int(k), ctypes.c_float(maxSqr), _p(ids), _p(d), _p(nf))
        assert rc == 0
        return ids, d, nf

    def tri_closest(self, nodes, prims, tris, verts, queries, maxSqr=np.inf):
        nodes = np.ascontiguousarray(nodes, dtype=NODE)
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        nq = queries.shape[0]
        ids = np.zeros(nq, dtype=np.int32)
        d = np.zeros(nq, dtype=np.float32)
        P = np.zeros((nq, 3), dtype=np.float32)
        rc = self.lib.ref_gpu_tri_closest(_p(nodes), ctypes.c_uint32(len(nodes)), _p(prims),
                                          ctypes.c_uint32(len(prims)), _p(tris), ctypes.c_uint32(len(tris)), _p(verts),
                                          _p(queries), ctypes.c_uint32(nq), ctypes.c_float(maxSqr), _p(ids), _p(d),
                                          _p(P))
        assert rc == 0
        return ids, d, P

    def pin(self, a, b, boxes):
        a, b, boxes = _f32(a), _f32(b), _f32(boxes)
        n = len(a)
        pp = np.zeros(n, dtype=np.float32)
        pb = np.zeros(n, dtype=np.float32)
        rc = self.lib.ref_gpu_pin(_p(a), _p(b), _p(boxes), ctypes.c_uint32(n), _p(pp), _p(pb))
        assert rc == 0
        return pp, pb

    def time_build(self, method, points, makeLeafThreshold=0, reps=5):
        points = _f32(points)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_build(ctypes.c_int(method), _p(points), ctypes.c_uint32(len(points)),
                                         ctypes.c_int(makeLeafThreshold), ctypes.c_int(reps), ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def time_build_boxes(self, method, boxes, makeLeafThreshold=0, reps=3):
        boxes = _f32(boxes).reshape(-1, 6)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_build_boxes(ctypes.c_int(method), _p(boxes), ctypes.c_uint32(len(boxes)),
                                               ctypes.c_int(makeLeafThreshold), ctypes.c_int(reps), ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def time_query(self, method, points, queries, kind, makeLeafThreshold=0, reps=5):
        points, queries = _f32(points), _f32(queries)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_query(ctypes.c_int(method), _p(points), ctypes.c_uint32(len(points)),
                                         ctypes.c_int(makeLeafThreshold), _p(queries), ctypes.c_uint32(len(queries)),
                                         ctypes.c_int(kind), ctypes.c_int(reps), ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def time_tri(self, method, tris, verts, queries, reps=3):
        """ms of the reference's triangles::findClosest kernel over a tree
        built with `method` on the triangle boxes (build not timed)."""
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        verts, queries = _f32(verts), _f32(queries)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_tri(ctypes.c_int(method), _p(tris), ctypes.c_uint32(len(tris)), _p(verts),
                                       _p(queries), ctypes.c_uint32(len(queries)), ctypes.c_int(reps),
                                       ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def time_batched_knn(self, points, offsets, queries, query_offsets, k):
        """ms of the reference serving a batch cloud by cloud: radixBuilder,
        its findKNN kernel over the cloud's queries, cuda::free."""
        points, queries = _f32(points), _f32(queries)
        off = np.ascontiguousarray(offsets, dtype=np.uint32)
        qoff = np.ascontiguousarray(query_offsets, dtype=np.uint32)
        ms = ctypes.c_float()
        rc = self.lib.ref_gpu_time_batched_knn(_p(points), _p(off), _p(queries), _p(qoff),
                                               ctypes.c_uint32(len(off) - 1), ctypes.c_int(k), ctypes.byref(ms))
        assert rc == 0
        return ms.value

    def time_box_query(self, method, points, query_boxes, makeLeafThreshold=0, reps=5):
        """(ms of count + fill kernels, total results) for the reference box
        query over a tree built on the point boxes."""
        points, qb = _f32(points), _f32(query_boxes).reshape(-1, 6)
        ms, tot = ctypes.c_float(), ctypes.c_uint64()
        rc = self.lib.ref_gpu_time_box_query(ctypes.c_int(method), _p(points), ctypes.c_uint32(len(points)),
                                             ctypes.c_int(makeLeafThreshold), _p(qb), ctypes.c_uint32(len(qb)),
                                             ctypes.c_int(reps), ctypes.byref(ms), ctypes.byref(tot))
        assert rc == 0
        return ms.value, tot.value


# ---------------------------------------------------------------------------
# structural invariants (testing/bvh/checkBuilders.cu:64-108)
# ---------------------------------------------------------------------------
def check_tree(nodes, prims, boxes, max_leaf=None, expect_prims=None, node1_unused=True):
    """Raises AssertionError unless: node 0 is the root, every valid prim
    is reached exactly once through the leaves, every node box equals the
    exact union of its children's (or prims') boxes, leaf counts respect
    max_leaf, and offsets stay in range."""
    boxes = np.asarray(boxes, dtype=np.float32).reshape(-1, 6)
    nn = len(nodes)
    if nn == 0:
        assert expect_prims in (None, 0)
        return
    off, cnt = offsets(nodes), counts(nodes)
    seen = np.zeros(len(boxes), dtype=np.int64)
    stack = [0]
    visited = 0
    while stack:
        i = stack.pop()
        visited += 1
        assert not (node1_unused and i == 1), "node 1 must be unused"
        lo, hi = nodes["lower"][i], nodes["upper"][i]
        if cnt[i]:
            assert max_leaf is None or cnt[i] <= max_leaf, f"leaf {i} has {cnt[i]} prims"
            assert off[i] + cnt[i] <= len(prims)
            ids = prims[off[i]: off[i] + cnt[i]]
            seen[ids] += 1
            b = boxes[ids]
            assert np.array_equal(lo, b[:, :3].min(0)) and np.array_equal(hi, b[:, 3:].max(0)), f"leaf {i} box"
        else:
            c = off[i]
            assert (2 if node1_unused else 1) <= c and c + 1 < nn, f"inner node {i} child offset {c}"
            stack += [c, c + 1]
            assert np.array_equal(lo, np.minimum(nodes["lower"][c], nodes["lower"][c + 1])), f"node {i} lower"
            assert np.array_equal(hi, np.maximum(nodes["upper"][c], nodes["upper"][c + 1])), f"node {i} upper"
        assert visited <= nn, "cycle"
    valid = ~(boxes[:, 0] > boxes[:, 3])
    assert np.all(seen[valid] == 1), "every valid prim exactly once"
    assert np.all(seen[~valid] == 0), "no empty prim in a leaf"
    if expect_prims is not None:
        assert int(seen.sum()) == expect_prims


REF_SHIM_SO = os.path.join(HERE, "_ref", "libref_shim.so")


def have_ref_shim():
    return os.path.exists(REF_SHIM_SO)


class RefShim:
    """The reference's types and findClosest kernel over trees built through
    include/bq_cubql.hpp (needs a GPU)."""

    def __init__(self):
        self.lib = _load(REF_SHIM_SO)

    def compare(self, points, queries):
        points, queries = _f32(points), _f32(queries)
        nq = len(queries)
        ri = np.zeros(nq, np.int32)
        rd = np.zeros(nq, np.float32)
        oi = np.zeros(nq, np.int32)
        od = np.zeros(nq, np.float32)
        nn = np.zeros(2, np.uint32)
        rc = self.lib.ref_shim_compare(_p(points), ctypes.c_uint32(len(points)), _p(queries), ctypes.c_uint32(nq),
                                       _p(ri), _p(rd), _p(oi), _p(od), _p(nn))
        assert rc == 0
        return ri, rd, oi, od, nn

    def compare_more(self, points, queries, tris, verts, tri_queries):
        """(ids (6, rows), d (6, rows), numNodes (4,)): rows 0/1 the reference's
        findClosest on its SAH tree / ours, 2/3 its wide findClosest on its
        WideBVH<4> / ours, 4/5 its triangles::findClosest kernel / the batched
        bq_cubql::triangles::findClosest, on one tree (ref_shim.cu)."""
        points, queries, verts, tq = _f32(points), _f32(queries), _f32(verts), _f32(tri_queries)
        tris = np.ascontiguousarray(tris, dtype=np.int32)
        rows = max(len(queries), len(tq))
        ids = np.zeros((6, rows), np.int32)
        d = np.zeros((6, rows), np.float32)
        nn = np.zeros(4, np.uint32)
        rc = self.lib.ref_shim_compare_more(_p(points), ctypes.c_uint32(len(points)), _p(queries),
                                            ctypes.c_uint32(len(queries)), _p(tris), ctypes.c_uint32(len(tris)),
                                            _p(verts), ctypes.c_uint32(len(verts)), _p(tq), ctypes.c_uint32(len(tq)),
                                            _p(ids), _p(d), _p(nn))
        assert rc == 0
        return ids, d, nn
