"""Writes the golden fixtures of tests/golden/ from the reference itself.

  python tests/golden/make_golden.py cpu   # here: the reference's host code
  python tests/golden/make_golden.py gpu   # on a B200: the reference's GPU
                                           # builders and query kernels
  python tests/golden/make_golden.py gpu_rebin   # on a B200: the reference's
                                           # rebinRadixBuilder trees
  python tests/golden/make_golden.py gpu_boxquery   # on a B200: the
                                           # reference's fixedBoxQuery results
  python tests/golden/make_golden.py gpu_wide   # on a B200: the reference's
                                           # WideBVH builds and queries
  python tests/golden/make_golden.py gpu_sah    # on a B200: the reference's
                                           # SAH and ELH builds, evaluateSAH/ELH

Both read oracle/_ref/ (the reference compiled from its own sources by
oracle/build_ref.sh).  Inputs are the seeded generators of
cubql_b200.workloads; trees are stored after BFS renumbering
(orc_canonicalize), because the reference's GPU builders number nodes in a
run-dependent order.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cubql_b200 import workloads as W  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def inputs():
    p = W.uniform_points(3000)
    q = W.uniform_points(600, W.SEED_QUERIES, -0.1, 1.1)
    g = W.gmm_points(3000)
    gq = W.gmm_points(600, seed=W.SEED_GMM + 100)
    verts, tris = W.icosphere(2)
    tq = W.uniform_points(400, W.SEED_QUERIES, -1.5, 1.5)
    return p, q, g, gq, verts, tris, tq


def cpu():
    from oracle.oracle import RefCPU
    r = RefCPU()
    p, q, g, gq, verts, tris, tq = inputs()
    out = {}
    for name, pts, qs in (("u", p, q), ("g", g, gq)):
        b = W.point_boxes(pts)
        for thr in (0, 8):
            n, pr = r.build(b, thr)
            out[f"{name}_cpu{thr}_nodes"] = n.view(np.uint8)
            out[f"{name}_cpu{thr}_prims"] = pr
        n, pr = r.build(b, 8)
        ids, d = r.closest_point(n, pr, pts, qs)
        out[f"{name}_cp_ids"], out[f"{name}_cp_d"] = ids, d
        # blacklists: exclude one id per query (here the query's own index, on
        # queries that are data points) or every point at the query position
        sq = pts[:400]
        out[f"{name}_exself_ids"], out[f"{name}_exself_d"] = r.closest_point_exclude(n, pr, pts, sq)
        exid = np.arange(400, dtype=np.int32)
        exid[::7] = -1
        out[f"{name}_exid_ids"], out[f"{name}_exid_d"] = r.closest_point_exclude(n, pr, pts, sq, exclude_ids=exid)
        for k in (5, 16):
            ki, kd, kn = r.knn(n, pr, pts, qs, k)
            out[f"{name}_knn{k}_ids"], out[f"{name}_knn{k}_d"], out[f"{name}_knn{k}_n"] = ki, kd, kn
    tb = np.stack([verts[tris].min(1), verts[tris].max(1)], 1).reshape(-1, 6)
    n, pr = r.build(tb, 4)
    ids, d, P = r.tri_closest(n, pr, tris, verts, tq)
    out["tri_nodes"], out["tri_prims"] = n.view(np.uint8), pr
    out["tri_ids"], out["tri_d"], out["tri_P"] = ids, d, P
    np.savez_compressed(os.path.join(HERE, "ref_cpu.npz"), **out)


def gpu():
    from oracle.oracle import RefGPU
    r = RefGPU()
    o = Oracle()
    p, q, g, gq, verts, tris, tq = inputs()
    out = {}
    for name, pts, qs in (("u", p, q), ("g", g, gq)):
        b = W.point_boxes(pts)
        for method, mname in ((RefGPU.RADIX, "radix"), (RefGPU.SPATIAL_MEDIAN, "sm")):
            for thr in (0, 8):
                n, pr = r.build(method, b, thr)
                cn, cp = o.canonicalize(n, pr)
                out[f"{name}_{mname}{thr}_nodes"] = cn.view(np.uint8)
                out[f"{name}_{mname}{thr}_prims"] = cp
        n, pr = r.build(RefGPU.RADIX, b, 0)
        ids, d = r.closest_point(n, pr, pts, qs)
        out[f"{name}_cp_ids"], out[f"{name}_cp_d"] = ids, d
        ki, kd, kn = r.knn(n, pr, pts, qs, 16)
        out[f"{name}_knn16_ids"], out[f"{name}_knn16_d"], out[f"{name}_knn16_n"] = ki, kd, kn
        cn, cp = o.canonicalize(n, pr)
        out[f"{name}_querytree_nodes"], out[f"{name}_querytree_prims"] = cn.view(np.uint8), cp
    # FMA shape of the two distance expressions
    a = W.uniform_points(4096, 5, -2, 2)
    bb = W.uniform_points(4096, 6, -2, 2)
    lo = W.uniform_points(4096, 7, -1, 1)
    hi = lo + np.abs(W.uniform_points(4096, 8, 0, 1))
    boxes = np.concatenate([lo, hi], 1)
    pp, pb = r.pin(a, bb, boxes)
    out["pin_a"], out["pin_b"], out["pin_boxes"], out["pin_pp"], out["pin_pbox"] = a, bb, boxes, pp, pb
    tb = np.stack([verts[tris].min(1), verts[tris].max(1)], 1).reshape(-1, 6)
    n, pr = r.build(RefGPU.RADIX, tb, 0)
    ids, d, P = r.tri_closest(n, pr, tris, verts, tq)
    cn, cp = o.canonicalize(n, pr)
    out["tri_nodes"], out["tri_prims"] = cn.view(np.uint8), cp
    out["tri_ids"], out["tri_d"], out["tri_P"] = ids, d, P
    dest = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu.npz")
    np.savez_compressed(dest, **out)


def rebin_inputs():
    """Uniform, GMM, and a tight cluster inside a wide cloud (many equal
    30-bit Morton keys: exercises the rebin restarts)."""
    u = W.uniform_points(3000)
    g = W.gmm_points(3000)
    wide = W.uniform_points(1000, 21, -1000.0, 1000.0)
    tight = W.uniform_points(3000, 22, 0.0, 1e-3)
    return (("u", u), ("g", g), ("c", np.concatenate([wide, tight]).astype(np.float32)))


def gpu_rebin():
    from oracle.oracle import RefGPU
    r = RefGPU()
    o = Oracle()
    out = {}
    for name, pts in rebin_inputs():
        b = W.point_boxes(pts)
        out[f"{name}_points"] = pts
        for thr in (0, 8):
            n, pr = r.build(RefGPU.REBIN, b, thr)
            cn, cp = o.canonicalize(n, pr)
            out[f"{name}_rebin{thr}_nodes"] = cn.view(np.uint8)
            out[f"{name}_rebin{thr}_prims"] = cp
    dest = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_rebin.npz")
    np.savez_compressed(dest, **out)


def boxquery_inputs():
    """Point boxes (uniform) and boxes with extents (GMM centres, half sizes
    up to 0.02), each with 500 query boxes of three sizes, some outside."""
    rng = np.random.default_rng(7)
    u = W.point_boxes(W.uniform_points(3000))
    g = W.gmm_points(3000, offset=0.0)
    h = rng.uniform(0.0, 0.02, size=g.shape).astype(np.float32)
    e = np.concatenate([g - h, g + h], 1).astype(np.float32)
    c = W.uniform_points(500, W.SEED_QUERIES, -0.1, 1.1)
    qh = np.repeat(np.array([0.0, 0.01, 0.08], np.float32), [100, 200, 200])[:, None] * np.ones((1, 3), np.float32)
    q = np.concatenate([c - qh, c + qh], 1).astype(np.float32)
    return (("u", u, q), ("e", e, q))


def gpu_boxquery():
    from oracle.oracle import RefGPU
    r = RefGPU()
    o = Oracle()
    out = {}
    for name, boxes, q in boxquery_inputs():
        out[f"{name}_boxes"], out[f"{name}_queries"] = boxes, q
        for thr in (0, 8):
            n, pr = r.build(RefGPU.RADIX, boxes, thr)
            cn, cp = o.canonicalize(n, pr)
            off, ids = r.box_query(cn, cp, boxes, q)
            out[f"{name}{thr}_nodes"], out[f"{name}{thr}_prims"] = cn.view(np.uint8), cp
            out[f"{name}{thr}_offsets"], out[f"{name}{thr}_ids"] = off, ids
    dest = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_boxquery.npz")
    np.savez_compressed(dest, **out)


def gpu_wide():
    """For uniform and GMM points (3000, unshifted): the reference's binary
    spatial-median tree and its WideBVH<float,3,4|8> builds (leaf 1 and 8),
    both BFS-renumbered, plus the raw wide trees with the reference's
    closest-point and box-query results on them."""
    from oracle.oracle import RefGPU
    r = RefGPU()
    o = Oracle()
    out = {}
    rng = np.random.default_rng(5)
    for name, pts in (("u", W.uniform_points(3000)), ("g", W.gmm_points(3000, offset=0.0))):
        b = W.point_boxes(pts)
        q = W.uniform_points(600, W.SEED_QUERIES, -0.1, 1.1)
        h = rng.uniform(0.0, 0.06, size=(600, 1)).astype(np.float32)
        qb = np.concatenate([q - h, q + h], 1).astype(np.float32)
        out[f"{name}_points"], out[f"{name}_queries"], out[f"{name}_qboxes"] = pts, q, qb
        for thr in (0, 8):
            n, pr = r.build(RefGPU.SPATIAL_MEDIAN, b, thr)
            cn, cp = o.canonicalize(n, pr)
            out[f"{name}{thr}_bin_nodes"], out[f"{name}{thr}_bin_prims"] = cn.view(np.uint8), cp
            for width in (4, 8):
                sl, wp = r.build_wide(width, b, thr)
                cs, cwp = o.wide_canonicalize(sl, width, wp)
                key = f"{name}{thr}_w{width}"
                out[f"{key}_canon"], out[f"{key}_canon_prims"] = cs.view(np.uint8), cwp
                out[f"{key}_raw"], out[f"{key}_raw_prims"] = sl.view(np.uint8), wp
                ids, d = r.wide_closest(width, sl, wp, pts, q)
                out[f"{key}_cp_ids"], out[f"{key}_cp_d"] = ids, d
                off, bids = r.wide_box_query(width, sl, wp, b, qb)
                out[f"{key}_box_off"], out[f"{key}_box_ids"] = off, bids
    dest = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_wide.npz")
    np.savez_compressed(dest, **out)


def sah_pin_inputs(n=4000, seed=9):
    """Seeded SAH bin sets for pinning evaluateSAH: half with coordinates on
    a 1/8 grid (many exactly equal costs: tie rules), half with full
    mantissas (rounding shapes); counts 0..4, empty bins as AtomicBox
    leaves them (+-FLT_MAX encoded); plus boxes for surfaceArea."""
    from oracle.oracle import SAH_BINS

    def enc(f):
        b = np.asarray(f, np.float32).view(np.int32)
        return np.where(b < 0, b ^ np.int32(0x7fffffff), b).astype(np.int32)

    rng = np.random.default_rng(seed)
    bins = np.zeros(n, dtype=SAH_BINS)
    cnt = rng.integers(0, 5, size=(n, 3, 16))
    cnt[rng.random((n, 3, 16)) < 0.3] = 0
    lo = rng.random((n, 3, 16, 3)).astype(np.float32)
    ext = (rng.random((n, 3, 16, 3)) * 0.3).astype(np.float32)
    grid = np.arange(n) < n // 2
    lo[grid] = np.floor(lo[grid] * 8) / 8
    ext[grid] = np.floor(ext[grid] * 8) / 8
    hi = (lo + ext).astype(np.float32)
    empty = cnt == 0
    flt_max = np.float32(3.4028234663852886e38)
    lo[empty] = flt_max
    hi[empty] = -flt_max
    bins["b"]["lo"] = enc(lo)
    bins["b"]["hi"] = enc(hi)
    bins["b"]["count"] = cnt
    bl = rng.random((n, 3)).astype(np.float32) * 10
    boxes = np.concatenate([bl, bl + rng.random((n, 3)).astype(np.float32)], 1).astype(np.float32)
    return bins, boxes


def sah_tree_inputs():
    """Point boxes (uniform, GMM), triangle boxes of an icosphere and boxes
    with random extents."""
    rng = np.random.default_rng(12)
    verts, tris = W.icosphere(3)
    tb = np.stack([verts[tris].min(1), verts[tris].max(1)], 1).reshape(-1, 6).astype(np.float32)
    c = W.uniform_points(2000, 33)
    h = (rng.random((2000, 3)) * 0.05).astype(np.float32)
    return (("u", W.point_boxes(W.uniform_points(3000))), ("g", W.point_boxes(W.gmm_points(3000, offset=0.0))),
            ("t", tb), ("e", np.concatenate([c - h, c + h], 1).astype(np.float32)))


def gpu_sah():
    from oracle.oracle import RefGPU
    r = RefGPU()
    o = Oracle()
    out = {}
    bins, boxes = sah_pin_inputs()
    out["pin_dims"], out["pin_bins"], out["pin_areas"] = r.sah_pin(bins, boxes)
    out["elh_pin_dims"], out["elh_pin_bins"] = r.elh_pin(bins)
    for name, b in sah_tree_inputs():
        out[f"{name}_boxes"] = b
        for thr in (0, 4):
            n, pr = r.build(RefGPU.SAH, b, thr)
            cn, cp = o.canonicalize(n, pr)
            out[f"{name}{thr}_nodes"], out[f"{name}{thr}_prims"] = cn.view(np.uint8), cp
            n, pr = r.build(RefGPU.ELH, b, thr)
            cn, cp = o.canonicalize(n, pr)
            out[f"{name}{thr}_elh_nodes"], out[f"{name}{thr}_elh_prims"] = cn.view(np.uint8), cp
    dest = sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "ref_gpu_sah.npz")
    np.savez_compressed(dest, **out)


if __name__ == "__main__":
    {"cpu": cpu, "gpu": gpu, "gpu_rebin": gpu_rebin, "gpu_boxquery": gpu_boxquery,
     "gpu_wide": gpu_wide, "gpu_sah": gpu_sah}[sys.argv[1]]()
