"""CPU-only checks: the oracle (C restatement) against the reference's own
outputs (golden fixtures made by tests/golden/make_golden.py from the
reference compiled from its sources), plus the oracle's own invariants."""
import os

import numpy as np
import pytest

from cubql_b200 import workloads as W
from oracle.oracle import NODE, check_tree
from tests.helpers import boxes_np, fp64_closest, same_tree, tri_boxes_np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path)


def test_generator_matches_c_restatement(oracle):
    for seed, lo, hi in ((W.SEED_DATA, 0.0, 1.0), (W.SEED_QUERIES, -0.1, 1.1), (3, -1.5, 1.5)):
        a = W.uniform_points(5000, seed, lo, hi)
        b = oracle.uniform_points(5000, seed, lo, hi)
        assert np.array_equal(a, b)


def test_cpu_builder_matches_reference(oracle):
    g = _load("ref_cpu.npz")
    p, q, gp, gq, verts, tris, tq = _inputs()
    for name, pts in (("u", p), ("g", gp)):
        for thr in (0, 8):
            n, pr = oracle.cpu_build(boxes_np(pts), thr)
            assert n.view(np.uint8).tobytes() == g[f"{name}_cpu{thr}_nodes"].tobytes()
            assert np.array_equal(pr, g[f"{name}_cpu{thr}_prims"])


def _inputs():
    p = W.uniform_points(3000)
    q = W.uniform_points(600, W.SEED_QUERIES, -0.1, 1.1)
    g = W.gmm_points(3000)
    gq = W.gmm_points(600, seed=W.SEED_GMM + 100)
    verts, tris = W.icosphere(2)
    tq = W.uniform_points(400, W.SEED_QUERIES, -1.5, 1.5)
    return p, q, g, gq, verts, tris, tq


def test_host_queries_match_reference(oracle):
    """Reference host build (no FMA on x86-64) + reference traversal rules."""
    g = _load("ref_cpu.npz")
    p, q, gp, gq, *_ = _inputs()
    for name, pts, qs in (("u", p, q), ("g", gp, gq)):
        n = g[f"{name}_cpu8_nodes"].view(NODE)
        pr = g[f"{name}_cpu8_prims"]
        ids, d, ovf, _ = oracle.closest_point(n, pr, pts, qs, fma_mode=0, tie_mode=1)
        assert not ovf.any()
        assert np.array_equal(ids, g[f"{name}_cp_ids"]) and np.array_equal(d, g[f"{name}_cp_d"])
        for k in (5, 16):
            ki, kd, kn, _ = oracle.knn(n, pr, pts, qs, k, fma_mode=0, tie_mode=1)
            assert np.array_equal(ki, g[f"{name}_knn{k}_ids"])
            assert np.array_equal(kd, g[f"{name}_knn{k}_d"])
            assert np.array_equal(kn, g[f"{name}_knn{k}_n"])


def test_host_triangles_match_reference(oracle):
    g = _load("ref_cpu.npz")
    *_, verts, tris, tq = _inputs()
    n = g["tri_nodes"].view(NODE)
    ids, d, P = oracle.tri_closest(n, g["tri_prims"], tris, verts, tq)
    assert np.array_equal(ids, g["tri_ids"])
    assert np.array_equal(d, g["tri_d"])
    assert np.array_equal(P, g["tri_P"])


def test_gpu_reference_trees_match_oracle(oracle):
    """Pins the Morton and spatial-median restatements on the reference's
    GPU builders (fixtures produced on a B200)."""
    g = _load("ref_gpu.npz")
    p, q, gp, gq, *_ = _inputs()
    for name, pts in (("u", p), ("g", gp)):
        b = boxes_np(pts)
        for thr in (0, 8):
            n, pr = oracle.radix_build(b, thr)
            ok, msg = same_tree(oracle, n, pr, g[f"{name}_radix{thr}_nodes"].view(NODE), g[f"{name}_radix{thr}_prims"])
            assert ok, f"radix {name} thr {thr}: {msg}"
    # spatial median: identical wherever no node is degenerate (uniform data)
    for thr in (0, 8):
        n, pr = oracle.sm_build(boxes_np(p), thr)
        ok, msg = same_tree(oracle, n, pr, g[f"u_sm{thr}_nodes"].view(NODE), g[f"u_sm{thr}_prims"])
        assert ok, f"spatial median thr {thr}: {msg}"


def test_gpu_reference_distance_contraction(oracle):
    """The FMA shapes the oracle uses for fma_mode=1 equal what nvcc made of
    the reference's two distance expressions on a B200."""
    g = _load("ref_gpu.npz")
    assert np.array_equal(oracle.sqr_pp(g["pin_a"], g["pin_b"], 1), g["pin_pp"])
    assert np.array_equal(oracle.sqr_pbox(g["pin_a"], g["pin_boxes"], 1), g["pin_pbox"])


def test_gpu_reference_queries_match_oracle(oracle):
    g = _load("ref_gpu.npz")
    p, q, gp, gq, *_ = _inputs()
    for name, pts, qs in (("u", p, q), ("g", gp, gq)):
        n = g[f"{name}_querytree_nodes"].view(NODE)
        pr = g[f"{name}_querytree_prims"]
        ids, d, ovf, _ = oracle.closest_point(n, pr, pts, qs, fma_mode=1, tie_mode=1)
        assert not ovf.any()
        assert np.array_equal(ids, g[f"{name}_cp_ids"]) and np.array_equal(d, g[f"{name}_cp_d"])
        ki, kd, kn, _ = oracle.knn(n, pr, pts, qs, 16, fma_mode=1, tie_mode=1)
        assert np.array_equal(ki, g[f"{name}_knn16_ids"]) and np.array_equal(kd, g[f"{name}_knn16_d"])
        assert np.array_equal(kn, g[f"{name}_knn16_n"])


@pytest.mark.parametrize("thr", [0, 1, 3, 8])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "invalid"])
def test_radix_oracle_invariants(oracle, thr, dist):
    pts = _dist(dist, 4000)
    b = boxes_np(pts)
    if dist == "invalid":
        b[::7, 0] = 2.0
        b[::7, 3] = 1.0
    n, pr = oracle.radix_build(b, thr)
    check_tree(n, pr, b, max_leaf=max(thr, 1))


@pytest.mark.parametrize("thr", [0, 1, 8])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "invalid"])
def test_spatial_median_oracle_invariants(oracle, thr, dist):
    pts = _dist(dist, 4000)
    b = boxes_np(pts)
    if dist == "invalid":
        b[::7, 0] = 2.0
        b[::7, 3] = 1.0
    n, pr = oracle.sm_build(b, thr)
    valid = ~(b[:, 0] > b[:, 3])
    check_tree(n, pr[: valid.sum()], b, max_leaf=max(thr, 1))


def _dist(dist, n):
    if dist == "uniform" or dist == "invalid":
        return W.uniform_points(n)
    if dist == "gmm":
        return W.gmm_points(n)
    pts = W.uniform_points(n // 10)
    return np.repeat(pts, 10, axis=0)  # every point ten times


def test_edge_sizes(oracle):
    for n in (1, 2, 3, 5):
        b = boxes_np(W.uniform_points(n))
        nr, pr = oracle.radix_build(b)
        assert len(nr) == 2 * n and sorted(pr.tolist()) == list(range(n))
        check_tree(nr, pr, b, max_leaf=1)
        ns, ps = oracle.sm_build(b)
        check_tree(ns, ps, b, max_leaf=1)
    nr, pr = oracle.radix_build(np.zeros((0, 6), np.float32))
    assert len(nr) == 0 and len(pr) == 0


def test_lowest_id_rule_is_tree_independent(oracle):
    pts = W.gmm_points(4000)
    qs = W.gmm_points(500, seed=123)
    b = boxes_np(pts)
    a = oracle.knn(*oracle.radix_build(b), pts, qs, 8, tie_mode=0)
    c = oracle.knn(*oracle.sm_build(b, 8), pts, qs, 8, tie_mode=0)
    d = oracle.knn(*oracle.cpu_build(b, 3), pts, qs, 8, tie_mode=0)
    for x in (c, d):
        assert np.array_equal(a[0], x[0]) and np.array_equal(a[1], x[1])


def test_closest_within_fp64(oracle):
    pts = W.uniform_points(5000)
    qs = W.uniform_points(700, W.SEED_QUERIES, -0.1, 1.1)
    ids, d, _, _ = oracle.closest_point(*oracle.radix_build(boxes_np(pts)), pts, qs)
    d64, i64 = fp64_closest(pts, qs)
    assert np.all(np.abs(d - d64) <= 1e-6 * d64 + 1e-30)


def test_canonicalize_idempotent(oracle):
    b = boxes_np(W.uniform_points(3000))
    c1 = oracle.canonicalize(*oracle.radix_build(b, 4))
    c2 = oracle.canonicalize(*c1)
    assert c1[0].tobytes() == c2[0].tobytes() and np.array_equal(c1[1], c2[1])


def test_adjoint_formula_matches_finite_differences(oracle):
    """FP64 analytic gradient of the point-to-triangle squared distance
    against FP64 central differences (tolerance 1e-5 relative)."""
    rng = np.random.default_rng(0)
    for _ in range(200):
        a, b, c = rng.normal(size=(3, 3))
        p = rng.normal(size=3) * 1.5
        d0, w = oracle.tri_cp_f64(a, b, c, p)
        X = w[0] * a + w[1] * b + w[2] * c
        gq = 2 * (p - X)
        h = 1e-6
        fd = np.zeros(3)
        for i in range(3):
            e = np.zeros(3)
            e[i] = h
            fd[i] = (oracle.tri_cp_f64(a, b, c, p + e)[0] - oracle.tri_cp_f64(a, b, c, p - e)[0]) / (2 * h)
        assert np.allclose(gq, fd, rtol=1e-5, atol=1e-7)
        fa = np.zeros(3)
        for i in range(3):
            e = np.zeros(3)
            e[i] = h
            fa[i] = (oracle.tri_cp_f64(a + e, b, c, p)[0] - oracle.tri_cp_f64(a - e, b, c, p)[0]) / (2 * h)
        assert np.allclose(-w[0] * gq, fa, rtol=1e-5, atol=1e-6)


def test_rebin_restatement_matches_reference_gpu_trees(oracle):
    """orc_rebin_build against the reference's rebinRadixBuilder run on a
    B200 (fixtures: uniform, GMM and a tight cluster inside a wide cloud,
    which forces nested rebins); trees after BFS renumbering, bit for bit,
    leaf prim order included."""
    g = _load("ref_gpu_rebin.npz")
    for name in ("u", "g", "c"):
        b = boxes_np(g[f"{name}_points"])
        for thr in (0, 8):
            n, pr = oracle.rebin_build(b, thr)
            cn, cp = oracle.canonicalize(n, pr)
            ref = g[f"{name}_rebin{thr}_nodes"].view(NODE).copy()
            cn = cn.copy()
            cn[1] = np.zeros(1, dtype=NODE)
            ref[1] = np.zeros(1, dtype=NODE)
            assert np.array_equal(cp, g[f"{name}_rebin{thr}_prims"]), (name, thr)
            assert cn.tobytes() == ref.tobytes(), (name, thr)
            check_tree(n, pr, b, max_leaf=max(thr, 32))


def test_exclude_blacklists_match_reference(oracle):
    """findClosest_exludeID / findClosest_exludeSelf (findClosest.h:278-334)
    restated in the oracle, against the reference's host code: 400 queries
    that are data points, excluding their own index (every 7th: -1, nothing
    excluded) or every point at their position."""
    g = _load("ref_cpu.npz")
    p, q, gp, gq, *_ = _inputs()
    for name, pts in (("u", p), ("g", gp)):
        n = g[f"{name}_cpu8_nodes"].view(NODE)
        pr = g[f"{name}_cpu8_prims"]
        sq = pts[:400]
        ids, d = oracle.closest_point_exclude(n, pr, pts, sq, exclude_self=True, fma_mode=0, tie_mode=1)
        assert np.array_equal(ids, g[f"{name}_exself_ids"]) and np.array_equal(d, g[f"{name}_exself_d"])
        exid = np.arange(400, dtype=np.int32)
        exid[::7] = -1
        ids, d = oracle.closest_point_exclude(n, pr, pts, sq, exclude_ids=exid, fma_mode=0, tie_mode=1)
        assert np.array_equal(ids, g[f"{name}_exid_ids"]) and np.array_equal(d, g[f"{name}_exid_d"])
        assert (ids[exid >= 0] != exid[exid >= 0]).all()


def _brute_box(boxes, q):
    lo, hi = boxes[:, :3], boxes[:, 3:]
    return ~((q[None, 3:] < lo).any(1) | (hi < q[None, :3]).any(1))


def test_box_query_oracle_matches_brute_force(oracle):
    """fixedBoxQuery restated (fixedBoxQuery.h:73-156, per-prim box test):
    each query's prims are exactly the closed-interval overlaps, each once;
    point boxes and boxes with extents, several leaf sizes, query boxes
    that are points, small, large, outside everything or inverted."""
    rng = np.random.default_rng(3)
    c = W.gmm_points(4000, offset=0.0)
    h = rng.uniform(0, 0.01, size=c.shape).astype(np.float32)
    for boxes in (boxes_np(W.uniform_points(4000)), np.concatenate([c - h, c + h], 1).astype(np.float32)):
        qc = W.uniform_points(300, W.SEED_QUERIES, -0.2, 1.2)
        qh = rng.choice(np.float32([0, 0.005, 0.05, 0.3, -0.01]), size=(300, 1)).astype(np.float32)
        q = np.concatenate([qc - qh, qc + qh], 1).astype(np.float32)
        q[0] = [5, 5, 5, 6, 6, 6]
        q[1] = [-1, -1, -1, 2, 2, 2]
        for thr in (0, 1, 8):
            n, pr = oracle.radix_build(boxes, thr)
            off, ids = oracle.box_query(n, pr, boxes, q)
            assert off[0] == 0 and off[1] == 0 and off[2] - off[1] == len(boxes)
            for i in range(len(q)):
                got = ids[off[i]:off[i + 1]]
                assert len(np.unique(got)) == len(got)
                assert np.array_equal(np.sort(got), np.nonzero(_brute_box(boxes, q[i]))[0]), (thr, i)


def test_box_query_matches_reference_gpu_fixtures(oracle):
    """The oracle's box query against the reference's fixedBoxQuery kernel
    run on a B200 (fixtures over the reference's radix trees, BFS
    renumbered): same prims in the same visiting order."""
    g = _load("ref_gpu_boxquery.npz")
    for name in ("u", "e"):
        boxes, q = g[f"{name}_boxes"], g[f"{name}_queries"]
        for thr in (0, 8):
            n = g[f"{name}{thr}_nodes"].view(NODE)
            pr = g[f"{name}{thr}_prims"]
            off, ids = oracle.box_query(n, pr, boxes, q)
            assert np.array_equal(off, g[f"{name}{thr}_offsets"]), (name, thr)
            assert np.array_equal(ids, g[f"{name}{thr}_ids"]), (name, thr)
            assert off[-1] > 2 * len(q)


def _wide_leaf_prims(slots, prims):
    v = (slots["admin"] & np.uint64(1)).astype(bool)
    cnt = ((slots["admin"] >> np.uint64(46)) & np.uint64(0xFFFF)).astype(np.int64)
    off = ((slots["admin"] >> np.uint64(1)) & np.uint64((1 << 45) - 1)).astype(np.int64)
    leaf = v & (cnt > 0)
    return np.concatenate([prims[o:o + c] for o, c in zip(off[leaf], cnt[leaf])]) if leaf.any() else np.zeros(0)


@pytest.mark.parametrize("width", [2, 4, 8])
def test_wide_collapse_oracle_invariants(oracle, width):
    """The collapse (wide_gpu_builder.h:40-158) restated: every prim reached
    once, inner slots point at wide nodes, slot boxes are binary node boxes,
    and the wide tree answers closest-point (lowest-id rule) and box
    queries exactly as the binary tree it came from."""
    pts = W.uniform_points(4000)
    b = boxes_np(pts)
    q = W.uniform_points(300, W.SEED_QUERIES, -0.1, 1.1)
    qb = np.concatenate([q - 0.03, q + 0.03], 1).astype(np.float32)
    for build in ("sm", "radix"):
        for thr in (0, 8):
            n, pr = oracle.sm_build(b, thr) if build == "sm" else oracle.radix_build(b, thr)
            sl = oracle.wide_collapse(n, width)
            nw = len(sl) // width
            assert np.array_equal(np.sort(_wide_leaf_prims(sl, pr)), np.arange(len(pts)))
            v = (sl["admin"] & np.uint64(1)).astype(bool)
            cnt = (sl["admin"] >> np.uint64(46)) & np.uint64(0xFFFF)
            off = (sl["admin"] >> np.uint64(1)) & np.uint64((1 << 45) - 1)
            inner = v & (cnt == 0)
            assert (off[inner] < nw).all() and (off[inner] > 0).all()
            assert np.all(sl["lower"][~v] == np.inf) and np.all(sl["upper"][~v] == -np.inf)
            cs, cp = oracle.wide_canonicalize(sl, width, pr)
            assert len(cs) == len(sl)
            bi, bd, _, _ = oracle.closest_point(n, pr, pts, q, fma_mode=1, tie_mode=0)
            wi, wd = oracle.wide_closest(sl, width, pr, pts, q, fma_mode=1, tie_mode=0)
            assert np.array_equal(bi, wi) and np.array_equal(bd, wd)
            off_b, ids_b = oracle.box_query(n, pr, b, qb)
            off_w, ids_w = oracle.wide_box_query(sl, width, pr, b, qb)
            assert np.array_equal(off_b, off_w)
            for i in range(len(q)):
                assert np.array_equal(np.sort(ids_b[off_b[i]:off_b[i + 1]]), np.sort(ids_w[off_w[i]:off_w[i + 1]]))


def test_wide_oracle_matches_reference_gpu_fixtures(oracle):
    """Against the reference run on a B200 (gpuBuilder into WideBVH<float,3,
    4|8>, uniform and GMM points, leaf 1 and 8): the oracle's collapse of the
    reference's binary tree equals the reference's wide tree after BFS
    renumbering; on the reference's own wide trees the oracle's closest point
    (reference tie rule, device FMA shapes) and box query equal the
    reference's kernels."""
    g = _load("ref_gpu_wide.npz")
    for name in ("u", "g"):
        pts, q, qb = g[f"{name}_points"], g[f"{name}_queries"], g[f"{name}_qboxes"]
        b = boxes_np(pts)
        for thr in (0, 8):
            n = g[f"{name}{thr}_bin_nodes"].view(NODE)
            pr = g[f"{name}{thr}_bin_prims"]
            for width in (4, 8):
                key = f"{name}{thr}_w{width}"
                sl = oracle.wide_collapse(n, width)
                cs, cp = oracle.wide_canonicalize(sl, width, pr)
                assert cs.tobytes() == g[f"{key}_canon"].tobytes(), key
                assert np.array_equal(cp, g[f"{key}_canon_prims"]), key
                raw, rp = g[f"{key}_raw"].view(NODE), g[f"{key}_raw_prims"]
                ids, d = oracle.wide_closest(raw, width, rp, pts, q, fma_mode=1, tie_mode=1)
                assert np.array_equal(ids, g[f"{key}_cp_ids"]) and np.array_equal(d, g[f"{key}_cp_d"]), key
                off, bids = oracle.wide_box_query(raw, width, rp, b, qb)
                assert np.array_equal(off, g[f"{key}_box_off"]) and np.array_equal(bids, g[f"{key}_box_ids"]), key


def test_sah_oracle_invariants(oracle):
    """SAH restatement (sah_builder.h): valid trees, every prim once, leaves
    in ascending primID order, and a lower SAH cost than spatial median on
    triangle boxes."""
    verts, tris = W.icosphere(3)
    tb = tri_boxes_np(verts, tris)
    for b in (boxes_np(W.uniform_points(3000)), tb):
        for thr in (0, 4):
            n, pr = oracle.sah_build(b, thr)
            check_tree(n, pr, b, max_leaf=None)
            cnt = (n["admin"] >> np.uint64(48)).astype(np.int64)
            off = (n["admin"] & np.uint64(0xFFFFFFFFFFFF)).astype(np.int64)
            for o, c in zip(off[cnt > 0], cnt[cnt > 0]):
                assert np.all(np.diff(pr[o:o + c].astype(np.int64)) > 0)

    def sah_cost(n):
        lo, hi = n["lower"].astype(np.float64), n["upper"].astype(np.float64)
        s = hi - lo
        a = s[:, 0] * s[:, 1] + s[:, 0] * s[:, 2] + s[:, 1] * s[:, 2]
        cnt = (n["admin"] >> np.uint64(48)).astype(np.float64)
        keep = np.ones(len(n), bool)
        keep[1] = False
        return float((a * np.where(cnt > 0, cnt, 1.0))[keep].sum() / a[0])
    assert sah_cost(oracle.sah_build(tb, 0)[0]) < sah_cost(oracle.sm_build(tb, 1)[0])


def test_sah_oracle_matches_reference_gpu_fixtures(oracle):
    """Against the reference's sahBuilder and evaluateSAH run on a B200:
    evaluateSAH decisions and surfaceArea values on seeded bin sets (1/8-grid
    coordinates for exact ties, full mantissas for rounding), and whole
    trees (point, triangle and extent boxes; leaf threshold 0 and 4) after
    BFS renumbering."""
    from tests.golden.make_golden import sah_pin_inputs
    g = _load("ref_gpu_sah.npz")
    bins, boxes = sah_pin_inputs()
    dims, sb = oracle.sah_evaluate(bins, fma_mode=1)
    assert np.array_equal(dims, g["pin_dims"])
    assert np.array_equal(np.where(dims < 0, 0, sb), g["pin_bins"])
    assert np.array_equal(oracle.sah_area(boxes, fma_mode=1), g["pin_areas"])
    for name in ("u", "g", "t", "e"):
        b = g[f"{name}_boxes"]
        for thr in (0, 4):
            for heur, tag in ((0, ""), (1, "_elh")):
                if f"{name}{thr}{tag}_nodes" not in g.files:
                    continue
                n, pr = oracle.sah_build(b, thr, heur=heur)
                cn, cp = oracle.canonicalize(n, pr)
                ref = g[f"{name}{thr}{tag}_nodes"].view(NODE).copy()
                cn = cn.copy()
                cn[1] = np.zeros(1, dtype=NODE)
                ref[1] = np.zeros(1, dtype=NODE)
                assert len(cn) == len(ref), (name, thr, heur)
                assert cn.tobytes() == ref.tobytes(), (name, thr, heur)
                assert np.array_equal(cp, g[f"{name}{thr}{tag}_prims"]), (name, thr, heur)


def test_elh_oracle_matches_reference_gpu_fixtures(oracle):
    """The edge-length heuristic (elh_builder.h, gpuBuilder with
    BuildConfig::ELH): evaluateELH decisions on the seeded bin sets (first 8
    bins per axis) against the reference's own device function; its trees are
    checked in test_sah_oracle_matches_reference_gpu_fixtures."""
    from tests.golden.make_golden import sah_pin_inputs
    g = _load("ref_gpu_sah.npz")
    if "elh_pin_dims" not in g.files:
        pytest.skip("ELH fixtures not generated")
    bins, _ = sah_pin_inputs()
    dims, sb = oracle.sah_evaluate(bins, fma_mode=1, heur=1)
    assert np.array_equal(dims, g["elh_pin_dims"])
    assert np.array_equal(np.where(dims < 0, 0, sb), g["elh_pin_bins"])
