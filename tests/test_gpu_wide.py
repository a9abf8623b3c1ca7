"""WideBVH<float,3,W> on the GPU: collapse, build, closest point and box
queries.

Bit-exact against (a) the oracle's restatement of the collapse and of the
wide traversals and (b) the reference's own gpuBuilder(WideBVH) and wide
query kernels compiled for sm_100a (trees compared after BFS renumbering,
since the reference numbers wide nodes in atomic order)."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np

pytestmark = pytest.mark.gpu


def _points(dist, n):
    if dist == "uniform":
        return W.uniform_points(n)
    if dist == "gmm":
        return W.gmm_points(n, offset=0.0)
    if dist == "dupes":
        return np.repeat(W.uniform_points(n // 8), 8, axis=0)
    raise ValueError(dist)


def _binary(bq, method, boxes, thr):
    b = torch.from_numpy(boxes).cuda()
    cfg = bq.BuildConfig(makeLeafThreshold=thr)
    if method == "morton":
        return bq.cuda.radixBuilder(b, cfg)
    if method == "rebin":
        return bq.cuda.rebinRadixBuilder(b, cfg)
    return bq.gpuBuilder(b, cfg)


def _wide_from_host(bq, slots, prims, width):
    """A WideBVH over device copies of host arrays (never freed through the
    library: torch owns the memory)."""
    st = torch.from_numpy(slots.view(np.uint8).copy()).cuda()
    pt = torch.from_numpy(np.ascontiguousarray(prims).view(np.int32).copy()).cuda()
    c = bq.bq_wide_bvh3f(st.data_ptr(), len(slots) // width, pt.data_ptr(), len(prims))
    w = bq.WideBVH(c, width, bq.default_allocator())
    w._keep = (st, pt)
    return w


@pytest.mark.parametrize("width", [2, 4, 8])
@pytest.mark.parametrize("method", ["morton", "sm", "rebin"])
@pytest.mark.parametrize("thr", [0, 8])
def test_collapse_matches_oracle(bq, oracle, width, method, thr):
    boxes = boxes_np(_points("gmm", 60000))
    bvh = _binary(bq, method, boxes, thr)
    n, pr = bvh.to_host()
    w = bq.collapse(bvh, width)
    sl, wp = w.to_host()
    osl = oracle.wide_collapse(n, width)
    assert sl.tobytes() == osl.tobytes()
    assert np.array_equal(wp, pr)
    w.free()
    bvh.free()


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("thr", [0, 8])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_wide_build_matches_reference(bq, oracle, ref_gpu, width, thr, dist):
    pts = _points(dist, 40000)
    boxes = boxes_np(pts)
    w = bq.gpuBuilderWide(torch.from_numpy(boxes).cuda(), width, bq.BuildConfig(makeLeafThreshold=thr))
    sl, wp = w.to_host()
    rsl, rwp = ref_gpu.build_wide(width, boxes, thr)
    cs, cp = oracle.wide_canonicalize(sl, width, wp)
    rcs, rcp = oracle.wide_canonicalize(rsl, width, rwp)
    assert len(cs) == len(rcs)
    assert cs.tobytes() == rcs.tobytes()
    # identical points (the seeded generators give a few even in "uniform")
    # may trade places: the reference's spatial-median builder is racy there
    assert np.array_equal(boxes[cp], boxes[rcp])
    assert np.array_equal(np.sort(cp), np.sort(rcp))
    w.free()


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_wide_closest_matches_oracle(bq, oracle, width, tie, dist):
    pts = _points(dist, 50000)
    qs = W.uniform_points(20000, W.SEED_QUERIES, -0.1, 1.1)
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    w = bq.gpuBuilderWide(torch.from_numpy(boxes_np(pts)).cuda(), width, bq.BuildConfig(makeLeafThreshold=8))
    sl, wp = w.to_host()
    for reorder in (0, 1):
        ids, d = bq.points.findClosest(w, tp, tq, qcfg=bq.query_config(tieMode=tie, reorder=reorder))
        oi, od = oracle.wide_closest(sl, width, wp, pts, qs, fma_mode=1, tie_mode=tie)
        assert np.array_equal(ids.cpu().numpy(), oi), reorder
        assert np.array_equal(d.cpu().numpy(), od), reorder
    if tie == 0:  # the lowest-id answer does not depend on the tree
        bvh = bq.cuda.radixBuilder(torch.from_numpy(boxes_np(pts)).cuda())
        bi, bd = bq.points.findClosest(bvh, tp, tq)
        assert torch.equal(bi, ids) and torch.equal(bd, d)
        bvh.free()
    w.free()


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_wide_queries_on_reference_trees(bq, ref_gpu, width, dist):
    """The reference's own wide tree (its numbering), our kernels with the
    reference tie rule against the reference's kernels."""
    pts = _points(dist, 30000)
    boxes = boxes_np(pts)
    qs = W.uniform_points(10000, W.SEED_QUERIES, -0.1, 1.1)
    rsl, rwp = ref_gpu.build_wide(width, boxes, 8)
    w = _wide_from_host(bq, rsl, rwp, width)
    ids, d = bq.points.findClosest(w, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(),
                                   qcfg=bq.query_config(tieMode=bq.TIES_REFERENCE))
    ri, rd = ref_gpu.wide_closest(width, rsl, rwp, pts, qs)
    assert np.array_equal(ids.cpu().numpy(), ri) and np.array_equal(d.cpu().numpy(), rd)
    rng = np.random.default_rng(2)
    h = rng.uniform(0, 0.03, size=(len(qs), 1)).astype(np.float32)
    qb = np.concatenate([qs - h, qs + h], 1).astype(np.float32)
    off, bids = bq.fixedBoxQuery.findPrims(w, torch.from_numpy(boxes).cuda(), torch.from_numpy(qb).cuda())
    roff, rbids = ref_gpu.wide_box_query(width, rsl, rwp, boxes, qb)
    assert np.array_equal(off.cpu().numpy(), roff) and np.array_equal(bids.cpu().numpy(), rbids)


@pytest.mark.parametrize("width", [2, 4, 8])
def test_wide_box_query_matches_oracle(bq, oracle, width):
    pts = _points("gmm", 50000)
    boxes = boxes_np(pts)
    w = bq.collapse(_binary(bq, "morton", boxes, 0), width)
    sl, wp = w.to_host()
    rng = np.random.default_rng(4)
    c = W.uniform_points(5000, W.SEED_QUERIES, -0.1, 1.1)
    h = rng.choice(np.float32([0, 0.005, 0.02, 0.1]), size=(5000, 1)).astype(np.float32)
    qb = np.concatenate([c - h, c + h], 1).astype(np.float32)
    off, ids = bq.fixedBoxQuery.findPrims(w, torch.from_numpy(boxes).cuda(), torch.from_numpy(qb).cuda())
    ooff, oids = oracle.wide_box_query(sl, width, wp, boxes, qb)
    assert np.array_equal(off.cpu().numpy(), ooff) and np.array_equal(ids.cpu().numpy(), oids)


@pytest.mark.parametrize("stack", [32, 64, 128])
def test_wide_stack_depths_and_deep_fallback(bq, oracle, stack):
    """W = 8 pushes up to 7 entries per level: with a 32-entry stack many
    clustered queries overflow and are re-run from the deep stack; the
    answers do not change."""
    pts = _points("gmm", 100000)
    qs = W.uniform_points(20000, W.SEED_QUERIES, -0.5, 1.5)
    w = bq.gpuBuilderWide(torch.from_numpy(boxes_np(pts)).cuda(), 8)
    sl, wp = w.to_host()
    for tie in (0, 1):
        ids, d = bq.points.findClosest(w, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(),
                                       qcfg=bq.query_config(tieMode=tie, stackDepth=stack))
        oi, od = oracle.wide_closest(sl, 8, wp, pts, qs, fma_mode=1, tie_mode=tie)
        assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)


def test_wide_edge_cases(bq, oracle):
    empty = bq.gpuBuilderWide(torch.zeros((0, 6), device="cuda"), 4)
    assert empty.numNodes == 0
    q = torch.from_numpy(W.uniform_points(100, W.SEED_QUERIES)).cuda()
    ids, d = bq.points.findClosest(empty, torch.zeros((0, 3), device="cuda"), q)
    assert (ids.cpu().numpy() == -1).all() and torch.isinf(d).all()
    one = W.uniform_points(1)
    w1 = bq.gpuBuilderWide(torch.from_numpy(boxes_np(one)).cuda(), 8)
    sl, wp = w1.to_host()
    assert w1.numNodes == 1 and wp.tolist() == [0]
    assert int(sl["admin"][0]) & 1 and all(int(a) & 1 == 0 for a in sl["admin"][1:])
    ids, d = bq.points.findClosest(w1, torch.from_numpy(one).cuda(), q)
    assert (ids.cpu().numpy() == 0).all()
    ids, d = bq.points.findClosest(w1, torch.from_numpy(one).cuda(), q, maxSqrDist=0.0)
    assert (ids.cpu().numpy() == -1).all()
    two = W.uniform_points(2)
    w2 = bq.gpuBuilderWide(torch.from_numpy(boxes_np(two)).cuda(), 4)
    oi, od = oracle.closest_point(*oracle.radix_build(boxes_np(two)), two, q.cpu().numpy(), fma_mode=1)[:2]
    ids, d = bq.points.findClosest(w2, torch.from_numpy(two).cuda(), q)
    assert np.array_equal(ids.cpu().numpy(), oi)
    with pytest.raises(bq.BQError):
        bq.gpuBuilderWide(torch.from_numpy(boxes_np(two)).cuda(), 3)


def test_wide_full_size_2m(bq, oracle):
    """2M uniform points, W = 4 and 8: the collapse equals the oracle's,
    200K queries equal the oracle's answers."""
    pts = W.uniform_points(2_000_000)
    boxes = boxes_np(pts)
    qs = W.uniform_points(200_000, W.SEED_QUERIES)
    bvh = _binary(bq, "sm", boxes, 8)
    n, pr = bvh.to_host()
    for width in (4, 8):
        w = bq.collapse(bvh, width)
        sl, wp = w.to_host()
        assert sl.tobytes() == oracle.wide_collapse(n, width).tobytes()
        ids, d = bq.points.findClosest(w, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda())
        oi, od = oracle.wide_closest(sl, width, wp, pts, qs, fma_mode=1, tie_mode=0)
        assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)
        w.free()
    bvh.free()
