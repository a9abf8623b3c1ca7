"""Fixed-box queries on the GPU (bq_box_query_count_f3 / bq_box_query_f3,
and the one-traversal bq_box_query_slab_f3 / bq_box_query_gather_f3).

Bit-exact, visiting order included, against (a) the oracle's restatement
of fixedBoxQuery::forEachPrim with a per-prim box test and (b) the
reference's own fixedBoxQuery kernel compiled for sm_100a, on the same
tree; sets checked against a brute force."""
import ctypes

import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np

pytestmark = pytest.mark.gpu


def _boxes(kind, n):
    if kind == "points":
        return boxes_np(W.uniform_points(n))
    rng = np.random.default_rng(11)
    c = W.gmm_points(n, offset=0.0)
    h = rng.uniform(0, 0.01, size=c.shape).astype(np.float32)
    return np.concatenate([c - h, c + h], 1).astype(np.float32)


def _queries(nq, seed=5):
    rng = np.random.default_rng(seed)
    c = W.uniform_points(nq, W.SEED_QUERIES, -0.2, 1.2)
    h = rng.choice(np.float32([0, 0.002, 0.01, 0.04, -0.01]), size=(nq, 1)).astype(np.float32)
    q = np.concatenate([c - h, c + h], 1).astype(np.float32)
    q[0] = [5, 5, 5, 6, 6, 6]          # outside everything
    q[1] = [-1, -1, -1, 2, 2, 2]       # contains everything
    return q


def _build(bq, method, boxes, thr):
    b = torch.from_numpy(boxes).cuda()
    cfg = bq.BuildConfig(makeLeafThreshold=thr)
    if method == "morton":
        return bq.cuda.radixBuilder(b, cfg)
    if method == "rebin":
        return bq.cuda.rebinRadixBuilder(b, cfg)
    return bq.gpuBuilder(b, bq.BuildConfig(makeLeafThreshold=thr or 8))


@pytest.mark.parametrize("method", ["morton", "sm", "rebin"])
@pytest.mark.parametrize("kind", ["points", "extents"])
@pytest.mark.parametrize("thr", [0, 8])
def test_box_query_matches_oracle(bq, oracle, method, kind, thr):
    boxes, q = _boxes(kind, 50000), _queries(5000)
    bvh = _build(bq, method, boxes, thr)
    n, pr = bvh.to_host()
    off, ids = bq.fixedBoxQuery.findPrims(bvh, torch.from_numpy(boxes).cuda(), torch.from_numpy(q).cuda())
    ooff, oids = oracle.box_query(n, pr, boxes, q)
    assert np.array_equal(off.cpu().numpy(), ooff)
    assert np.array_equal(ids.cpu().numpy(), oids)
    assert ooff[2] - ooff[1] == len(boxes) and ooff[1] == 0


@pytest.mark.parametrize("kind", ["points", "extents"])
def test_box_query_matches_reference_kernel(bq, oracle, ref_gpu, kind):
    boxes, q = _boxes(kind, 30000), _queries(3000, seed=9)
    bvh = _build(bq, "morton", boxes, 0)
    n, pr = bvh.to_host()
    off, ids = bq.fixedBoxQuery.findPrims(bvh, torch.from_numpy(boxes).cuda(), torch.from_numpy(q).cuda())
    roff, rids = ref_gpu.box_query(n, pr, boxes, q)
    assert np.array_equal(off.cpu().numpy(), roff)
    assert np.array_equal(ids.cpu().numpy(), rids)


@pytest.mark.parametrize("width", [0, 4, 8])
@pytest.mark.parametrize("cap", [0, 1, 4, 17, None])
def test_box_query_slab_capacities(bq, oracle, width, cap):
    """The one-traversal form (slab rows of `cap` ids, overflowing queries
    traversed again) equals the two-pass form (cap 0) and the oracle, for
    every row size: none, some or all of the queries overflow."""
    boxes, q = _boxes("extents", 40000), _queries(4000, seed=21)
    bvh = _build(bq, "morton", boxes, 8)
    n, pr = bvh.to_host()
    t = bvh if width == 0 else bq.collapse(bvh, width)
    off, ids = bq.fixedBoxQuery.findPrims(t, torch.from_numpy(boxes).cuda(), torch.from_numpy(q).cuda(), slabCap=cap)
    if width == 0:
        ooff, oids = oracle.box_query(n, pr, boxes, q)
    else:
        ws, wp = t.to_host()
        ooff, oids = oracle.wide_box_query(ws, width, wp, boxes, q)
    assert np.array_equal(off.cpu().numpy(), ooff)
    assert np.array_equal(ids.cpu().numpy(), oids)


def test_box_query_sets_match_brute_force(bq):
    boxes, q = _boxes("extents", 20000), _queries(500, seed=13)
    bvh = _build(bq, "morton", boxes, 0)
    off, ids = bq.fixedBoxQuery.findPrims(bvh, torch.from_numpy(boxes).cuda(), torch.from_numpy(q).cuda())
    off, ids = off.cpu().numpy(), ids.cpu().numpy()
    lo, hi = boxes[:, :3], boxes[:, 3:]
    for i in range(len(q)):
        want = np.nonzero(~((q[i, 3:] < lo).any(1) | (hi < q[i, :3]).any(1)))[0]
        assert np.array_equal(np.sort(ids[off[i]:off[i + 1]]), want), i


def test_box_query_edge_cases(bq):
    # no queries; one prim; an empty tree; capacity smaller than the results
    boxes = _boxes("points", 1000)
    bvh = _build(bq, "morton", boxes, 0)
    db = torch.from_numpy(boxes).cuda()
    off, ids = bq.fixedBoxQuery.findPrims(bvh, db, torch.empty((0, 6), device="cuda"))
    assert off.tolist() == [0] and ids.numel() == 0
    one = boxes[:1]
    b1 = _build(bq, "morton", one, 0)
    off, ids = bq.fixedBoxQuery.findPrims(b1, torch.from_numpy(one).cuda(),
                                          torch.from_numpy(np.float32([[-1, -1, -1, 2, 2, 2],
                                                                       [3, 3, 3, 4, 4, 4]])).cuda())
    assert off.tolist() == [0, 1, 1] and ids.tolist() == [0]
    e = _build(bq, "morton", np.zeros((0, 6), np.float32), 0)
    cnt = bq.fixedBoxQuery.count(e, torch.zeros((0, 6), device="cuda"), torch.from_numpy(_queries(10)).cuda())
    assert cnt.tolist() == [0] * 10
    q = torch.from_numpy(_queries(64)).cuda()
    counts = bq.fixedBoxQuery.count(bvh, db, q)
    offs = torch.zeros(64, dtype=torch.int32, device="cuda")
    offs[1:] = torch.cumsum(counts, 0)[:-1].to(torch.int32)
    total = int(counts.sum())
    cap = total - 1
    out = torch.full((total,), -7, dtype=torch.int32, device="cuda")
    rc = bq._lib.bq_box_query_f3(ctypes.byref(bvh.c), bq._ptr(db), bq._ptr(q), 64, bq._ptr(offs), cap,
                                 bq._ptr(out), ctypes.byref(bvh.allocator.c), bq._stream())
    assert rc == 1  # BQ_ERR_INVALID_ARGUMENT: results past the capacity
    assert int(out[cap]) == -7  # nothing written past it


def test_box_query_1m_prims(bq, oracle):
    """1M point boxes, 200K query boxes (half size 0.002-0.01)."""
    boxes = boxes_np(W.uniform_points(1 << 20))
    rng = np.random.default_rng(17)
    c = W.uniform_points(200000, W.SEED_QUERIES)
    h = rng.uniform(0.002, 0.01, size=(200000, 1)).astype(np.float32)
    q = np.concatenate([c - h, c + h], 1).astype(np.float32)
    bvh = _build(bq, "morton", boxes, 0)
    n, pr = bvh.to_host()
    off, ids = bq.fixedBoxQuery.findPrims(bvh, torch.from_numpy(boxes).cuda(), torch.from_numpy(q).cuda())
    ooff, oids = oracle.box_query(n, pr, boxes, q)
    assert np.array_equal(off.cpu().numpy(), ooff)
    assert np.array_equal(ids.cpu().numpy(), oids)
