"""Closest-point and kNN queries on the GPU.

Bit-exact against (a) the oracle's restatement of the traversal with the
same tie rule and (b) the reference's own query kernels compiled for
sm_100a, on the same tree; FP32 squared distances within 1e-6 relative of
an FP64 brute force."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np, fp64_closest

pytestmark = pytest.mark.gpu


def _data(dist, n, nq):
    if dist == "uniform":
        return W.uniform_points(n), W.uniform_points(nq, W.SEED_QUERIES, -0.1, 1.1)
    if dist == "gmm":
        return W.gmm_points(n), W.gmm_points(nq, seed=W.SEED_GMM + 100)
    if dist == "dupes":
        p = np.repeat(W.uniform_points(n // 8), 8, axis=0)
        return p, W.uniform_points(nq, W.SEED_QUERIES)
    raise ValueError(dist)


def _tree(bq, kind, pts, thr=0):
    b = torch.from_numpy(boxes_np(pts)).cuda()
    if kind == "morton":
        return bq.cuda.radixBuilder(b, bq.BuildConfig(makeLeafThreshold=thr))
    return bq.gpuBuilder(b, bq.BuildConfig(makeLeafThreshold=thr or 8))


@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("kind", ["morton", "sm"])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_closest_point_matches_oracle(bq, oracle, tie, kind, dist):
    pts, qs = _data(dist, 40000, 20000)
    bvh = _tree(bq, kind, pts)
    n, pr = bvh.to_host()
    for reorder in (0, 1):
        ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(),
                                       qcfg=bq.query_config(tieMode=tie, reorder=reorder))
        oi, od, ovf, _ = oracle.closest_point(n, pr, pts, qs, fma_mode=1, tie_mode=tie)
        assert np.array_equal(ids.cpu().numpy(), oi), f"reorder {reorder}"
        assert np.array_equal(d.cpu().numpy(), od)


@pytest.mark.parametrize("k", [1, 4, 5, 16, 32, 64])
@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_knn_matches_oracle(bq, oracle, k, tie, dist):
    pts, qs = _data(dist, 30000, 5000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    ids, d, nf = bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), k,
                                   qcfg=bq.query_config(tieMode=tie))
    oi, od, onf, _ = oracle.knn(n, pr, pts, qs, k, fma_mode=1, tie_mode=tie)
    assert np.array_equal(ids.cpu().numpy(), oi)
    assert np.array_equal(d.cpu().numpy(), od)
    assert np.array_equal(nf.cpu().numpy(), onf)


@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_matches_reference_query_kernels(bq, oracle, ref_gpu, dist):
    """Reference tie rules, same tree: our results equal the reference's
    findClosest / findKNN kernels bit for bit, ties included."""
    pts, qs = _data(dist, 100000, 30000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    _, _, ovf, _ = oracle.closest_point(n, pr, pts, qs, tie_mode=1, stack=64)
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(),
                                   qcfg=bq.query_config(tieMode=1))
    ri, rd = ref_gpu.closest_point(n, pr, pts, qs)
    ok = ~ovf  # the reference silently returns early on a 64-entry stack overflow
    assert np.array_equal(ids.cpu().numpy()[ok], ri[ok]) and np.array_equal(d.cpu().numpy()[ok], rd[ok])
    ki, kd, kn = bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 16,
                                   qcfg=bq.query_config(tieMode=1))
    rki, rkd, rkn = ref_gpu.knn(n, pr, pts, qs, 16)
    _, _, _, kovf = oracle.knn(n, pr, pts, qs, 16, tie_mode=1, stack=64)
    ok = ~kovf
    assert np.array_equal(ki.cpu().numpy()[ok], rki[ok]) and np.array_equal(kd.cpu().numpy()[ok], rkd[ok])
    assert np.array_equal(kn.cpu().numpy()[ok], rkn[ok])


def test_lowest_id_ties_against_reference(bq, oracle, ref_gpu):
    """Default tie rule: same distances as the reference kernel, and our id is
    the lowest among all points at that FP32 distance."""
    pts, qs = _data("dupes", 80000, 20000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda())
    ids, d = ids.cpu().numpy(), d.cpu().numpy()
    ri, rd = ref_gpu.closest_point(n, pr, pts, qs)
    assert np.array_equal(d, rd)
    # every point at exactly that distance has an id >= ours
    same = pts[ids]
    for j in range(0, len(qs), 997):
        dj = oracle.sqr_pp(pts, np.repeat(qs[j:j + 1], len(pts), 0), 1)
        assert ids[j] == np.nonzero(dj == d[j])[0].min()
    assert same.shape == (len(qs), 3)


@pytest.mark.parametrize("kind", ["morton", "sm"])
def test_closest_within_fp64_brute_force(bq, kind):
    pts, qs = _data("uniform", 50000, 4000)
    bvh = _tree(bq, kind, pts)
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda())
    d64, i64 = fp64_closest(pts, qs)
    d = d.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(d - d64) <= 1e-6 * d64), "FP32 squared distance within 1e-6 relative of FP64"


def test_knn_within_fp64_brute_force(bq):
    pts, qs = _data("uniform", 20000, 1000)
    bvh = _tree(bq, "morton", pts)
    _, d, nf = bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 16)
    p = pts.astype(np.float64)
    ref = np.sort(((qs[:, None, :].astype(np.float64) - p[None]) ** 2).sum(-1), axis=1)[:, :16]
    assert np.all(nf.cpu().numpy() == 16)
    assert np.all(np.abs(d.cpu().numpy() - ref) <= 1e-6 * ref)


def test_max_radius_and_empty_tree(bq, oracle):
    pts, qs = _data("uniform", 10000, 5000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    r2 = 0.0004
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), maxSqrDist=r2)
    oi, od, _, _ = oracle.closest_point(n, pr, pts, qs, maxSqr=r2)
    assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)
    assert (oi == -1).any() and (oi >= 0).any()
    ki, kd, kn = bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 8, maxSqrDist=r2)
    oki, okd, okn, _ = oracle.knn(n, pr, pts, qs, 8, maxSqr=r2)
    assert np.array_equal(ki.cpu().numpy(), oki) and np.array_equal(kn.cpu().numpy(), okn)
    empty = bq.cuda.radixBuilder(torch.zeros((0, 6), dtype=torch.float32, device="cuda"))
    ids, d = bq.points.findClosest(empty, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda())
    assert (ids.cpu().numpy() == -1).all() and np.isinf(d.cpu().numpy()).all()


@pytest.mark.parametrize("stack", [32, 64, 128])
def test_stack_overflow_falls_back_to_deep_stack(bq, oracle, stack):
    """Clustered duplicates make deep trees; queries that overflow the fast
    stack are re-run with the deep one and still match the oracle."""
    pts, qs = _data("gmm", 200000, 20000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(),
                                   qcfg=bq.query_config(stackDepth=stack))
    oi, od, ovf, _ = oracle.closest_point(n, pr, pts, qs, stack=stack)
    assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)


def test_full_size_10m_queries(bq, oracle):
    """10M points, 10M queries: bit-exact against the oracle on a seeded
    sample of queries, plus whole-batch properties (sorted kNN rows)."""
    pts = W.uniform_points(10_000_000)
    qs = W.uniform_points(10_000_000, W.SEED_QUERIES)
    bvh = _tree(bq, "morton", pts)
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    ids, d = bq.points.findClosest(bvh, tp, tq)
    ki, kd, kn = bq.points.findKNN(bvh, tp, tq, 16)
    n, pr = bvh.to_host()
    sel = np.arange(0, 10_000_000, 4999)
    oi, od, _, _ = oracle.closest_point(n, pr, pts, qs[sel])
    assert np.array_equal(ids.cpu().numpy()[sel], oi) and np.array_equal(d.cpu().numpy()[sel], od)
    oki, okd, _, _ = oracle.knn(n, pr, pts, qs[sel], 16)
    assert np.array_equal(ki.cpu().numpy()[sel], oki) and np.array_equal(kd.cpu().numpy()[sel], okd)
    kdh = kd.cpu().numpy()
    assert np.all(np.diff(kdh, axis=1) >= 0) and np.all(kn.cpu().numpy() == 16)
    assert np.array_equal(kdh[:, 0], d.cpu().numpy())


@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_closest_exclude_variants_match_oracle(bq, oracle, tie, dist):
    """findClosest_exludeID / findClosest_exludeSelf (findClosest.h:278-334)
    with the data points as queries ("nearest other point"), bit for bit
    against the oracle with the same tie rule; on "dupes" exclude-self
    skips every copy of the point and exclude-id only the query's own one."""
    pts, _ = _data(dist, 40000, 1)
    qs = pts[::4].copy()
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    qc = bq.query_config(tieMode=tie)
    exid = np.arange(0, len(pts), 4, dtype=np.int32)
    exid[::9] = -1
    ids, d = bq.points.findClosest_exludeID(bvh, tp, tq, torch.from_numpy(exid), qcfg=qc)
    oi, od = oracle.closest_point_exclude(n, pr, pts, qs, exclude_ids=exid, fma_mode=1, tie_mode=tie)
    assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)
    ids, d = bq.points.findClosest_exludeSelf(bvh, tp, tq, qcfg=qc)
    oi, od = oracle.closest_point_exclude(n, pr, pts, qs, exclude_self=True, fma_mode=1, tie_mode=tie)
    assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)
    assert (d.cpu().numpy() > 0).all()  # no query finds a copy of itself


@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_closest_exclude_variants_match_reference_kernels(bq, oracle, ref_gpu, dist):
    """The reference's own findClosest_exludeID / _exludeSelf kernels,
    compiled for sm_100a, on our tree: identical ids and distances under the
    reference tie rule."""
    pts, _ = _data(dist, 40000, 1)
    qs = pts[1::5].copy()
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    qc = bq.query_config(tieMode=1)
    exid = np.arange(1, len(pts), 5, dtype=np.int32)
    ids, d = bq.points.findClosest_exludeID(bvh, tp, tq, torch.from_numpy(exid), qcfg=qc)
    ri, rd = ref_gpu.closest_point_exclude(n, pr, pts, qs, exclude_ids=exid)
    assert np.array_equal(ids.cpu().numpy(), ri) and np.array_equal(d.cpu().numpy(), rd)
    ids, d = bq.points.findClosest_exludeSelf(bvh, tp, tq, qcfg=qc)
    ri, rd = ref_gpu.closest_point_exclude(n, pr, pts, qs)
    assert np.array_equal(ids.cpu().numpy(), ri) and np.array_equal(d.cpu().numpy(), rd)


@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_visit_counts_match_oracle_traversal(bq, oracle, tie, dist):
    """The measurement pass behind the query rooflines counts exactly the
    node pairs the oracle's traversal expands (it counts 2 per expansion)."""
    pts, qs = _data(dist, 50000, 8000)
    bvh = _tree(bq, "morton", pts)
    n, pr = bvh.to_host()
    c = bq.points.visitCounts(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 0,
                              qcfg=bq.query_config(tieMode=tie))
    _, _, ovf, vis = oracle.closest_point(n, pr, pts, qs, tie_mode=tie, stack=128)
    assert not ovf.any()
    assert c["inner_nodes"] == int(vis.astype(np.int64).sum()) // 2
    assert c["admin_loads"] >= len(qs) and c["prims"] >= len(qs)
    k16 = bq.points.visitCounts(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 16,
                                qcfg=bq.query_config(tieMode=tie))
    assert k16["inner_nodes"] > c["inner_nodes"] and k16["prims"] >= 16 * len(qs)


@pytest.mark.parametrize("lanes,k", [(4, 4), (8, 5), (16, 16), (32, 16), (32, 32)])
@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_knn_lane_groups_match_oracle(bq, oracle, lanes, k, tie, dist):
    """kNN with a group of lanes per query (the top-k list spread over the
    group, one candidate per lane, merged by warp shuffles) gives exactly the
    per-thread answers, on leaf-1 and leaf-8 trees."""
    pts, qs = _data(dist, 30000, 5000)
    for thr in (0, 8):
        bvh = _tree(bq, "morton", pts, thr)
        n, pr = bvh.to_host()
        ids, d, nf = bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), k,
                                       qcfg=bq.query_config(tieMode=tie, lanesPerQuery=lanes))
        oi, od, onf, _ = oracle.knn(n, pr, pts, qs, k, fma_mode=1, tie_mode=tie)
        assert np.array_equal(ids.cpu().numpy(), oi), f"leaf {thr}"
        assert np.array_equal(d.cpu().numpy(), od)
        assert np.array_equal(nf.cpu().numpy(), onf)


def test_knn_lane_groups_reject_k_above_group(bq):
    pts, qs = _data("uniform", 1000, 100)
    bvh = _tree(bq, "morton", pts)
    with pytest.raises(bq.BQError):
        bq.points.findKNN(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda(), 16,
                          qcfg=bq.query_config(lanesPerQuery=8))
