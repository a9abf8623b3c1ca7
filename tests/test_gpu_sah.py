"""Binned SAH builder on the GPU (bq_build_sah_f3, and gpuBuilder with
BuildConfig::SAH) and its edge-length sibling (gpuBuilder with
BuildConfig::ELH).

Trees equal the oracle's restatement node for node (after BFS renumbering,
leaf prim order included) and the reference's own sahBuilder compiled for
sm_100a; queries over SAH trees equal the oracle's."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np, tri_boxes_np

pytestmark = pytest.mark.gpu


def _boxes(kind, n):
    rng = np.random.default_rng(21)
    if kind == "uniform":
        return boxes_np(W.uniform_points(n))
    if kind == "gmm":
        return boxes_np(W.gmm_points(n, offset=0.0))
    if kind == "dupes":
        return boxes_np(np.repeat(W.uniform_points(max(n // 16, 1)), 16, axis=0))
    if kind == "extents":
        c = W.uniform_points(n, 33)
        h = (rng.random((n, 3)) ** 3 * 0.05).astype(np.float32)
        return np.concatenate([c - h, c + h], 1).astype(np.float32)
    if kind == "mesh":
        verts, tris = W.icosphere(6)
        return tri_boxes_np(verts, tris)[:n]
    raise ValueError(kind)


def _heur_build(bq, heur, t, thr=0):
    """heur 0: cuda::sahBuilder; 1: gpuBuilder with BuildConfig::ELH."""
    if heur == 0:
        return bq.cuda.sahBuilder(t, bq.BuildConfig(makeLeafThreshold=thr))
    return bq.gpuBuilder(t, bq.BuildConfig(makeLeafThreshold=thr).enableELH())


def _same(oracle, a, b):
    ca, pa = oracle.canonicalize(*a)
    cb, pb = oracle.canonicalize(*b)
    ca, cb = ca.copy(), cb.copy()
    if len(ca) > 1:
        ca[1] = np.zeros(1, dtype=ca.dtype)
        cb[1] = np.zeros(1, dtype=cb.dtype)
    return len(ca) == len(cb) and ca.tobytes() == cb.tobytes() and np.array_equal(pa, pb)


@pytest.mark.parametrize("heur", [0, 1])
@pytest.mark.parametrize("kind", ["uniform", "gmm", "dupes", "extents", "mesh"])
@pytest.mark.parametrize("thr", [0, 1, 4, 8])
def test_sah_matches_oracle(bq, oracle, heur, kind, thr):
    b = _boxes(kind, 60000)
    bvh = _heur_build(bq, heur, torch.from_numpy(b).cuda(), thr)
    assert _same(oracle, bvh.to_host(), oracle.sah_build(b, thr, heur=heur))
    bvh.free()


@pytest.mark.parametrize("heur", [0, 1])
@pytest.mark.parametrize("kind", ["uniform", "gmm", "extents", "mesh"])
def test_sah_matches_reference_builder(bq, oracle, ref_gpu, heur, kind):
    b = _boxes(kind, 40000)
    from oracle.oracle import RefGPU
    for thr in (0, 4):
        bvh = _heur_build(bq, heur, torch.from_numpy(b).cuda(), thr)
        assert _same(oracle, bvh.to_host(), ref_gpu.build(RefGPU.ELH if heur else RefGPU.SAH, b, thr)), thr
        bvh.free()


def test_gpubuilder_sah_dispatch(bq, oracle):
    """gpuBuilder with BuildConfig::SAH (gpu_builder.h:41-53) builds the
    same tree as cuda::sahBuilder."""
    b = _boxes("mesh", 30000)
    t = torch.from_numpy(b).cuda()
    a = bq.gpuBuilder(t, bq.BuildConfig().enableSAH())
    c = bq.cuda.sahBuilder(t)
    assert _same(oracle, a.to_host(), c.to_host())
    with pytest.raises(bq.BQError):
        bq.gpuBuilder(t, bq.BuildConfig(buildMethod=7))


@pytest.mark.parametrize("heur", [0, 1])
def test_sah_large_levels(bq, oracle, heur):
    """327,680 triangle boxes (icosphere level 7): several global levels
    before the warp phase."""
    verts, tris = W.icosphere(7)
    b = tri_boxes_np(verts, tris)
    bvh = _heur_build(bq, heur, torch.from_numpy(b).cuda())
    assert _same(oracle, bvh.to_host(), oracle.sah_build(b, 0, heur=heur))
    bvh.free()


def test_sah_degenerate_and_edge_cases(bq, oracle):
    # 70000 identical points: the heuristic finds no split; more than
    # 65535 prims are split in halves, the halves become leaves
    same = np.repeat(np.float32([[0.25, 0.5, 0.75, 0.25, 0.5, 0.75]]), 70000, axis=0)
    bvh = bq.cuda.sahBuilder(torch.from_numpy(same).cuda())
    n, pr = bvh.to_host()
    assert _same(oracle, (n, pr), oracle.sah_build(same, 0))
    cnt = (n["admin"] >> np.uint64(48)).astype(np.int64)
    assert sorted(cnt[cnt > 0].tolist()) == [35000, 35000]
    # 5000 identical points: one leaf of 5000, as the reference builds it
    bvh = bq.cuda.sahBuilder(torch.from_numpy(same[:5000].copy()).cuda())
    n, pr = bvh.to_host()
    assert len(n) == 2 and int(n["admin"][0] >> np.uint64(48)) == 5000
    # empty input, one prim, empty boxes mixed in
    e = bq.cuda.sahBuilder(torch.zeros((0, 6), device="cuda"))
    assert e.numNodes == 0
    one = bq.cuda.sahBuilder(torch.from_numpy(_boxes("uniform", 1)).cuda())
    n, pr = one.to_host()
    assert int(n["admin"][0] >> np.uint64(48)) == 1 and pr.tolist() == [0]
    b = _boxes("extents", 20000)
    b[::7, 0], b[::7, 3] = 1.0, 0.0  # empty boxes (lower.x > upper.x) are left out
    bvh = bq.cuda.sahBuilder(torch.from_numpy(b).cuda())
    n, pr = bvh.to_host()
    assert _same(oracle, (n, pr), oracle.sah_build(b, 0))
    assert np.array_equal(pr[-len(b[::7]):], np.arange(0, 20000, 7))


def test_queries_on_sah_trees(bq, oracle):
    pts = W.uniform_points(50000)
    qs = W.uniform_points(20000, W.SEED_QUERIES, -0.1, 1.1)
    bvh = bq.cuda.sahBuilder(torch.from_numpy(boxes_np(pts)).cuda())
    n, pr = bvh.to_host()
    ids, d = bq.points.findClosest(bvh, torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda())
    oi, od, _, _ = oracle.closest_point(n, pr, pts, qs, fma_mode=1, tie_mode=0)
    assert np.array_equal(ids.cpu().numpy(), oi) and np.array_equal(d.cpu().numpy(), od)
