"""Rebinning Morton-30 builder (cuBQL::cuda::rebinRadixBuilder,
cuBQL/builder/cuda/rebinMortonBuilder.h:1161-1488) against the oracle's
restatement and against the reference's own GPU builder compiled for
sm_100a.  Trees are compared bit for bit after BFS renumbering (the
reference allocates nodes with atomics), leaf prim order included."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from helpers import boxes_np, same_tree
from oracle.oracle import NODE, check_tree

pytestmark = pytest.mark.gpu


def _points(dist, n):
    if dist in ("uniform", "invalid"):
        return W.uniform_points(n)
    if dist == "gmm":
        return W.gmm_points(n)
    if dist == "dupes":
        return np.repeat(W.uniform_points(max(n // 10, 1)), 10, axis=0)[:n]
    if dist == "line":
        p = np.zeros((n, 3), np.float32)
        p[:, 0] = W.uniform_points(n)[:, 0]
        return p
    if dist == "cluster":  # tight clusters inside a wide cloud: nested rebins
        k = n // 4
        wide = W.uniform_points(n - 3 * k, 21, -1000.0, 1000.0)
        t1 = W.uniform_points(k, 22, 0.0, 1e-3)
        t2 = W.uniform_points(k, 23, 5.0, 5.0 + 1e-6)
        t3 = np.repeat(W.uniform_points(max(k // 50, 1), 24, -3.0, -2.0), 50, axis=0)[:k]
        return np.concatenate([wide, t1, t2, t3]).astype(np.float32)
    raise ValueError(dist)


def _boxes(dist, n):
    b = boxes_np(_points(dist, n))
    if dist == "invalid":
        b[::5, 0] = 2.0
        b[::5, 3] = 1.0
    return b


def _build(bq, b, thr):
    return bq.cuda.rebinRadixBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))


@pytest.mark.parametrize("thr", [0, 1, 8, 40])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "invalid", "line", "cluster"])
def test_rebin_matches_oracle(bq, oracle, thr, dist):
    b = _boxes(dist, 30000)
    bvh = _build(bq, b, thr)
    gn, gp = bvh.to_host()
    valid = ~(b[:, 0] > b[:, 3])
    assert bvh.numPrims == valid.sum()
    on, op = oracle.rebin_build(b, thr)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    check_tree(gn, gp, b, max_leaf=max(thr, 32))
    bvh.free()


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 64, 100, 4097])
def test_rebin_small_sizes(bq, oracle, n):
    for dist in ("gmm", "dupes", "cluster"):
        b = _boxes(dist, n)
        for thr in (0, 3):
            bvh = _build(bq, b, thr)
            gn, gp = bvh.to_host()
            on, op = oracle.rebin_build(b, thr)
            ok, msg = same_tree(oracle, gn, gp, on, op)
            assert ok, f"{dist} thr {thr}: {msg}"


def test_rebin_unsplittable_runs(bq, oracle):
    """Runs whose centroid bounds are narrower than 1e-20 but not a point:
    up to 32 prims the reference makes them one leaf whatever the
    threshold; above that the library stops rebinning at depth 40 and splits
    by position (where the reference would restart forever)."""
    base = W.uniform_points(2000)
    small = np.zeros((20, 3), np.float32)
    small[:, 0] = np.arange(20, dtype=np.float32) * np.float32(1e-30)
    large = np.zeros((300, 3), np.float32)
    large[:, 0] = (np.arange(300) % 2).astype(np.float32) * np.float32(1e-30)
    for extra in (small, large):
        b = boxes_np(np.concatenate([base, extra]))
        for thr in (0, 4):
            bvh = _build(bq, b, thr)
            gn, gp = bvh.to_host()
            on, op = oracle.rebin_build(b, thr)
            ok, msg = same_tree(oracle, gn, gp, on, op)
            assert ok, msg


@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "cluster"])
def test_rebin_matches_reference_gpu_builder(bq, oracle, ref_gpu, dist):
    b = _boxes(dist, 100000)
    for thr in (0, 8):
        bvh = _build(bq, b, thr)
        gn, gp = bvh.to_host()
        rn, rp = ref_gpu.build(ref_gpu.REBIN, b, thr)
        ok, msg = same_tree(oracle, gn, gp, rn, rp)
        assert ok, f"thr {thr}: {msg}"


def test_rebin_golden_trees(bq, oracle):
    """The reference's rebin trees stored as fixtures (tests/golden)."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_rebin.npz")
    if not os.path.exists(path):
        pytest.skip("no rebin fixtures")
    g = np.load(path)
    for name in ("u", "g", "c"):
        b = boxes_np(g[f"{name}_points"])
        for thr in (0, 8):
            bvh = _build(bq, b, thr)
            gn, gp = bvh.to_host()
            cn, cp = oracle.canonicalize(gn, gp)
            assert np.array_equal(cp, g[f"{name}_rebin{thr}_prims"]), (name, thr)
            ref = g[f"{name}_rebin{thr}_nodes"].view(cn.dtype)
            cn = cn.copy()
            ref = ref.copy()
            cn[1] = np.zeros(1, dtype=NODE)
            ref[1] = np.zeros(1, dtype=NODE)
            assert cn.tobytes() == ref.tobytes(), (name, thr)


def test_rebin_full_size_2m(bq, oracle):
    b = _boxes("gmm", 2_000_000)
    bvh = _build(bq, b, 0)
    gn, gp = bvh.to_host()
    on, op = oracle.rebin_build(b, 0)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
