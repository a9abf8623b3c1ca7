"""Builders on the GPU against the oracle and the reference's own GPU
builders.  Morton trees must be identical node for node (after BFS
renumbering); spatial-median trees must satisfy the reference's structural
invariants and equal the oracle's canonical tree."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from oracle.oracle import check_tree
from tests.helpers import boxes_np, same_tree

pytestmark = pytest.mark.gpu


def _dist(dist, n):
    if dist == "uniform" or dist == "invalid":
        return W.uniform_points(n)
    if dist == "gmm":
        return W.gmm_points(n)
    if dist == "dupes":
        return np.repeat(W.uniform_points(max(n // 10, 1)), 10, axis=0)[:n]
    if dist == "line":  # all on one axis-aligned line: degenerate centroid boxes
        p = np.zeros((n, 3), np.float32)
        p[:, 0] = W.uniform_points(n)[:, 0]
        return p
    raise ValueError(dist)


def _boxes(dist, n):
    b = boxes_np(_dist(dist, n))
    if dist == "invalid":
        b[::5, 0] = 2.0
        b[::5, 3] = 1.0
    return b


@pytest.mark.parametrize("n", [1, 2, 3, 17, 1000, 4096, 65537])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "invalid", "line"])
def test_morton_matches_oracle(bq, oracle, n, dist):
    b = _boxes(dist, n)
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda())
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b)
    assert bvh.numNodes == len(on) and bvh.numPrims == len(op)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    bvh.free()


@pytest.mark.parametrize("thr", [2, 3, 8, 33])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes"])
def test_morton_leaf_threshold_matches_oracle(bq, oracle, thr, dist):
    b = _boxes(dist, 20000)
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b, thr)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    check_tree(gn, gp, b, max_leaf=thr)


@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_morton_matches_reference_gpu_builder(bq, oracle, ref_gpu, dist):
    b = _boxes(dist, 200000)
    for thr in (0, 8):
        bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
        gn, gp = bvh.to_host()
        rn, rp = ref_gpu.build(ref_gpu.RADIX, b, thr)
        ok, msg = same_tree(oracle, gn, gp, rn, rp)
        assert ok, f"thr {thr}: {msg}"


def test_morton_full_size_10m(bq, oracle):
    """The benchmark workload itself: 10M uniform points, leaf 1."""
    b = boxes_np(W.uniform_points(10_000_000))
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda())
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b)
    assert len(gn) == 20_000_000
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg


@pytest.mark.parametrize("dist", ["uniform", "gmm"])
def test_morton_4pass_matches_oracle(bq, oracle, dist):
    """Above 2^24 prims the top 32 key bits are sorted (4 passes) instead of
    24: 17M prims, uniform and the duplicate-heavy GMM (long runs)."""
    b = boxes_np(_dist(dist, 17_000_000))
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda())
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    bvh.free()


@pytest.mark.parametrize("seed", [0, 1])
def test_morton_runs_across_tiles(bq, oracle, seed):
    """Runs of equal top key bits of every length from 1 to 40 prims (an
    8-bit-per-axis cell each, some points duplicated), so that runs of
    every size begin, end and cross the run-ordering tiles (1024 sorted
    positions) at every offset."""
    rng = np.random.default_rng(100 + seed)
    cells = rng.choice(256 ** 3, 6000, replace=False)
    sizes = rng.integers(1, 41, len(cells))
    cxyz = np.stack([cells % 256, (cells // 256) % 256, cells // 65536], 1).astype(np.float64)
    pts = []
    for c, k in zip(cxyz, sizes):
        p = (c + 0.05 + 0.9 * rng.random((k, 3))) / 256.0
        if k > 2 and rng.random() < 0.3:
            p[1:k // 2 + 1] = p[0]  # identical points: equal full keys inside the run
        pts.append(p)
    p = np.concatenate(pts).astype(np.float32)
    p = np.concatenate([p, np.float32([[0, 0, 0], [1, 1, 1]])])  # bounds: the unit cube
    b = boxes_np(p[rng.permutation(len(p))])
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda())
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    bvh.free()


@pytest.mark.parametrize("builder", ["morton", "sm", "sah"])
def test_allocator_scratch_modes(bq, oracle, builder):
    """bq_allocator::scratchFromPool 0 (every temporary through the torch
    callbacks) and 1 (temporaries from the library's pool) give the same
    tree; the returned arrays always come from the callbacks."""
    b = torch.from_numpy(_boxes("gmm", 50000)).cuda()
    trees = []
    for mode in (0, 1):
        a = bq.TorchAllocator()
        a.c.scratchFromPool = mode
        if builder == "morton":
            t = bq.cuda.radixBuilder(b, allocator=a)
        elif builder == "sm":
            t = bq.gpuBuilder(b, bq.BuildConfig(makeLeafThreshold=4), allocator=a)
        else:
            t = bq.cuda.sahBuilder(b, allocator=a)
        assert t.c.nodes in a.live and t.c.primIDs in a.live
        trees.append(t.to_host())
        t.free()
    assert trees[0][0].tobytes() == trees[1][0].tobytes() and np.array_equal(trees[0][1], trees[1][1])


def test_morton_is_deterministic(bq):
    b = torch.from_numpy(_boxes("gmm", 300000)).cuda()
    a = bq.cuda.radixBuilder(b).to_host()
    c = bq.cuda.radixBuilder(b).to_host()
    assert a[0].tobytes() == c[0].tobytes() and np.array_equal(a[1], c[1])


def test_empty_and_all_invalid(bq):
    bvh = bq.cuda.radixBuilder(torch.zeros((0, 6), dtype=torch.float32, device="cuda"))
    assert bvh.numNodes == 0 and bvh.numPrims == 0
    b = _boxes("uniform", 100)
    b[:, 0] = 2.0
    b[:, 3] = 1.0
    bvh = bq.cuda.radixBuilder(torch.from_numpy(b).cuda())
    assert bvh.numNodes == 0 and bvh.numPrims == 0
    bvh = bq.gpuBuilder(torch.from_numpy(b).cuda())
    assert bvh.numNodes == 0


@pytest.mark.parametrize("thr", [0, 1, 8, 40, 5000])
@pytest.mark.parametrize("dist", ["uniform", "gmm", "dupes", "invalid", "line"])
def test_spatial_median_invariants_and_oracle(bq, oracle, thr, dist):
    b = _boxes(dist, 30000)
    bvh = bq.gpuBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
    gn, gp = bvh.to_host()
    valid = ~(b[:, 0] > b[:, 3])
    assert bvh.numPrims == len(b)
    check_tree(gn, gp[: valid.sum()], b, max_leaf=max(thr, 1))
    assert np.array_equal(np.sort(gp[valid.sum():]), np.nonzero(~valid)[0])
    on, op = oracle.sm_build(b, thr)
    ok, msg = same_tree(oracle, gn, gp[: valid.sum()], on, op[: valid.sum()])
    assert ok, msg


@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 64, 4095, 4096, 4097, 8193])
def test_spatial_median_small_and_boundary_sizes(bq, oracle, n):
    """Sizes around the one-warp register subtree (32) and the one-warp
    subtree limit (4096)."""
    b = _boxes("gmm", n)
    for thr in (0, 3):
        bvh = bq.gpuBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
        gn, gp = bvh.to_host()
        check_tree(gn, gp, b, max_leaf=max(thr, 1))
        on, op = oracle.sm_build(b, thr)
        ok, msg = same_tree(oracle, gn, gp, on, op)
        assert ok, f"thr {thr}: {msg}"


def test_spatial_median_matches_reference_gpu_builder(bq, oracle, ref_gpu):
    """Uniform input: the reference's tree is determined up to the order of
    exactly identical prims (the seeded generator repeats a point whenever
    two indices get the same TEA seed, ~5 pairs per 200K points, and the
    reference deals identical prims to the two sides in atomic order)."""
    b = _boxes("uniform", 200000)
    for thr in (0, 8):
        bvh = bq.gpuBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
        gn, gp = bvh.to_host()
        rn, rp = ref_gpu.build(ref_gpu.SPATIAL_MEDIAN, b, thr)
        ok, msg = same_tree(oracle, gn, gp, rn, rp, boxes=b)
        assert ok, f"thr {thr}: {msg}"


def test_spatial_median_reference_invariants_on_degenerate_input(bq, oracle, ref_gpu):
    """Where the reference itself is racy (dim == -1 nodes) both trees pass
    the invariants and have the same number of nodes."""
    b = _boxes("dupes", 50000)
    bvh = bq.gpuBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=8))
    gn, gp = bvh.to_host()
    rn, rp = ref_gpu.build(ref_gpu.SPATIAL_MEDIAN, b, 8)
    check_tree(gn, gp, b, max_leaf=8)
    check_tree(rn, rp, b, max_leaf=8)
    assert len(gn) == len(rn)


def test_spatial_median_full_size_10m(bq, oracle):
    b = boxes_np(W.uniform_points(10_000_000))
    bvh = bq.gpuBuilder(torch.from_numpy(b).cuda(), bq.BuildConfig(makeLeafThreshold=8))
    gn, gp = bvh.to_host()
    on, op = oracle.sm_build(b, 8)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg


@pytest.mark.parametrize("builder", ["morton", "sm"])
def test_refit_after_moving_prims(bq, oracle, builder):
    pts = W.uniform_points(50000)
    b = torch.from_numpy(boxes_np(pts)).cuda()
    bvh = bq.cuda.radixBuilder(b, bq.BuildConfig(makeLeafThreshold=4)) if builder == "morton" else \
        bq.gpuBuilder(b, bq.BuildConfig(makeLeafThreshold=4))
    moved = boxes_np(pts + np.float32(0.01) * W.uniform_points(50000, 99, -1, 1))
    bq.refit(bvh, torch.from_numpy(moved).cuda())
    gn, gp = bvh.to_host()
    check_tree(gn, gp, moved, max_leaf=4)


def _tree_properties_on_gpu(bq, bvh, boxes_t):
    """Size-independent invariants checked on the device: primIDs are a
    permutation, every node but 0 and 1 is the child of exactly one inner
    node, leaves cover every sorted position once, and every inner node's
    box is exactly the union of its children's (leaf boxes exactly the
    prims' boxes)."""
    n = boxes_t.shape[0]
    nodes = bvh.nodes_tensor()  # (numNodes, 8) float32: lower, upper, admin words
    admin = nodes[:, 6:8].contiguous().view(torch.int64).view(-1)
    count = (admin >> 48) & 0xFFFF
    off = admin & 0xFFFFFFFFFFFF
    nn = nodes.shape[0]
    prims = bvh.primids_tensor().long()
    assert torch.equal(torch.sort(prims).values, torch.arange(n, device="cuda"))
    inner = count == 0
    inner[1] = False
    io = off[inner]
    assert bool(((io >= 2) & (io + 1 < nn) & (io % 2 == 0)).all())
    refs = torch.zeros(nn, dtype=torch.int32, device="cuda")
    one = torch.ones_like(io, dtype=torch.int32)
    refs.index_add_(0, io, one)
    refs.index_add_(0, io + 1, one)
    assert bool((refs[2:] == 1).all()) and int(refs[0]) == 0
    leaf = count > 0
    lo, lc = off[leaf], count[leaf]
    cover = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    cover.index_add_(0, lo, torch.ones_like(lo, dtype=torch.int32))
    cover.index_add_(0, lo + lc, -torch.ones_like(lo, dtype=torch.int32))
    assert bool((torch.cumsum(cover, 0)[:n] == 1).all())
    box = nodes[:, :6]
    step = 1 << 24
    idx_inner = torch.nonzero(inner).view(-1)
    for s in range(0, idx_inner.numel(), step):
        p = idx_inner[s:s + step]
        c0, c1 = box[off[p]], box[off[p] + 1]
        u = torch.cat([torch.minimum(c0[:, :3], c1[:, :3]), torch.maximum(c0[:, 3:], c1[:, 3:])], 1)
        assert torch.equal(u, box[p])
    idx_leaf = torch.nonzero(leaf & (count == 1)).view(-1)
    for s in range(0, idx_leaf.numel(), step):
        p = idx_leaf[s:s + step]
        assert torch.equal(box[p], boxes_t[prims[off[p]]])
    root = box[0]
    assert torch.equal(root[:3], boxes_t[:, :3].min(0).values) and torch.equal(root[3:], boxes_t[:, 3:].max(0).values)


@pytest.mark.parametrize("builder", ["morton", "sm", "sah"])
def test_builders_100m_properties(bq, builder):
    """Ten times the benchmark size (100M point boxes, 2.4 GB; 200M nodes),
    leaf 1: the trees' structural invariants, checked on the device."""
    n = 100_000_000
    free, _ = torch.cuda.mem_get_info()
    if free < 40 << 30:
        pytest.skip("needs 40 GB of free device memory")
    g = torch.Generator(device="cuda")
    g.manual_seed(12345)
    pts = torch.rand((n, 3), generator=g, device="cuda", dtype=torch.float32)
    boxes_t = torch.cat([pts, pts], 1).contiguous()
    del pts
    build = {"morton": bq.cuda.radixBuilder, "sm": bq.gpuBuilder, "sah": bq.cuda.sahBuilder}[builder]
    bvh = build(boxes_t)
    assert bvh.numNodes == 2 * n and bvh.numPrims == n
    _tree_properties_on_gpu(bq, bvh, boxes_t)
    bvh.free()
