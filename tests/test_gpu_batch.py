"""Batched (segmented) build and kNN: every cloud's tree equals the single
build of that cloud (and the oracle's), batched kNN equals per-cloud kNN
bit for bit, the whole batch replays inside a CUDA graph, and the
autotuner's choice does not change the answers."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np, same_tree

pytestmark = pytest.mark.gpu


def _batch(num=40, lo=50, hi=20000, nq=700, seed=5):
    pts, off, qs, qoff = W.cloud_batch(num, lo, hi, nq, seed)
    return pts, off, qs, qoff


@pytest.mark.parametrize("thr", [0, 1, 3, 8])
def test_batched_trees_equal_single_builds(bq, oracle, thr):
    pts, off, qs, qoff = _batch()
    b = boxes_np(pts)
    batch = bq.Batch(torch.from_numpy(b).cuda(), torch.from_numpy(off), bq.BuildConfig(makeLeafThreshold=thr))
    for s in range(len(off) - 1):
        cb = b[off[s]:off[s + 1]]
        gn, gp = batch.tree_host(s)
        on, op = oracle.radix_build(cb, thr)
        assert len(gn) == len(on), f"cloud {s}"
        ok, msg = same_tree(oracle, gn, gp, on, op)
        assert ok, f"cloud {s}: {msg}"
        if s % 7 == 0:
            single = bq.cuda.radixBuilder(torch.from_numpy(cb).cuda(), bq.BuildConfig(makeLeafThreshold=thr))
            sn, sp = single.to_host()
            assert gn.tobytes() == sn.tobytes() and np.array_equal(gp, sp), f"cloud {s} vs single build"


@pytest.mark.parametrize("tie", [0, 1])
@pytest.mark.parametrize("k", [1, 16, 40])
def test_batched_knn_equals_per_cloud(bq, oracle, tie, k):
    pts, off, qs, qoff = _batch()
    b = boxes_np(pts)
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    batch = bq.Batch(torch.from_numpy(b).cuda(), torch.from_numpy(off))
    ids, d, nf = bq.batched_knn(batch, tp, torch.from_numpy(off), tq, torch.from_numpy(qoff), k,
                                qcfg=bq.query_config(tieMode=tie, queriesPerWarp=64))
    ids, d, nf = ids.cpu().numpy(), d.cpu().numpy(), nf.cpu().numpy()
    for s in range(len(off) - 1):
        cp = pts[off[s]:off[s + 1]]
        cq = qs[qoff[s]:qoff[s + 1]]
        gn, gp = batch.tree_host(s)
        oi, od, onf, _ = oracle.knn(gn, gp, cp, cq, k, tie_mode=tie)
        sl = slice(qoff[s], qoff[s + 1])
        assert np.array_equal(ids[sl], oi) and np.array_equal(d[sl], od) and np.array_equal(nf[sl], onf), f"cloud {s}"


def test_batch_in_cuda_graph(bq):
    pts, off, qs, qoff = _batch(num=30)
    b = torch.from_numpy(boxes_np(pts)).cuda()
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    toff, tqoff = torch.from_numpy(off).cuda().int(), torch.from_numpy(qoff).cuda().int()
    ref = bq.batched_knn(bq.Batch(b, toff), tp, toff, tq, tqoff, 16)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):  # warm-up outside capture (first use of the scratch pool)
        bq.batched_knn(bq.Batch(b, toff, stream_alloc_null=True), tp, toff, tq, tqoff, 16, stream_alloc_null=True)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch = bq.Batch(b, toff, stream_alloc_null=True)
        out = bq.batched_knn(batch, tp, toff, tq, tqoff, 16, stream_alloc_null=True)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out[0], ref[0]) and torch.equal(out[1], ref[1])
    del g


def test_autotuner_choice_keeps_answers(bq):
    pts, off, qs, qoff = _batch(num=20)
    b = torch.from_numpy(boxes_np(pts)).cuda()
    tp, tq = torch.from_numpy(pts).cuda(), torch.from_numpy(qs).cuda()
    toff, tqoff = torch.from_numpy(off), torch.from_numpy(qoff)
    best = bq.autotune_batched_knn(b, tp, toff, tq, tqoff, 16)
    assert best["makeLeafThreshold"] in (1, 2, 4, 8) and best["queryMs"] > 0
    ref = bq.batched_knn(bq.Batch(b, toff), tp, toff, tq, tqoff, 16)
    tuned_batch = bq.Batch(b, toff, bq.BuildConfig(makeLeafThreshold=best["makeLeafThreshold"]))
    q = bq.query_config(stackDepth=best["stackDepth"], blockSize=best["blockSize"],
                        queriesPerWarp=best["queriesPerWarp"])
    out = bq.batched_knn(tuned_batch, tp, toff, tq, tqoff, 16, qcfg=q)
    assert torch.equal(out[0], ref[0]) and torch.equal(out[1], ref[1])
