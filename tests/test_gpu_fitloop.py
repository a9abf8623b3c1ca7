"""Batched meshes: batched refit + closest triangle + adjoint, the step of
a differentiable fitting loop.  Every step's forward on the refitted trees
must equal the forward on trees rebuilt from scratch (default tie rule:
the answer does not depend on the tree), and the batched forward must equal
per-mesh single queries."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_batched_tri_matches_single_meshes(bq, oracle):
    verts, tris, toff, qs, qoff = W.mesh_batch(num=8, lo=200, hi=3000, queries_per_mesh=2000)
    tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    tq = torch.from_numpy(qs).cuda()
    boxes = bq.triangles.boxes(tt, tv)
    batch = bq.Batch(boxes, torch.from_numpy(toff))
    ids, d, P = bq.batched_tri_closest(batch, tt, tv, tq, torch.from_numpy(qoff))
    ids, d = ids.cpu().numpy(), d.cpu().numpy()
    for m in range(len(toff) - 1):
        mt = tt[toff[m]:toff[m + 1]]
        single = bq.cuda.radixBuilder(bq.triangles.boxes(mt, tv))
        si, sd, _ = bq.triangles.findClosest(single, mt, tv, tq[qoff[m]:qoff[m + 1]])
        sl = slice(qoff[m], qoff[m + 1])
        assert np.array_equal(d[sl], sd.cpu().numpy()), f"mesh {m}"
        assert np.array_equal(ids[sl], si.cpu().numpy() + toff[m]), f"mesh {m}"


def test_fit_loop_refit_equals_rebuild(bq, oracle):
    verts, tris, toff, qs, qoff = W.mesh_batch(num=12, lo=300, hi=5000, queries_per_mesh=3000)
    tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    tq = torch.from_numpy(qs).cuda()
    toff_t, qoff_t = torch.from_numpy(toff), torch.from_numpy(qoff)
    batch = bq.Batch(bq.triangles.boxes(tt, tv), toff_t)
    g = torch.full((len(qs),), 1.0 / len(qs), device="cuda")
    losses = []
    for step in range(6):
        boxes = bq.triangles.boxes(tt, tv)
        if step:
            bq.batched_refit(batch, boxes)
        ids, d, _ = bq.batched_tri_closest(batch, tt, tv, tq, qoff_t)
        fresh = bq.Batch(boxes, toff_t)
        fi, fd, _ = bq.batched_tri_closest(fresh, tt, tv, tq, qoff_t)
        assert torch.equal(ids, fi) and torch.equal(d, fd), f"step {step}: refit forward != rebuilt forward"
        losses.append(float(d.double().mean()))
        gq, gv = bq.triangles.distanceBackward(tt, tv, tq, ids, g)
        tv = tv - 0.5 * gv  # gradient step on the vertices
    assert losses[-1] < losses[0]
