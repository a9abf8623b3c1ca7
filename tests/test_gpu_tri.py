"""Point-to-triangle distance: forward against the reference kernel and an
FP64 brute force; adjoint against the FP64 analytic gradient and FP64
central finite differences (tolerance 1e-5 relative, norm-wise)."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import tri_boxes_np

pytestmark = pytest.mark.gpu


def _mesh(level=3, nq=20000, seed=W.SEED_QUERIES):
    verts, tris = W.icosphere(level)
    qs = W.uniform_points(nq, seed, -1.5, 1.5)
    return verts, tris, qs


def _bvh(bq, verts, tris):
    tv, tt = torch.from_numpy(verts).cuda(), torch.from_numpy(tris).cuda()
    boxes = bq.triangles.boxes(tt, tv)
    assert np.array_equal(boxes.cpu().numpy(), tri_boxes_np(verts, tris))
    return bq.cuda.radixBuilder(boxes), tv, tt


def test_forward_matches_reference_kernel(bq, oracle, ref_gpu):
    verts, tris, qs = _mesh(4)
    bvh, tv, tt = _bvh(bq, verts, tris)
    n, pr = bvh.to_host()
    ids, d, P = bq.triangles.findClosest(bvh, tt, tv, torch.from_numpy(qs).cuda(), qcfg=bq.query_config(tieMode=1))
    ri, rd, rP = ref_gpu.tri_closest(n, pr, tris, verts, qs)
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(d.cpu().numpy(), rd)
    assert np.array_equal(P.cpu().numpy(), rP)


def test_forward_within_fp64(bq, oracle):
    verts, tris, qs = _mesh(3, 3000)
    bvh, tv, tt = _bvh(bq, verts, tris)
    ids, d, P = bq.triangles.findClosest(bvh, tt, tv, torch.from_numpy(qs).cuda())
    d64, i64 = oracle.tri_brute_f64(tris, verts, qs)
    d = d.cpu().numpy().astype(np.float64)
    # FP32 evaluation of a projection: |d - d64| <= 1e-6 d64 + 4 ulp(|q|^2)-scale absolute slack
    assert np.all(np.abs(d - d64) <= 1e-6 * d64 + 1e-6), np.abs(d - d64).max()


def test_forward_lowest_id_rule(bq, oracle):
    """Default rule: never farther than the reference rule (whose node culling
    can drop a triangle by one ulp of box-versus-triangle rounding), equal
    distances almost everywhere, and the lowest id among equal distances."""
    verts, tris, qs = _mesh(3, 5000)
    bvh, tv, tt = _bvh(bq, verts, tris)
    ids0, d0, _ = bq.triangles.findClosest(bvh, tt, tv, torch.from_numpy(qs).cuda())
    ids1, d1, _ = bq.triangles.findClosest(bvh, tt, tv, torch.from_numpy(qs).cuda(), qcfg=bq.query_config(tieMode=1))
    d0, d1 = d0.cpu().numpy(), d1.cpu().numpy()
    i0, i1 = ids0.cpu().numpy(), ids1.cpu().numpy()
    assert np.all(d0 <= d1)
    assert np.mean(d0 == d1) > 0.99
    eq = d0 == d1
    assert np.all(i0[eq] <= i1[eq])
    d64, _ = oracle.tri_brute_f64(tris, verts, qs)
    assert np.all(np.abs(d0 - d64) <= 1e-6 * d64 + 1e-6)


def test_adjoint_matches_fp64_analytic(bq, oracle):
    verts, tris, qs = _mesh(4, 50000)
    bvh, tv, tt = _bvh(bq, verts, tris)
    tq = torch.from_numpy(qs).cuda()
    ids, d, P = bq.triangles.findClosest(bvh, tt, tv, tq)
    g = torch.from_numpy(W.uniform_points(len(qs), 21, 0.5, 1.5)[:, 0].copy()).cuda()
    gq, gv = bq.triangles.distanceBackward(tt, tv, tq, ids, g)
    rq, rv = oracle.tri_grad_f64(tris, verts, qs, ids.cpu().numpy(), g.cpu().numpy())
    gq, gv = gq.cpu().numpy().astype(np.float64), gv.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(gq - rq) <= 1e-5 * np.linalg.norm(rq)
    assert np.linalg.norm(gv - rv) <= 1e-5 * np.linalg.norm(rv)


def test_adjoint_matches_finite_differences(bq, oracle):
    """Central differences of the FP64 distance to the chosen triangle, for
    query points and for a sample of vertices."""
    verts, tris, qs = _mesh(2, 400)
    bvh, tv, tt = _bvh(bq, verts, tris)
    tq = torch.from_numpy(qs).cuda()
    ids, d, _ = bq.triangles.findClosest(bvh, tt, tv, tq)
    ones = torch.ones(len(qs), dtype=torch.float32, device="cuda")
    gq, gv = bq.triangles.distanceBackward(tt, tv, tq, ids, ones)
    ids = ids.cpu().numpy()
    gq = gq.cpu().numpy().astype(np.float64)
    V = verts.astype(np.float64)
    h = 1e-6

    def dist(q, vv, t):
        return oracle.tri_cp_f64(vv[tris[t, 0]], vv[tris[t, 1]], vv[tris[t, 2]], q)[0]

    fq = np.zeros_like(gq)
    for i in range(len(qs)):
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            q = qs[i].astype(np.float64)
            fq[i, a] = (dist(q + e, V, ids[i]) - dist(q - e, V, ids[i])) / (2 * h)
    assert np.linalg.norm(gq - fq) <= 1e-5 * np.linalg.norm(fq)
    gvh = gv.cpu().numpy().astype(np.float64)
    for vi in range(0, len(verts), 7):
        users = np.nonzero((tris[ids] == vi).any(1))[0]
        for a in range(3):
            Vp, Vm = V.copy(), V.copy()
            Vp[vi, a] += h
            Vm[vi, a] -= h
            fd = sum((dist(qs[i].astype(np.float64), Vp, ids[i]) - dist(qs[i].astype(np.float64), Vm, ids[i]))
                     / (2 * h) for i in users)
            assert abs(gvh[vi, a] - fd) <= 1e-5 * max(1.0, abs(fd)) + 1e-6


def test_adjoint_is_bitwise_reproducible(bq):
    verts, tris, qs = _mesh(3, 100000)
    bvh, tv, tt = _bvh(bq, verts, tris)
    tq = torch.from_numpy(qs).cuda()
    ids, d, _ = bq.triangles.findClosest(bvh, tt, tv, tq)
    g = torch.ones(len(qs), dtype=torch.float32, device="cuda")
    a = bq.triangles.distanceBackward(tt, tv, tq, ids, g)
    b = bq.triangles.distanceBackward(tt, tv, tq, ids, g)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
