"""Seeded synthetic inputs for the build-and-query workloads.

Points follow the reference's sample generator: one LCG<8> per element,
seeded by TEA from (seed, index) (cuBQL/math/random.h:24-68), three draws
mapped as lo + u*(hi-lo) in double and rounded to float
(samples/common/Generator.cpp:201-215).  Everything is vectorised numpy so
a 10M-point set takes well under a second; the same streams come out of
the C restatement (orc_uniform_points), which the tests check.
"""
import numpy as np

SEED_DATA = 290374      # samples/s01_closestPoint_points_gpu/closestPoint.cu:77
SEED_QUERIES = 1234567  # samples/s01_closestPoint_points_gpu/closestPoint.cu:83
SEED_GMM = 7
SEED_GMM_QUERIES = 8  # fresh samples of the same mixture (queries)
SEED_MESH = 11
SEED_BATCH = 13

_M32 = np.uint32(0xFFFFFFFF)


def _tea8(v0, v1):
    v0 = v0.astype(np.uint32).copy()
    v1 = v1.astype(np.uint32).copy()
    s0 = np.uint32(0)
    with np.errstate(over="ignore"):
        for _ in range(8):
            s0 = np.uint32((int(s0) + 0x9E3779B9) & 0xFFFFFFFF)
            v0 += ((v1 << np.uint32(4)) + np.uint32(0xA341316C)) ^ (v1 + s0) ^ ((v1 >> np.uint32(5)) + np.uint32(0xC8013EA4))
            v1 += ((v0 << np.uint32(4)) + np.uint32(0xAD90777D)) ^ (v0 + s0) ^ ((v0 >> np.uint32(5)) + np.uint32(0x7E95761E))
    return v0


def lcg_streams(n, seed, draws, start=0):
    """(n, draws) float32 uniforms in [0,1): draw j of LCG<8>(seed, start+i)."""
    idx = np.arange(start, start + n, dtype=np.uint64).astype(np.uint32)
    st = _tea8(np.full(n, seed, dtype=np.uint32), idx)
    out = np.empty((n, draws), dtype=np.float32)
    with np.errstate(over="ignore"):
        for j in range(draws):
            st = st * np.uint32(1664525) + np.uint32(1013904223)
            out[:, j] = (st & np.uint32(0x00FFFFFF)).astype(np.float32) / np.float32(16777216.0)
    return out


def uniform_points(n, seed=SEED_DATA, lo=0.0, hi=1.0):
    """(n,3) float32, U[lo,hi)^3 as the reference's UniformPointGenerator."""
    u = lcg_streams(n, seed, 3).astype(np.float64)
    return (lo + u * (hi - lo)).astype(np.float32)


def gmm_points(n, seed=SEED_GMM, components=64, offset=1e5, sigma_lo=1e-4, sigma_hi=1e-1, sample_seed=None):
    """(n,3) float32 from a `components`-Gaussian mixture: centres U[0,1]^3,
    sigma log-uniform in [sigma_lo, sigma_hi], equal weights, every
    coordinate shifted by `offset` (at 1e5 the float spacing is ~0.0078, so
    the tight clusters collapse into exact duplicates).  The mixture comes
    from `seed`, the samples from `sample_seed` (default: `seed`), so queries
    from the same distribution are gmm_points(nq, sample_seed=...)."""
    c = lcg_streams(components, seed ^ 0x5bd1e995, 4).astype(np.float64)
    centres = c[:, :3]
    sig = np.exp(np.log(sigma_lo) + c[:, 3] * (np.log(sigma_hi) - np.log(sigma_lo)))
    u = lcg_streams(n, seed if sample_seed is None else sample_seed, 7).astype(np.float64)
    comp = np.minimum((u[:, 0] * components).astype(np.int64), components - 1)
    u1 = np.maximum(u[:, 1:4], 1e-12)
    u2 = u[:, 4:7]
    g = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)  # Box-Muller
    pts = centres[comp] + sig[comp, None] * g + offset
    return pts.astype(np.float32)


def point_boxes(pts):
    """box3f().including(p): lower = upper = p, as (n,6) float32."""
    pts = np.asarray(pts, dtype=np.float32)
    return np.concatenate([pts, pts], axis=1)


def icosphere(level, seed=SEED_MESH, amp=0.05):
    """Icosphere subdivided `level` times (20*4^level faces,
    10*4^level+2 vertices), every vertex scaled radially by (1 + amp*u),
    u ~ U[-1,1] seeded.  Returns (verts (V,3) float32, tris (T,3) int32)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, dtype=np.int64)
    for _ in range(level):
        nv = verts.shape[0]
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (nv + 1), uniq % (nv + 1)
        mid = verts[a] + verts[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        verts = np.concatenate([verts, mid], axis=0)
        nf = faces.shape[0]
        m = inv.reshape(3, nf) + nv  # midpoints of edges 01, 12, 20
        m01, m12, m20 = m[0], m[1], m[2]
        faces = np.concatenate([
            np.stack([faces[:, 0], m01, m20], 1), np.stack([faces[:, 1], m12, m01], 1),
            np.stack([faces[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)], axis=0)
    u = lcg_streams(verts.shape[0], seed, 1)[:, 0].astype(np.float32) * np.float32(2.0) - np.float32(1.0)
    scale = np.float32(1.0) + np.float32(amp) * u
    out = (verts.astype(np.float32) * scale[:, None]).astype(np.float32)
    return out, faces.astype(np.int32)


def cloud_batch(num=512, lo=1000, hi=200000, queries_per_cloud=50000, seed=SEED_BATCH):
    """Batched workload: `num` clouds with sizes floor(exp(U[ln lo, ln hi])),
    each by a seeded coin flip either uniform in [0,1]^3 or an 8-cluster
    Gaussian mixture (sigma 0.02), plus `queries_per_cloud` uniform queries
    per cloud.  Returns (points (N,3), offsets (num+1,), queries (Q,3),
    query offsets (num+1,)), clouds stored back to back."""
    u = lcg_streams(num, seed, 2).astype(np.float64)
    sizes = np.floor(np.exp(np.log(lo) + u[:, 0] * (np.log(hi) - np.log(lo)))).astype(np.int64)
    pts, qs = [], []
    for c in range(num):
        n = int(sizes[c])
        s = seed * 1000 + c
        if u[c, 1] < 0.5:
            p = uniform_points(n, s)
        else:
            cen = lcg_streams(8, s ^ 0x2545F491, 3).astype(np.float64)
            v = lcg_streams(n, s, 7).astype(np.float64)
            k = np.minimum((v[:, 0] * 8).astype(np.int64), 7)
            g = np.sqrt(-2.0 * np.log(np.maximum(v[:, 1:4], 1e-12))) * np.cos(2.0 * np.pi * v[:, 4:7])
            p = (cen[k] + 0.02 * g).astype(np.float32)
        pts.append(p)
        qs.append(uniform_points(queries_per_cloud, s ^ 0x68E31DA4))
    off = np.zeros(num + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    qoff = np.arange(num + 1, dtype=np.int64) * queries_per_cloud
    return np.concatenate(pts), off, np.concatenate(qs), qoff


_ICO_CACHE = {}


def mesh_batch(num=128, lo=2000, hi=100000, queries_per_mesh=50000, seed=SEED_MESH):
    """Batched-mesh workload: `num` icosphere-derived meshes with target
    triangle counts log-uniform in [lo, hi]; each takes the smallest
    icosphere level with at least that many faces and keeps its first
    `target` faces (open meshes allowed), plus `queries_per_mesh` queries
    uniform in [-1.5, 1.5]^3.  Returns (verts (V,3), tris (T,3) int32 with
    global vertex indices, tri offsets (num+1,), queries (Q,3), query
    offsets (num+1,))."""
    u = lcg_streams(num, seed, 1)[:, 0].astype(np.float64)
    targets = np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)
    verts, tris, qs = [], [], []
    vbase = 0
    toff = [0]
    for m in range(num):
        level = 0
        while 20 * 4 ** level < targets[m]:
            level += 1
        key = (level, seed * 1000 + m)
        v, t = icosphere(level, seed=seed * 1000 + m)
        t = t[: targets[m]]
        verts.append(v)
        tris.append(t + vbase)
        vbase += len(v)
        toff.append(toff[-1] + len(t))
        qs.append(uniform_points(queries_per_mesh, seed * 7919 + m, -1.5, 1.5))
    qoff = np.arange(num + 1, dtype=np.int64) * queries_per_mesh
    return (np.concatenate(verts), np.concatenate(tris).astype(np.int32), np.array(toff, dtype=np.int64),
            np.concatenate(qs), qoff)
