"""Shared helpers of the test-suite (CPU/GPU conversions, tree compare)."""
import numpy as np

from oracle.oracle import NODE


def boxes_np(pts):
    pts = np.asarray(pts, dtype=np.float32)
    return np.concatenate([pts, pts], 1)


def tri_boxes_np(verts, tris):
    v = verts[tris]
    return np.concatenate([v.min(1), v.max(1)], 1).astype(np.float32)


def same_tree(oracle, a_nodes, a_prims, b_nodes, b_prims, boxes=None):
    """Bit-exact equality after BFS renumbering (node 1 ignored).  With
    `boxes`, leaf prim sequences are compared through the prims' boxes, so
    identical prims may trade places (the reference's spatial-median
    builder sends identical prims to either side in atomic order)."""
    ca, pa = oracle.canonicalize(a_nodes, a_prims)
    cb, pb = oracle.canonicalize(b_nodes, b_prims)
    if len(ca) != len(cb):
        return False, f"node count {len(ca)} != {len(cb)}"
    if boxes is not None:
        bx = np.asarray(boxes, dtype=np.float32).reshape(-1, 6)
        same = np.array_equal(bx[pa], bx[pb]) and np.array_equal(np.sort(pa), np.sort(pb))
    else:
        same = np.array_equal(pa, pb)
    if not same:
        return False, f"leaf prim sequences differ at {np.nonzero(pa != pb)[0][:5]}"
    ca, cb = ca.copy(), cb.copy()
    if len(ca) > 1:
        ca[1] = np.zeros(1, dtype=NODE)
        cb[1] = np.zeros(1, dtype=NODE)
    if ca.tobytes() != cb.tobytes():
        bad = np.nonzero(ca.view(np.uint8).reshape(-1, 32).any(1) != cb.view(np.uint8).reshape(-1, 32).any(1))[0]
        diff = np.nonzero((ca.view(np.uint8).reshape(-1, 32) != cb.view(np.uint8).reshape(-1, 32)).any(1))[0]
        return False, f"{len(diff)} nodes differ, first {diff[:5]}"
    return True, ""


def fp64_closest(points, queries):
    """FP64 brute force (pattern of testing/points/closestPoint.cpp:37-59):
    squared distance and the lowest id attaining the FP64 minimum."""
    p = np.asarray(points, dtype=np.float64)
    out_d = np.empty(len(queries))
    out_i = np.empty(len(queries), dtype=np.int64)
    for s in range(0, len(queries), 256):
        q = np.asarray(queries[s:s + 256], dtype=np.float64)
        d = ((q[:, None, :] - p[None, :, :]) ** 2).sum(-1)
        out_i[s:s + 256] = d.argmin(1)
        out_d[s:s + 256] = d.min(1)
    return out_d, out_i
