"""Refit of a caller's tree: every index read from the tree is range-checked
on the device, and a malformed tree is reported (BQ_ERR_INVALID_ARGUMENT)
instead of being followed out of range.  The trees are built on the host;
every access the kernels make on them stays inside the arrays given (the
checks skip the bad ones), so these run safely on the GPU."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _tree(admins, nprims):
    """nodes (len(admins), 8) float32 with zero boxes and the given
    (offset, count) admin words; primIDs 0..nprims-1; one box per prim."""
    nodes = np.zeros((len(admins), 8), np.float32)
    a = nodes.view(np.uint64).reshape(-1, 4)
    for i, (off, cnt) in enumerate(admins):
        a[i, 3] = np.uint64(off) | (np.uint64(cnt) << np.uint64(48))
    prims = np.arange(nprims, dtype=np.uint32)
    rng = np.random.default_rng(3)
    lo = rng.random((nprims, 3), dtype=np.float32)
    boxes = np.concatenate([lo, lo + np.float32(0.1)], 1).astype(np.float32)
    return nodes, prims, boxes


# a valid 4-prim tree: root 0 -> (2, 3), 2 -> (4, 5), 3 -> (6, 7), leaves 4..7 hold prims 0..3
VALID = [(2, 0), (0, 0), (4, 0), (6, 0), (0, 1), (1, 1), (2, 1), (3, 1)]


def malformed_trees():
    out = []
    bad = list(VALID)
    bad[0] = (7, 0)  # root's children 7, 8: node 8 does not exist
    out.append(("child past the node array",) + _tree(bad, 4))
    bad = list(VALID)
    bad[7] = (3, 2)  # prims 3, 4: prim 4 does not exist
    out.append(("leaf past the prim array",) + _tree(bad, 4))
    bad = list(VALID)
    bad[2] = (0, 0)  # children 0 (the root) and 1 (the unused node)
    out.append(("child at the root / unused node",) + _tree(bad, 4))
    return out


def _refit(bq, nodes, prims, boxes):
    tn, tp, tb = (torch.from_numpy(x).cuda() for x in (nodes, prims, boxes))
    c = bq.bq_bvh3f(tn.data_ptr(), len(nodes), tp.data_ptr(), len(prims))
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = bq._lib.bq_refit_f3(ctypes.byref(c), ctypes.c_void_p(tb.data_ptr()), None, s)
    torch.cuda.synchronize()
    return rc, tn.cpu().numpy()


def test_refit_of_a_valid_host_tree(bq):
    nodes, prims, boxes = _tree(VALID, 4)
    rc, out = _refit(bq, nodes, prims, boxes)
    assert rc == bq.BQ_OK, bq._lib.bq_last_error_string()
    for leaf, p in zip(range(4, 8), range(4)):
        assert np.array_equal(out[leaf, :6], boxes[p])
    u = lambda a, b: np.concatenate([np.minimum(a[:3], b[:3]), np.maximum(a[3:], b[3:])])  # noqa: E731
    assert np.array_equal(out[2, :6], u(boxes[0], boxes[1]))
    assert np.array_equal(out[3, :6], u(boxes[2], boxes[3]))
    assert np.array_equal(out[0, :6], u(out[2, :6], out[3, :6]))
    assert np.array_equal(out.view(np.uint64)[:, 3], nodes.view(np.uint64)[:, 3]), "admin words changed"


@pytest.mark.parametrize("case", range(3))
def test_refit_rejects_malformed_tree(bq, case):
    what, nodes, prims, boxes = malformed_trees()[case]
    rc, _ = _refit(bq, nodes, prims, boxes)
    assert rc == bq.BQ_ERR_INVALID_ARGUMENT, what
    assert b"malformed tree" in bq._lib.bq_last_error_string(), what
    # the context is still usable
    assert torch.ones(4, device="cuda").sum().item() == 4
