"""The allocation-free refit (bq_refit_noalloc_f3), called through the C ABI.

This entry point exists for callers that may not allocate device memory
at the moment they refit; it uses a fixed scratch array inside the
library.  Its boxes must equal those of the regular bq_refit_f3 bit for
bit (min/max is exact, so the test tolerance is zero), on two calls in a
row (the second call finds the first call's leftovers in the shared
scratch array).  Collected last, so a stop at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np

pytestmark = pytest.mark.gpu


def _clone_tree(bq, bvh):
    """A second tree with the same topology in its own buffers."""
    nodes = bvh.nodes_tensor().clone()
    prims = bvh.primids_tensor().clone()
    c = bq.bq_bvh3f(nodes.data_ptr(), bvh.numNodes, prims.data_ptr(), bvh.numPrims)
    return c, nodes, prims


def test_noalloc_refit_matches_regular_refit_twice(bq):
    pts = W.uniform_points(200000)
    b0 = torch.from_numpy(boxes_np(pts)).cuda()
    bvh = bq.cuda.radixBuilder(b0, bq.BuildConfig(makeLeafThreshold=4))
    assert 2 < bvh.numNodes <= 1 << 20
    c, nodes, prims = _clone_tree(bq, bvh)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call, seed in enumerate((101, 202)):
        moved = torch.from_numpy(boxes_np(pts + np.float32(0.02) * W.uniform_points(len(pts), seed, -1, 1))).cuda()
        bq.refit(bvh, moved)  # regular entry point (allocates its scratch)
        rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(moved.data_ptr()), stream)
        assert rc == bq.BQ_OK, bq._lib.bq_last_error_string()
        torch.cuda.synchronize()
        a = bvh.nodes_tensor().cpu().numpy().view(np.uint8)
        b = nodes.cpu().numpy().view(np.uint8)
        assert np.array_equal(a, b), f"call {call}: boxes differ from bq_refit_f3"


def test_noalloc_refit_rejects_oversized_tree(bq):
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    c = bq.bq_bvh3f(dummy.data_ptr(), (1 << 20) + 2, dummy.data_ptr(), 1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(dummy.data_ptr()), stream)
    assert rc == bq.BQ_ERR_INVALID_ARGUMENT
    assert b"at most 1048576" in bq._lib.bq_last_error_string()
