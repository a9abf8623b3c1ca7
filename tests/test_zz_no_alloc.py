"""The allocation-free refit (bq_refit_noalloc_f3), called through the C ABI.

This entry point exists for callers that may not allocate device memory
at the moment they refit (memory reserved up front for their own pool, a
real-time loop, a framework that allocates only during set-up); it uses a
fixed scratch array inside the library.  Its boxes must equal those of the
regular bq_refit_f3 bit for bit (min/max is exact, so the test tolerance is
zero), on two calls in a row (the second call finds the first call's
leftovers in the shared scratch array), on a small tree and on one of
exactly BQ_NOALLOC_REFIT_MAX_NODES nodes; around a call neither torch's
allocator nor the device's free memory may change.  Collected last, so a
stop at the first failure has already run every other test."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np

pytestmark = pytest.mark.gpu

MAX_NODES = 1 << 20
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _clone_tree(bq, bvh):
    """A second tree with the same topology in its own buffers."""
    nodes = bvh.nodes_tensor().clone()
    prims = bvh.primids_tensor().clone()
    c = bq.bq_bvh3f(nodes.data_ptr(), bvh.numNodes, prims.data_ptr(), bvh.numPrims)
    return c, nodes, prims


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _setup(bq):
    """The set-up call: numNodes == 0 places the scratch array on this device."""
    empty = bq.bq_bvh3f(None, 0, None, 0)
    rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(empty), None, _stream())
    assert rc == bq.BQ_OK, bq._lib.bq_last_error_string()
    torch.cuda.synchronize()


def _compare_two_calls(bq, pts, leaf):
    b0 = torch.from_numpy(boxes_np(pts)).cuda()
    bvh = bq.cuda.radixBuilder(b0, bq.BuildConfig(makeLeafThreshold=leaf))
    assert 2 < bvh.numNodes <= MAX_NODES
    c, nodes, prims = _clone_tree(bq, bvh)
    _setup(bq)
    for call, seed in enumerate((101, 202)):
        moved = torch.from_numpy(boxes_np(pts + np.float32(0.02) * W.uniform_points(len(pts), seed, -1, 1))).cuda()
        bq.refit(bvh, moved)  # regular entry point (allocates its scratch)
        torch.cuda.synchronize()
        torch_before = torch.cuda.memory_allocated()
        free_before = torch.cuda.mem_get_info()[0]
        rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(moved.data_ptr()), _stream())
        assert rc == bq.BQ_OK, bq._lib.bq_last_error_string()
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == torch_before, f"call {call}: torch allocated memory"
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {call}: device free memory changed"
        a = bvh.nodes_tensor().cpu().numpy().view(np.uint8)
        b = nodes.cpu().numpy().view(np.uint8)
        assert np.array_equal(a, b), f"call {call}: boxes differ from bq_refit_f3"
    return bvh.numNodes


def test_noalloc_refit_matches_regular_refit_twice(bq):
    _compare_two_calls(bq, W.uniform_points(200000), 4)


def test_noalloc_refit_at_the_node_limit(bq):
    # leaf 1: a Morton tree over n prims has 2n nodes, so 2^19 prims fill the array exactly
    assert _compare_two_calls(bq, W.uniform_points(MAX_NODES // 2, 77), 1) == MAX_NODES


def test_noalloc_refit_rejects_oversized_tree(bq):
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    c = bq.bq_bvh3f(dummy.data_ptr(), MAX_NODES + 2, dummy.data_ptr(), 1)
    rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(dummy.data_ptr()), _stream())
    assert rc == bq.BQ_ERR_INVALID_ARGUMENT
    assert b"at most 1048576" in bq._lib.bq_last_error_string()


def test_noalloc_refit_rejects_malformed_tree(bq):
    from tests.test_gpu_refit_guard import malformed_trees
    for what, nodes, prims, boxes in malformed_trees():
        tn, tp, tb = (torch.from_numpy(x).cuda() for x in (nodes, prims, boxes))
        c = bq.bq_bvh3f(tn.data_ptr(), len(nodes), tp.data_ptr(), len(prims))
        rc = bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(tb.data_ptr()), _stream())
        assert rc == bq.BQ_ERR_INVALID_ARGUMENT, what
        assert b"malformed tree" in bq._lib.bq_last_error_string(), what


_LAZY_CHILD = r"""
import ctypes, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import cubql_b200 as bq
from cubql_b200 import workloads as W
pts = W.uniform_points(50000)
boxes = torch.from_numpy(np.concatenate([pts, pts], 1)).cuda()
bvh = bq.cuda.radixBuilder(boxes, bq.BuildConfig(makeLeafThreshold=2))
nodes = bvh.nodes_tensor().clone(); prims = bvh.primids_tensor().clone()
c = bq.bq_bvh3f(nodes.data_ptr(), bvh.numNodes, prims.data_ptr(), bvh.numPrims)
s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
empty = bq.bq_bvh3f(None, 0, None, 0)
assert bq._lib.bq_refit_noalloc_f3(ctypes.byref(empty), None, s) == 0
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
for seed in (5, 6):
    q = pts + np.float32(0.01) * W.uniform_points(len(pts), seed, -1, 1)
    moved = torch.from_numpy(np.concatenate([q, q], 1)).cuda()
    torch.cuda.synchronize()
    f = torch.cuda.mem_get_info()[0]
    assert bq._lib.bq_refit_noalloc_f3(ctypes.byref(c), ctypes.c_void_p(moved.data_ptr()), s) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == f, "a call after the set-up call changed the device's free memory"
    bq.refit(bvh, moved)
    assert torch.equal(bvh.nodes_tensor().view(torch.int32), nodes.view(torch.int32))
print("setup_bytes", free0 - free1)
"""


def test_noalloc_refit_setup_call_under_lazy_loading():
    """In a fresh process with lazy module loading: after the set-up call,
    refits leave the device's free memory unchanged."""
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", _LAZY_CHILD, ROOT], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "setup_bytes" in r.stdout
