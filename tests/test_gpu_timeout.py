"""The radix sort's bounded look-back wait, made to run out on purpose from
the host (bq_debug_inject_sort_timeout: the first tile holds back its
totals, so every wait on it gives up after a short spin).  The call must
return BQ_ERR_TIMEOUT, everything downstream of the aborted sort must
still see in-range indices, and the next call must work normally."""
import numpy as np
import pytest
import torch

from cubql_b200 import workloads as W
from tests.helpers import boxes_np, same_tree

pytestmark = pytest.mark.gpu


def test_query_order_sort_timeout_is_reported_and_harmless(bq):
    pts = W.uniform_points(200_000)
    qs = torch.from_numpy(W.uniform_points(300_000, W.SEED_QUERIES)).cuda()
    tp = torch.from_numpy(pts).cuda()
    bvh = bq.cuda.radixBuilder(torch.from_numpy(boxes_np(pts)).cuda())
    ref_ids, ref_d = bq.points.findClosest(bvh, tp, qs)
    import ctypes
    ids = torch.full_like(ref_ids, -7)
    d = torch.full_like(ref_d, -7.0)
    q = bq.query_config()
    bq._check(bq._lib.bq_debug_inject_sort_timeout(1))
    rc = bq._lib.bq_closest_point_f3(ctypes.byref(bvh.c), tp.data_ptr(), qs.data_ptr(), qs.shape[0],
                                     float("inf"), ctypes.byref(q), ids.data_ptr(), d.data_ptr(),
                                     ctypes.byref(bvh.allocator.c), torch.cuda.current_stream().cuda_stream)
    assert rc == bq.BQ_ERR_TIMEOUT
    assert b"timed out" in bq._lib.bq_last_error_string()
    # the aborted sort's output was repaired to the identity order (in range),
    # so the query kernel after it still answered every query exactly
    assert torch.equal(ids, ref_ids) and torch.equal(d, ref_d)
    ids2, d2 = bq.points.findClosest(bvh, tp, qs)  # the hook was used up: a normal call
    assert torch.equal(ids2, ref_ids) and torch.equal(d2, ref_d)


def test_morton_build_sort_timeout_is_reported_and_next_build_is_exact(bq, oracle):
    b = boxes_np(W.uniform_points(300_000))
    tb = torch.from_numpy(b).cuda()
    bq._check(bq._lib.bq_debug_inject_sort_timeout(1))
    with pytest.raises(bq.BQError) as e:
        bq.cuda.radixBuilder(tb)
    assert e.value.code == bq.BQ_ERR_TIMEOUT
    assert torch.ones(8, device="cuda").sum().item() == 8  # the context is healthy
    bvh = bq.cuda.radixBuilder(tb)
    gn, gp = bvh.to_host()
    on, op = oracle.radix_build(b)
    ok, msg = same_tree(oracle, gn, gp, on, op)
    assert ok, msg
    assert np.all(gp < len(b))
