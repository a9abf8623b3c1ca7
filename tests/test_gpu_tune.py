"""The single-tree autotuner (bq_autotune_query_f3) through the JSON cache:
it returns one of the timed launch shapes, a second call is a cache hit,
and queries run with the tuned shape give exactly the default answers
(the knobs change the time, never the result)."""
import numpy as np
import pytest
import torch

from cubql_b200 import tuning
from cubql_b200 import workloads as W
from tests.helpers import boxes_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [0, 16])
def test_tuned_query_shape_and_answers(bq, tmp_path, k):
    pts = W.uniform_points(100_000)
    b = torch.from_numpy(boxes_np(pts)).cuda()
    tp = torch.from_numpy(pts).cuda()
    qs = torch.from_numpy(W.uniform_points(50_000, W.SEED_QUERIES)).cuda()
    path = str(tmp_path / "tuning.json")
    t = tuning.tuned_query(b, tp, qs, k, path=path)
    assert not t["cached"]
    assert t["makeLeafThreshold"] in (1, 2, 4, 8) and t["stackDepth"] in (32, 64, 128)
    assert t["blockSize"] in (64, 128) and t["buildMs"] > 0 and t["queryMs"] > 0
    assert tuning.tuned_query(b, tp, qs, k, path=path)["cached"]
    bvh = bq.cuda.radixBuilder(b, bq.BuildConfig(makeLeafThreshold=t["makeLeafThreshold"]))
    ref = bq.cuda.radixBuilder(b)
    qc = tuning.query_config_of(t)
    if k == 0:
        a = bq.points.findClosest(bvh, tp, qs, qcfg=qc)
        r = bq.points.findClosest(ref, tp, qs)
    else:
        a = bq.points.findKNN(bvh, tp, qs, k, qcfg=qc)[:2]
        r = bq.points.findKNN(ref, tp, qs, k)[:2]
    assert all(torch.equal(x, y) for x, y in zip(a, r))
