"""Drop-in check: code written against the reference (its BinaryBVH,
box3f, BuildConfig and GpuMemoryResource types, its findClosest device
query) switched to this library through include/bq_cubql.hpp by changing
the builder call only; the reference's own traversal reads our tree and
gives the same answers as on the tree its own builder made."""
import numpy as np
import pytest

from cubql_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_reference_query_kernel_on_our_tree():
    from oracle.oracle import RefShim, have_ref_shim
    if not have_ref_shim():
        pytest.skip("oracle/_ref/libref_shim.so not built (reference sources unavailable)")
    pts = W.uniform_points(300000)
    qs = W.uniform_points(100000, W.SEED_QUERIES, -0.1, 1.1)
    ri, rd, oi, od, nn = RefShim().compare(pts, qs)
    assert nn[0] == nn[1] == 600000
    assert np.array_equal(ri, oi) and np.array_equal(rd, od)
