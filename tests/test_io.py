"""The reference samples' binary-dump format (samples/common/IO.h:27-70):
files written by the reference's saveBinary read back by bq_load_binary /
bq_load_points_f64_as_f32 and the other way round.  Host only."""
import ctypes

import numpy as np
import pytest

import cubql_b200 as bq
from cubql_b200 import workloads as W


def _pts(n):
    rng = np.random.default_rng(1)
    p = rng.normal(size=(n, 3)) * np.array([1e-3, 1.0, 1e5])
    p[:4] = [[0.1, 1 / 3, 2 / 3], [1e-40, -0.0, 3.4e38], [1 + 2 ** -30, 1 - 2 ** -30, 0.5 + 2 ** -25], [7, 8, 9]]
    return p


def test_reference_files_read_back(tmp_path, ref_cpu):
    p = _pts(5000)
    path = tmp_path / "ref.bin"
    ref_cpu.save_points_f64(str(path), p)
    raw = path.read_bytes()
    assert len(raw) == 8 + 24 * len(p) and int.from_bytes(raw[:8], "little") == len(p)
    d = bq.io.loadBinary(path, ("<f8", 3))
    assert d.shape == (5000, 3) and np.array_equal(d, p)
    f = bq.io.loadPoints(path)
    assert np.array_equal(f, ref_cpu.load_points_f64_as_f32(str(path), len(p)))
    assert np.array_equal(f, p.astype(np.float32))


def test_our_files_read_by_reference(tmp_path, ref_cpu):
    p = _pts(3001)
    path = tmp_path / "ours.bin"
    bq.io.saveBinary(path, p)
    assert np.array_equal(ref_cpu.load_points_f64_as_f32(str(path), len(p)), p.astype(np.float32))
    # other element types: float boxes, u32 ids
    b = W.point_boxes(W.uniform_points(100))
    bq.io.saveBinary(tmp_path / "boxes.bin", b)
    assert np.array_equal(bq.io.loadBinary(tmp_path / "boxes.bin", ("<f4", 6)), b)
    ids = np.arange(77, dtype=np.uint32)
    bq.io.saveBinary(tmp_path / "ids.bin", ids)
    assert np.array_equal(bq.io.loadBinary(tmp_path / "ids.bin", np.uint32), ids)


def test_empty_and_bad_files(tmp_path):
    bq.io.saveBinary(tmp_path / "empty.bin", np.zeros((0, 3)))
    assert (tmp_path / "empty.bin").read_bytes() == bytes(8)
    assert bq.io.loadPoints(tmp_path / "empty.bin").shape == (0, 3)
    with pytest.raises(bq.BQError):
        bq.io.loadPoints(tmp_path / "missing.bin")
    (tmp_path / "short.bin").write_bytes((10).to_bytes(8, "little") + bytes(24 * 9))
    with pytest.raises(bq.BQError):
        bq.io.loadPoints(tmp_path / "short.bin")
    (tmp_path / "tiny.bin").write_bytes(bytes(3))
    with pytest.raises(bq.BQError):
        bq.io.loadBinary(tmp_path / "tiny.bin", np.float64)
    n = ctypes.c_uint64()
    out = np.zeros((2, 3), dtype=np.float32)
    bq.io.saveBinary(tmp_path / "five.bin", _pts(5))
    rc = bq._lib.bq_load_points_f64_as_f32(str(tmp_path / "five.bin").encode(), 3,
                                           out.ctypes.data_as(ctypes.c_void_p), 2, ctypes.byref(n))
    assert rc == 1 and n.value == 5  # capacity too small: BQ_ERR_INVALID_ARGUMENT, count still reported
