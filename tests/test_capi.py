"""The C ABI: libbq.so loads and exports every entry point include/bq.h
declares; the Python bindings cover all of them.  No GPU needed."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "bq.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bq_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(ROOT, "cubql_b200", "libbq.so"))
    names = declared()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    import cubql_b200
    assert sorted(cubql_b200.exported_symbols()) == declared()


def test_version_and_error_string():
    import cubql_b200
    assert cubql_b200.version() == 100
    assert isinstance(cubql_b200._lib.bq_last_error_string(), bytes)


def test_node_layout_matches_reference():
    import cubql_b200
    assert ctypes.sizeof(cubql_b200.bq_bvh3f) == 32  # BinaryBVH<float,3>: ptr, u32, ptr, u32
    assert cubql_b200.node_dtype().itemsize == 32    # BinaryBVH<float,3>::Node
    from oracle.oracle import have_ref_cpu, RefCPU
    if have_ref_cpu():
        assert RefCPU().lib.ref_cpu_node_size() == 32


def test_invalid_arguments_are_reported_not_raised():
    import cubql_b200 as bq
    c = bq.bq_bvh3f()
    # NULL boxes with n > 0: rejected before any CUDA call
    rc = bq._lib.bq_build_morton63_f3(ctypes.byref(c), None, 10, None, None, None)
    assert rc == bq.BQ_ERR_INVALID_ARGUMENT
    assert b"boxes" in bq._lib.bq_last_error_string()
    rc = bq._lib.bq_build_spatial_median_f3(None, None, 0, None, None, None)
    assert rc == bq.BQ_ERR_INVALID_ARGUMENT
