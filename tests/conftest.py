import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the libbq kernels")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")):
        build()
    return Oracle()


@pytest.fixture(scope="session")
def ref_cpu():
    from oracle.oracle import RefCPU, have_ref_cpu
    if not have_ref_cpu():
        pytest.skip("oracle/_ref/libref_cpu.so not built (reference sources unavailable)")
    return RefCPU()


@pytest.fixture(scope="session")
def ref_gpu():
    from oracle.oracle import RefGPU, have_ref_gpu
    if not have_ref_gpu():
        pytest.skip("oracle/_ref/libref_gpu.so not built (reference sources unavailable)")
    return RefGPU()


@pytest.fixture(scope="session")
def bq():
    import cubql_b200
    return cubql_b200
