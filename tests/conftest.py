import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libklft_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, build
    build()
    return Oracle()


@pytest.fixture(scope="session")
def refshim():
    from oracle.oracle import REF_SO, RefShim, build
    build()
    if not os.path.exists(REF_SO):
        pytest.skip("reference shim library not built (reference sources were not available at build time)")
    return RefShim()


def has_gpu():
    try:
        import klft_b200
        return klft_b200.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def refadj():
    from oracle.oracle import REF_ADJ_SO, RefAdjoint, build
    build()
    if not os.path.exists(REF_ADJ_SO):
        pytest.skip("reference adjoint library not built (reference sources were not available at build time)")
    return RefAdjoint()
