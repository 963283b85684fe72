"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on the CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref_harness():
    """The reference's own sources compiled here (oracle/_ref); skipped where it was not built."""
    from oracle.bindings import REF_LIB, RefHarness
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libswref.so not built (reference sources unavailable)")
    return RefHarness()


@pytest.fixture(scope="session")
def device():
    import swpathtracer_b200 as spt
    d = spt.Device(0)
    yield d
    d.close()
