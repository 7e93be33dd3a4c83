import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def ref_lib():
    """RabbitBin's own code (oracle/_ref), or skip when it was never built."""
    import oracle
    lib = oracle.ref()
    if lib is None:
        pytest.skip("reference harness not built (reference tree absent)")
    return lib


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.restated()


@pytest.fixture(scope="session")
def gpu_ctx():
    from rabbitbin_b200 import api
    return api.Context(0)
