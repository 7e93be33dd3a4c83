import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


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


_FP64 = {}


@pytest.fixture(scope="session")
def fp64_report():
    """Per-case FP64 edge-weight error reports, printed at the end of the run."""
    return _FP64


def pytest_terminal_summary(terminalreporter):
    if _FP64:
        terminalreporter.write_line("edge weights vs FP64: max abs error over edges with the "
                                    "same cut; edges; cut disagreements (FP64 value on a "
                                    "threshold) and their largest FP64 distance to it")
        for k, v in sorted(_FP64.items()):
            terminalreporter.write_line(f"  {k}: {v['max_abs_err_fp64']:.3e}  {v['edges']}  "
                                        f"{v['cut_disagreements']}  "
                                        f"{v['max_margin_disagreeing']:.3e}")
