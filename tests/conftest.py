import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle and the native library when they are missing or stale."""
    import oracle
    from ctas_b200 import build
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    build.build()
    yield
