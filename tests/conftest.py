"""Test configuration: import paths for the library, the oracle and the test helpers, the `gpu`
marker, and a session-wide library context for the GPU tests."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("rum-testing-gpu_b200", "oracle", "baseline", "tests", os.path.join("tests", "golden")):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_rumb")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the CUDA library)")


@pytest.fixture(scope="session")
def ctx():
    from rumb import _lib
    c = _lib.Context(0)
    yield c
    c.close()
