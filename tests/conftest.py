import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA engine)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native libraries in-tree once per session (no-op when fresh)."""
    from ucns3d_b200 import build
    build.build_prep()
    import oracle as orc
    orc.build()
    yield
