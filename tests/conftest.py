import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libqm_gpu.so")


@pytest.fixture(scope="session")
def ctx():
    """A qm_ctx on cuda:0.  GPU tests fail loudly when the library or the
    device is missing: there is no CPU fallback."""
    from querymode_b200.engine import Context
    c = Context(0)
    yield c
    c.close()
