import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200, sm_100a) device")


@pytest.fixture(scope="session")
def ctx():
    """One CUDA context for the GPU tests (fails loudly without the library
    or a device: there is no CPU fallback)."""
    from protomol_b200 import Context
    c = Context(0)
    yield c
    c.close()
