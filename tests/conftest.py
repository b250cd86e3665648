import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and libsoil_cuda.so")


@pytest.fixture(scope="session")
def ctx():
    """A soil_b200 context on cuda:0.  Fails (does not skip) without a GPU:
    GPU tests are selected with -m gpu and must run the CUDA path."""
    from soil_b200.system import Context
    return Context(0)
