import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# the reference tree (read only by CPU tests that need it; absent on GPU machines)
REFERENCE = os.environ.get("PFVS_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def lib():
    """The built libpfvs_gpu.so (built here if missing)."""
    from pfvs_b200 import build, gpu
    build.build()
    return gpu._require()


@pytest.fixture(scope="session")
def ref_available():
    from oracle import ref
    return ref.available()
