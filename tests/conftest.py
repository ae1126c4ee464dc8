import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def product_lib():
    from bioneuroncore_b200 import build, load_library
    build.ensure_built()
    return load_library()


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    # Build once if missing (the prebuilt .so files travel with the tree; a fresh
    # checkout builds here).  No rebuild when they exist: a copied tree may carry
    # source mtimes newer than its binaries.
    from bioneuroncore_b200 import build
    build.ensure_built()
    yield


def gpu_available():
    try:
        from bioneuroncore_b200 import build, load_library
        build.ensure_built()
        return load_library().gpu_backend_device_count() > 0
    except Exception:
        return False
