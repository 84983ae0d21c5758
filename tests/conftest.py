import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "pfsf-core_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpfsf.so")


@pytest.fixture(scope="session")
def lib_built():
    """Build libpfsf.so if needed (no GPU required to build)."""
    from build import build  # pfsf-core_b200/build.py

    return build()
