import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU; calls the CUDA path through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Make sure the oracle port and the product library exist (incremental; nvcc cross-compiles)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)
    from euler3d_b200 import build as b

    b.build()
    yield
