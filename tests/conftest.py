import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_INPUT = os.path.join(GOLDEN, "ab5_input.txt")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """The CPU tests use the host half of libedus_b200.so; build it if absent."""
    from edus_b200 import lib

    if not os.path.exists(lib.library_path()):
        from edus_b200 import build

        build.build()
    yield


@pytest.fixture
def workdir(tmp_path):
    return str(tmp_path)
