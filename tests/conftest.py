import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhedft.so")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle (CPU) and, when nvcc is present, libhedft.so before any test."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    from he_dft_2024_b200 import build
    try:
        build.build()
    except RuntimeError:
        if os.path.exists(build.LIB):
            pass
        else:
            raise
    yield
