import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libfenixcuda.so")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the oracle (g++) and, where nvcc exists, the CUDA library before the tests."""
    from oracle import build as orc_build

    orc_build.build()
    from fenix_b200 import build as fx_build

    if fx_build.needs_build() or fx_build.needs_build(fx_build.OUTPUT_FAST):
        try:
            fx_build.build()
        except Exception:  # no nvcc on this machine: the GPU tests fail loudly on load
            pass
