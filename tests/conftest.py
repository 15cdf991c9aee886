import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Builds libwindfvm.so (nvcc cross-compiles without a GPU) and the CPU oracle."""
    from unitywindsimulation_b200.build import build
    from oracle import build_oracle
    build()
    build_oracle()
    return True
