import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built CUDA library")


@pytest.fixture(scope="session")
def backend():
    """One CUDA context for the GPU tests (fails loudly without a GPU: no CPU fallback)."""
    from fastwarp_b200 import CudaBackend
    b = CudaBackend(0)
    yield b
    b.close()
