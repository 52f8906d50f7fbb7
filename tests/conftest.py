import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session", autouse=True)
def _native_libs():
    """Build the in-tree native libraries once if they are missing (nvcc cross-compiles)."""
    from grhd_b200 import build
    build.build_host()
    if not os.path.exists(os.path.join(build.LIB, "libgrhd2gpu.so")):
        build.build_gpu()
    from oracle import binding
    if not os.path.exists(binding.LIB):
        binding.build()
    yield


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
