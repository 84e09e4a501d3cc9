import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _have_gpu():
    try:
        import ctypes
        cudart = None
        for name in ("libcudart.so", "libcudart.so.12"):
            try:
                cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if cudart is None:
            import torch  # noqa: F401
            return torch.cuda.is_available()
        n = ctypes.c_int(0)
        return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return _have_gpu()


def pytest_collection_modifyitems(config, items):
    # GPU tests run where a GPU is present; they are never silently skipped on
    # a GPU box (a missing library there is a failure, not a skip).
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this container")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
