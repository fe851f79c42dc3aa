import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the native library's kernels")


_GPU = None


def gpu_available() -> bool:
    global _GPU
    if _GPU is None:
        try:
            import torch
            _GPU = bool(torch.cuda.is_available())
        except Exception:
            _GPU = False
    return _GPU


def pytest_collection_modifyitems(config, items):
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords and not gpu_available():
            it.add_marker(skip)


@pytest.fixture(scope="session")
def built_lib():
    from hacc_gpm_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    from hacc_gpm_b200 import binding
    return binding.lib()
