import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("lasp-d3_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libd3.so")


def _have_gpu():
    """True when the CUDA driver reports at least one device (no torch import)."""
    import ctypes

    try:
        cu = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    if cu.cuInit(0) != 0:
        return False
    n = ctypes.c_int(0)
    return cu.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
