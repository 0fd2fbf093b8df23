import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cpu-free-model_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


def _have_gpu():
    import cfm  # noqa: E402  (raises if libcfm.so is missing: no fallback)
    st, *_ = cfm.device_info()
    return st == cfm.OK


def pytest_collection_modifyitems(config, items):
    gpu_items = [it for it in items if "gpu" in it.keywords]
    if not gpu_items:
        return
    if not _have_gpu():
        skip = pytest.mark.skip(reason="no CUDA device visible")
        for it in gpu_items:
            it.add_marker(skip)
