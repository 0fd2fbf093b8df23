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


def ref_cg_fixtures():
    """tests/golden/ref_cg_*.npz: x written by the reference's own single-GPU
    CG (made by tests/golden/make_ref_fixtures.py)."""
    import glob
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_cg_*.npz")))


def ref_cg_system(path):
    """(rowptr, col, val, niter, x_ref) of a reference CG fixture, the matrix
    in the index base the reference was given."""
    import numpy as np

    import cfm
    f = np.load(path)
    if str(f["matrix"]) == "tridiag":
        rowptr, col, val = f["rowptr"], f["col"], f["val"]
    else:
        rowptr, col, val = cfm.poisson3d(int(f["size"]))
    if bool(f["one_based"]):
        rowptr, col = rowptr + 1, col + 1
    return rowptr, col, val, int(f["niter"]), f["x"]


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
