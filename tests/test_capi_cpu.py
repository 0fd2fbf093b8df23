"""C-ABI surface without a GPU: the library loads, exports every declared
symbol, rejects bad arguments with status codes, and its host-side
generators are right."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import cfm
import oracle
from conftest import PKG, ROOT


def declared_functions():
    hdr = open(os.path.join(ROOT, "include", "cfm.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(cfm_[a-z0-9_]+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 25
    lib = ctypes.CDLL(cfm.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert not [n for n in names if n not in cfm._SIGS]


def test_status_strings_and_version():
    assert cfm.lib.cfm_api_version() == 1
    assert cfm.lib.cfm_status_string(cfm.BARRIER_TIMEOUT) == b"grid barrier timeout"
    assert cfm.lib.cfm_status_string(99) == b"unknown status"


def test_bad_arguments_are_status_codes():
    p = cfm.JacobiParams(2, 2, 5, 1, cfm.FP64, 0, cfm.JACOBI_PERSISTENT)
    buf = np.zeros(10)
    assert cfm.lib.cfm_jacobi_problem_host(ctypes.byref(p), 0, buf.ctypes.data) == cfm.BAD_ARG
    p = cfm.JacobiParams(4, 8, 8, 8, cfm.FP64, 0, cfm.JACOBI_PERSISTENT)
    assert cfm.lib.cfm_jacobi_problem_host(ctypes.byref(p), 0, buf.ctypes.data) == cfm.BAD_ARG
    assert b"dims" in cfm.lib.cfm_last_error()
    assert cfm.lib.cfm_set_barrier_timeout_ms(-1.0) == cfm.BAD_ARG
    h = ctypes.c_void_p()
    rp = np.array([0, 2, 1], np.int32)  # decreasing rowptr
    assert cfm.lib.cfm_csr_create(2, 1, rp.ctypes.data, rp.ctypes.data, buf.ctypes.data,
                                  ctypes.byref(h)) == cfm.BAD_ARG


@pytest.mark.parametrize("dims,shape,problem,prec", [
    (2, (9, 12), 0, cfm.FP64), (2, (9, 12), 1, cfm.FP32),
    (3, (5, 6, 7), 0, cfm.FP32), (3, (5, 6, 7), 1, cfm.FP64), (3, (4, 9, 3), 0, cfm.FP64)])
def test_host_problem_matches_oracle_init(dims, shape, problem, prec):
    dt = cfm.np_dtype(prec)
    if dims == 2:
        ny, nx = shape
        p = cfm.JacobiParams(2, nx, ny, 1, prec, 1, cfm.JACOBI_PERSISTENT)
        want = oracle.jacobi2d_init(nx, ny, dt)
    else:
        nz, ny, nx = shape
        p = cfm.JacobiParams(3, nx, ny, nz, prec, problem, cfm.JACOBI_PERSISTENT)
        want = oracle.jacobi3d_init(nx, ny, nz, problem, dt)
    got = np.empty(shape, dt)
    cfm.check("problem", cfm.lib.cfm_jacobi_problem_host(ctypes.byref(p), problem, got.ctypes.data))
    np.testing.assert_array_equal(got, want)


def test_poisson_csr_matches_scipy():
    g = 5
    rowptr, col, val = cfm.poisson3d(g)
    one = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(g, g))
    eye = sp.identity(g)
    ref = (sp.kron(sp.kron(eye, eye), one) + sp.kron(sp.kron(eye, one), eye) +
           sp.kron(sp.kron(one, eye), eye)).tocsr()
    ref.sum_duplicates()
    ref.eliminate_zeros()
    ref.sort_indices()
    np.testing.assert_array_equal(rowptr, ref.indptr)
    np.testing.assert_array_equal(col, ref.indices)
    np.testing.assert_array_equal(val, ref.data)
    assert cfm.lib.cfm_poisson3d_nnz(128, 128, 128) == 14581760


def test_tridiag_structure():
    rowptr, col, val = cfm.tridiag(6)
    A = sp.csr_matrix((val, col, rowptr), shape=(6, 6))
    d = A.toarray()
    np.testing.assert_array_equal(d, d.T)  # the sub-diagonal copies the super-diagonal
    assert np.all(np.diag(d) >= 10) and np.all(np.diag(d) < 11)
    assert rowptr[-1] == 3 * 6 - 2


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    np.testing.assert_array_equal(cfm.philox([0, 0, 0, 0], [0, 0]),
                                  [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8])
    np.testing.assert_array_equal(cfm.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2),
                                  [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD])
    np.testing.assert_array_equal(
        cfm.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]),
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1])


def test_uniform_stream():
    u = cfm.uniform(0, 100001)
    assert u.min() >= -1 and u.max() < 1
    assert abs(u.mean()) < 0.01
    np.testing.assert_array_equal(u[:1000], cfm.uniform(0, 1000))
    assert not np.array_equal(u[:1000], cfm.uniform(1, 1000))


def _run(binary, *args):
    return subprocess.run([os.path.join(PKG, "bin", binary), *args], capture_output=True, text=True,
                          timeout=60)


def test_cli_version_table_and_rejections():
    r = _run("jacobi3D", "-v", "6")
    assert r.returncode == 2
    assert "0:\tBaseline Copy" in r.stdout and "5:\tPERKS" in r.stdout
    assert "Running Baseline Copy (No computation)" in r.stdout
    r = _run("jacobi2D", "-v", "42")
    assert r.returncode == 1 and "out of range" in r.stderr
    r = _run("cg", "-v", "0,99")
    assert r.returncode == 1
