"""CG parity on the GPU through the C ABI: the persistent kernel and the
host-controlled comparator reproduce the oracle's solution and iteration
count exactly (same reduction tree), in tolerance and fixed-count modes."""
import numpy as np
import pytest

import cfm
import oracle
from conftest import ref_cg_fixtures, ref_cg_system

pytestmark = pytest.mark.gpu

IMPLS = [cfm.CG_DISCRETE, cfm.CG_PERSISTENT]


def poisson_system(g, seed=0):
    rowptr, col, val = cfm.poisson3d(g)
    A = cfm.CSR(rowptr, col, val)
    xs = cfm.uniform(seed, A.n)
    return A, xs, A.spmv(xs)


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("g", [3, 10, 16, 33])
def test_cg_poisson_tolerance_bitexact(impl, g):
    A, xs, b = poisson_system(g)
    np.testing.assert_array_equal(b, oracle.spmv(A.rowptr, A.col, A.val, xs))
    x_o, st_o, it_o, rr_o = oracle.cg(A.rowptr, A.col, A.val, b, 20000, 1e-8)
    x, st = cfm.CG(A, impl, 20000, 1e-8).solve(b)
    assert st.status == cfm.OK and st_o == 0
    assert st.iterations == it_o
    np.testing.assert_array_equal(x, x_o)
    assert st.residual <= 1e-8
    assert abs(st.residual - rr_o) <= 1e-20 + 1e-12 * rr_o


@pytest.mark.parametrize("impl", IMPLS)
def test_cg_reference_mode_fixed_count_tridiag(impl):
    """The reference's default run: its random tridiagonal matrix, b = ones,
    x0 = 0, exactly -niter iterations, no tolerance exit."""
    rowptr, col, val = cfm.tridiag(5000)
    A = cfm.CSR(rowptr, col, val)
    x_o, st_o, it_o, _ = oracle.cg(rowptr, col, val, None, 25, 0.0)
    x, st = cfm.CG(A, impl, 25, 0.0).solve(None)
    assert st.iterations == 25 == it_o
    np.testing.assert_array_equal(x, x_o)


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("path", ref_cg_fixtures(), ids=lambda p: p.rsplit("/", 1)[-1])
def test_cg_matches_reference_run(impl, path):
    """Parity with the reference's own single-GPU CG (x written by
    SingleGPUDiscreteStandard::run_single_gpu(), CG/src/common.cu:399-538, on a
    B200): b = ones, x0 = 0, the same fixed count; x within 1e-12 relative
    (the reference's dots are atomicAdd sums in arrival order)."""
    rowptr, col, val, niter, x_ref = ref_cg_system(path)
    x, st = cfm.CG(cfm.CSR(rowptr, col, val), impl, niter, 0.0).solve(None)
    assert st.iterations == niter
    rel = np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)
    assert rel <= 1e-12, rel


def test_cg_one_based_csr_same_result():
    rowptr, col, val = cfm.poisson3d(7)
    A0 = cfm.CSR(rowptr, col, val)
    A1 = cfm.CSR(rowptr + 1, col + 1, val)
    b = np.linspace(-1, 1, A0.n)
    x0, _ = cfm.CG(A0, cfm.CG_PERSISTENT, 500, 1e-10).solve(b)
    x1, _ = cfm.CG(A1, cfm.CG_PERSISTENT, 500, 1e-10).solve(b)
    np.testing.assert_array_equal(x0, x1)


def test_cg_breakdown_and_not_converged_statuses():
    A = cfm.CSR(np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.array([1.0, -1.0, 2.0]))
    _, st = cfm.CG(A, cfm.CG_PERSISTENT, 10, 1e-12).solve(np.array([1.0, 1.0, 0.0]),
                                                          allowed=(cfm.BREAKDOWN,))
    assert st.status == cfm.BREAKDOWN
    A, xs, b = poisson_system(12)
    _, st = cfm.CG(A, cfm.CG_PERSISTENT, 5, 1e-12).solve(b)
    assert st.status == cfm.NOT_CONVERGED and st.iterations == 5


def test_cg_config3_poisson128_persistent_vs_oracle():
    """The 128^3 Poisson CSR system (n = 2,097,152, nnz = 14,581,760) to 1e-8:
    same iteration count and the same x as the oracle."""
    A, xs, b = poisson_system(128)
    assert len(A.val) == 14581760
    x_o, st_o, it_o, rr_o = oracle.cg(A.rowptr, A.col, A.val, b, 20000, 1e-8)
    x, st = cfm.CG(A, cfm.CG_PERSISTENT, 20000, 1e-8).solve(b)
    assert st_o == 0 and st.status == cfm.OK
    assert abs(st.iterations - it_o) <= 1
    rel = np.linalg.norm(x - x_o) / np.linalg.norm(x_o)
    assert rel <= 1e-12, rel
    assert st.residual <= 1e-8
    assert st.launches == 1


def test_cg_on_matrixmarket_file(tmp_path):
    """-matrix_path input: a symmetric MatrixMarket file (lower triangle
    stored) read back, uploaded with its 1-based indices and solved with
    b = ones, equals the same system built in memory, bit for bit."""
    import os
    import subprocess

    import scipy.io
    import scipy.sparse as sp

    rowptr, col, val = cfm.poisson3d(9)
    n = len(rowptr) - 1
    A = sp.csr_matrix((val, col, rowptr), shape=(n, n))
    p = tmp_path / "poisson9.mtx"
    scipy.io.mmwrite(str(p), A.tocoo(), symmetry="symmetric")
    r2, c2, v2, m, n2 = cfm.mm_read(str(p))
    assert m == n2 == n and r2[0] == 1
    x_file, st = cfm.CG(cfm.CSR(r2, c2, v2), cfm.CG_PERSISTENT, 2000, 1e-10).solve(None)
    x_mem, st_mem = cfm.CG(cfm.CSR(rowptr, col, val), cfm.CG_PERSISTENT, 2000, 1e-10).solve(None)
    assert st.status == cfm.OK and st.iterations == st_mem.iterations
    np.testing.assert_array_equal(x_file, x_mem)
    binary = os.path.join(os.path.dirname(cfm.__file__), "bin", "cg")
    out = subprocess.run([binary, "-v", "1", "-s", "-matrix_path", str(p), "-niter", "50"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    first = next(t for t in out.stdout.split() if t.replace(".", "", 1).isdigit())
    assert float(first) > 0  # the first float is the time, as the reference prints it


@pytest.mark.parametrize("version,method", [(2, "std"), (3, "pipelined"), (5, "std"), (9, "pipelined")])
def test_cg_binary_versions_run_their_kernel(version, method):
    """The binary's "Single Stream Standard / Pipelined" versions run the
    standard and the pipelined persistent kernels: the iteration count and
    the restarts (the pipelined kernel's residual replacement every 50
    iterations) are that method's (the oracle's), in one launch."""
    import os
    import re
    import subprocess

    g = 16
    rowptr, col, val = cfm.poisson3d(g)
    b = cfm.CSR(rowptr, col, val).spmv(cfm.uniform(0, len(rowptr) - 1))
    m = oracle.STD if method == "std" else oracle.PIPELINED
    _, st_o, it_o, rs_o, _ = oracle.krylov_csr(rowptr, col, val, b, m, 20000, 1e-8)
    binary = os.path.join(os.path.dirname(cfm.__file__), "bin", "cg")
    out = subprocess.run([binary, "-v", str(version), "-s", "-problem", "poisson", "-grid", str(g), "-tol", "1e-8"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    its, rs = map(int, re.search(r"Iterations: (\d+), restarts: (\d+)", out.stdout).groups())
    assert st_o == 0 and (its, rs) == (it_o, rs_o)
    assert rs == (1 if method == "pipelined" else 0)
    assert "1 launches" in out.stdout
