"""The CPU oracle against independent restatements (numpy, SciPy) and against
the reference's own outputs (golden fixtures).  No GPU needed."""
import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
from conftest import GOLDEN, ref_cg_fixtures, ref_cg_system


# ---------------------------------------------------------------- numpy restatements
def np_jacobi2d(a, niter):
    """Vectorised single_gpu() (Stencil/jacobi2D/src/common.cu:154-273)."""
    a = a.copy()
    b = a.copy()
    q = 0.25 if a.dtype == np.float64 else np.float32(0.25)
    for _ in range(niter):
        s = a[1:-1, 2:] + a[1:-1, :-2]
        s = s + a[2:, 1:-1]
        s = s + a[:-2, 1:-1]
        b[1:-1, 1:-1] = q * s
        b[0, :] = b[-2, :]
        b[-1, :] = b[1, :]
        a, b = b, a
    return a


def np_jacobi3d(a, niter, periodic_y):
    """Vectorised 3D single_gpu() (Stencil/jacobi3D/src/common.cu:110-239)."""
    a = a.copy()
    b = a.copy()
    c6 = a.dtype.type(1) / a.dtype.type(6)
    for _ in range(niter):
        s = a[1:-1, 1:-1, 2:] + a[1:-1, 1:-1, :-2]
        s = s + a[1:-1, 2:, 1:-1]
        s = s + a[1:-1, :-2, 1:-1]
        s = s + a[2:, 1:-1, 1:-1]
        s = s + a[:-2, 1:-1, 1:-1]
        b[1:-1, 1:-1, 1:-1] = c6 * s
        if periodic_y:
            b[1:-1, 0, :] = b[1:-1, -2, :]
            b[1:-1, -1, :] = b[1:-1, 1, :]
        b[0] = b[-2]
        b[-1] = b[1]
        a, b = b, a
    return a


def rand_grid(shape, dtype, seed):
    return np.random.default_rng(seed).uniform(-1, 1, shape).astype(dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("shape,niter", [((3, 3), 1), ((9, 7), 5), ((17, 33), 11), ((40, 24), 0)])
def test_oracle_jacobi2d_matches_numpy(dtype, shape, niter):
    a = rand_grid(shape, dtype, 1)
    np.testing.assert_array_equal(oracle.jacobi2d(a, niter), np_jacobi2d(a, niter))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("periodic_y", [0, 1])
@pytest.mark.parametrize("shape,niter", [((3, 3, 3), 2), ((5, 6, 7), 4), ((9, 17, 12), 9)])
def test_oracle_jacobi3d_matches_numpy(dtype, periodic_y, shape, niter):
    a = rand_grid(shape, dtype, 2)
    np.testing.assert_array_equal(oracle.jacobi3d(a, niter, periodic_y),
                                  np_jacobi3d(a, niter, periodic_y))


def test_oracle_thread_count_does_not_change_results():
    a = rand_grid((20, 30, 40), np.float64, 3)
    np.testing.assert_array_equal(oracle.jacobi3d(a, 6, 1, threads=1), oracle.jacobi3d(a, 6, 1, threads=7))


def test_oracle_mirror_matches_numpy():
    a = rand_grid((12, 64), np.float32, 4)
    ref = a.copy()
    b = a.copy()
    for _ in range(5):
        e = np.concatenate([ref[1:-1, 1:], ref[1:-1, -1:]], axis=1)
        w = np.concatenate([ref[1:-1, :1], ref[1:-1, :-1]], axis=1)
        s = ref[2:, :] + ref[:-2, :]
        s = s + e
        s = s + w
        b[1:-1, :] = np.float32(0.25) * s
        b[0] = b[-2]
        b[-1] = b[1]
        ref, b = b, ref
    np.testing.assert_array_equal(oracle.jacobi2d_mirror(a, 5), ref)


def test_oracle_init_3d_reference_quirk():
    # x = 0 face is z - y - (nx - 1) (last write of the ix loop), x = nx-1 face 0
    a = oracle.jacobi3d_init(6, 5, 4, 0, np.float32)
    z, y = np.meshgrid(np.arange(4), np.arange(5), indexing="ij")
    np.testing.assert_array_equal(a[:, :, 0], (z - y - 5).astype(np.float32))
    assert not a[:, :, 1:].any()


def test_oracle_init_config():
    nx, ny, nz = 7, 9, 11
    a = oracle.jacobi3d_init(nx, ny, nz, 1, np.float64)
    f = np.outer(np.sin(2 * np.pi * np.arange(nz) / (nz - 1)), np.sin(2 * np.pi * np.arange(ny) / (ny - 1)))
    np.testing.assert_allclose(a[:, :, 0], f, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(a[:, :, 0], a[:, :, -1])
    assert not a[:, :, 1:-1].any()
    b = oracle.jacobi2d_init(8, 10, np.float64)
    np.testing.assert_allclose(b[:, 0], np.sin(2 * np.pi * np.arange(10) / 9), atol=1e-15)


# ------------------------------------------------------------- reference fixtures
def _fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_jacobi*.npz")))


def test_reference_fixtures_present():
    assert _fixtures(), "tests/golden/ref_jacobi*.npz missing (made by tests/golden/make_ref_fixtures.py)"


@pytest.mark.parametrize("path", _fixtures(), ids=os.path.basename)
def test_oracle_matches_reference_run(path):
    """Pin: the oracle reproduces grids written by the reference's own
    single_gpu() bit-for-bit (FP32, reference initial state)."""
    f = np.load(path)
    out = f["out"]
    niter = int(f["niter"])
    kind = str(f["kind"])
    if kind == "2d":
        ny, nx = out.shape
        a = oracle.jacobi2d_init(nx, ny, np.float32)
        # the boundary columns were computed by the reference with device sin;
        # they are never changed by a sweep, so the output carries them
        np.testing.assert_array_equal(a[1:-1, 0], out[1:-1, 0])
        np.testing.assert_array_equal(oracle.jacobi2d(a, niter), out)
    elif kind == "2d_mirror":
        ny, nx = out.shape
        a = oracle.jacobi2d_init(nx, ny, np.float32)
        np.testing.assert_array_equal(oracle.jacobi2d_mirror(a, niter), out)
    else:
        nz, ny, nx = out.shape
        a = oracle.jacobi3d_init(nx, ny, nz, 0, np.float32)
        np.testing.assert_array_equal(oracle.jacobi3d(a, niter, 0), out)


# -------------------------------------------------------------------------- CG
def poisson_scipy(g):
    one = sp.diags([-1.0, 2.0, -1.0], [-1, 0, 1], shape=(g, g))
    eye = sp.identity(g)
    lap = (sp.kron(sp.kron(eye, eye), one) + sp.kron(sp.kron(eye, one), eye) +
           sp.kron(sp.kron(one, eye), eye)).tocsr()
    lap.sum_duplicates()
    lap.eliminate_zeros()
    lap.sort_indices()
    return lap


def test_oracle_dot_close_to_numpy():
    rng = np.random.default_rng(5)
    for n in (1, 31, 1024, 1025, 5000, 100003):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        d = oracle.dot(a, b)
        assert abs(d - np.dot(a, b)) <= 1e-12 * np.sum(np.abs(a * b))


def test_oracle_spmv_matches_scipy():
    A = poisson_scipy(6)
    x = np.random.default_rng(6).uniform(-1, 1, A.shape[0])
    y = oracle.spmv(A.indptr, A.indices, A.data, x)
    np.testing.assert_allclose(y, A @ x, rtol=0, atol=1e-13)
    # 1-based CSR gives the same result
    y1 = oracle.spmv(A.indptr + 1, A.indices + 1, A.data, x)
    np.testing.assert_array_equal(y, y1)


@pytest.mark.parametrize("g", [4, 12])
def test_oracle_cg_solves_poisson(g):
    A = poisson_scipy(g)
    xs = np.random.default_rng(g).uniform(-1, 1, A.shape[0])
    b = A @ xs
    x, st, it, rr = oracle.cg(A.indptr, A.indices, A.data, b, 20000, 1e-10)
    assert st == 0 and rr <= 1e-10
    np.testing.assert_allclose(x, xs, rtol=0, atol=1e-8)
    # SciPy's CG on the same system needs about as many iterations
    its = []
    spla.cg(A, b, rtol=1e-10, maxiter=20000, callback=lambda _: its.append(1))
    assert abs(it - len(its)) <= max(2, 0.05 * len(its))


def test_oracle_cg_fixed_count_reference_mode():
    # reference mode: b = ones, fixed iteration count, no tolerance exit
    A = poisson_scipy(5)
    x, st, it, rr = oracle.cg(A.indptr, A.indices, A.data, None, 30, 0.0)
    assert st == 0 and it == 30
    np.testing.assert_allclose(A @ x, np.ones(A.shape[0]), atol=1e-9)


def test_reference_cg_fixtures_present():
    assert len(ref_cg_fixtures()) >= 5, "tests/golden/ref_cg_*.npz missing"


@pytest.mark.parametrize("path", ref_cg_fixtures(), ids=os.path.basename)
def test_oracle_cg_matches_reference_run(path):
    """Pin: the CG restatement agrees with x written by the reference's own
    SingleGPUDiscreteStandard::run_single_gpu() (CG/src/common.cu:399-538;
    b = ones, x0 = 0, a fixed count) to 1e-12 relative.  Not bit for bit: the
    reference sums its dots with atomicAdd(double) in arrival order, the
    oracle in a fixed tree."""
    rowptr, col, val, niter, x_ref = ref_cg_system(path)
    x, st, it, _ = oracle.cg(rowptr, col, val, None, niter, 0.0)
    assert st == 0 and it == niter
    rel = np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref)
    assert rel <= 1e-12, rel


def test_tridiag_generator_matches_reference():
    """cfm_tridiag_csr from libc rand()'s unseeded state is the reference's
    genTridiag (CG/src/common.cu:46-76) bit for bit: the fixtures store the
    matrix the reference generated."""
    import ctypes

    import cfm
    paths = [p for p in ref_cg_fixtures() if "tridiag" in os.path.basename(p)]
    assert paths
    for p in paths:
        f = np.load(p)
        ctypes.CDLL(None).srand(1)
        rowptr, col, val = cfm.tridiag(int(f["size"]))
        np.testing.assert_array_equal(rowptr, f["rowptr"])
        np.testing.assert_array_equal(col, f["col"])
        np.testing.assert_array_equal(val, f["val"])


def test_oracle_cg_breakdown_on_indefinite():
    A = sp.diags([1.0, -1.0, 2.0]).tocsr()
    _, st, _, _ = oracle.cg(A.indptr, A.indices, A.data, np.array([1.0, 1.0, 0.0]), 10, 1e-12)
    assert st == 4


@pytest.mark.parametrize("g", [6, 14])
def test_oracle_mixed_reliable_updates_keep_the_fp64_count(g):
    """The mixed-precision restatement (FP32 CG with FP64 reliable updates)
    keeps the search direction across its updates: on Poisson it needs the
    FP64 iteration count, with several FP64 updates, and its answer meets
    the FP64 true-residual tolerance and SciPy's solution."""
    A = poisson_scipy(g)
    xs = np.random.default_rng(g).uniform(-1, 1, A.shape[0])
    b = A @ xs
    _, st64, it64, _, _ = oracle.krylov_csr(A.indptr, A.indices, A.data, b, oracle.STD, 20000, 1e-9)
    x, st, it, ups, rr = oracle.krylov_csr(A.indptr, A.indices, A.data, b, oracle.MIXED, 20000, 1e-9)
    assert st64 == 0 and st == 0 and rr <= 1e-9
    assert abs(it - it64) <= 1 and ups >= 2
    np.testing.assert_allclose(x, spla.spsolve(A.tocsc(), b), rtol=0, atol=1e-7)


def test_oracle_mixed_independent_of_threads():
    A = poisson_scipy(11)
    b = A @ np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    runs = [oracle.krylov_csr(A.indptr, A.indices, A.data, b, oracle.MIXED, 20000, 1e-9, threads=t)
            for t in (1, 3)]
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    assert runs[0][1:4] == runs[1][1:4]


# ------------------------------------------------------------------ FPCG
def test_oracle_fpcg_restatement_converges_and_mixed_keeps_the_count():
    """The FPCG restatement (identity in place of the network) reaches 1e-8
    and agrees with plain CG's solution; its mixed form (FP32 Krylov
    vectors, FP64 reliable updates) takes about the FP64 form's iterations
    and as accurate a solution."""
    import cfm
    for shape, seed in (((96, 64), 3), ((60, 100), 4)):
        ny, nx = shape
        k, f = cfm.varcoef_problem(shape, seed)
        c = cfm.varcoef_coeffs(k)
        xs, st, its, _, _ = oracle.krylov_stencil(2, (nx, ny, 1), c, f.ravel(), 0, 50000, 1e-11)
        assert st == 0
        x64, it64, up64, d64 = oracle.fpcg2d((nx, ny), c, f, 4, 1, False)
        x32, it32, up32, d32 = oracle.fpcg2d((nx, ny), c, f, 4, 1, True)
        assert d64 == d32 == 1 and up64 == 0 and up32 >= 1
        assert it64 < 0.25 * its  # smoothing + coarse correction beat plain CG
        assert abs(it32 - it64) <= max(2, 0.1 * it64)
        for x in (x64, x32):
            assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
            r = f.ravel() - oracle.stencil_apply(2, (nx, ny, 1), c, x)
            assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(f)


def test_oracle_fpcg_truncation_and_bad_arguments():
    import cfm
    k, f = cfm.varcoef_problem((64, 64), 5)
    c = cfm.varcoef_coeffs(k)
    _, it1, _, _ = oracle.fpcg2d((64, 64), c, f, 2, 1, False)
    _, it8, _, _ = oracle.fpcg2d((64, 64), c, f, 2, 8, False)
    assert it8 <= it1 + 2  # a linear preconditioner: FCG(8) ~ the one-term recurrence
    we, wn, _, dg = (np.ascontiguousarray(a, np.float64) for a in c)
    x = np.empty(64 * 64)
    p = oracle._p
    assert oracle.lib.orc_fpcg2d(64, 64, p(we), p(wn), p(dg), p(np.ascontiguousarray(f.ravel())), 3, 2, 1,
                                 0, 0.1, 100, 1e-8, p(x), None, None, None) == 1  # f must be 1 or 2
