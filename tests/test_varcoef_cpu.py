"""Variable-coefficient problem, its operator and the oracle's persistent-
solver restatements, on the CPU: the generators have the stated statistics,
the stencil coefficients equal an independent SciPy assembly of the
harmonic-mean finite-volume matrix, and every oracle method solves the
systems it is given."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import cfm
import oracle


def fv_matrix(k):
    """-div(k grad u), unit cells, u = 0 on the boundary (boundary faces 2 k_i),
    interior faces 2 k_i k_j / (k_i + k_j); assembled independently with SciPy."""
    shape = k.shape
    n = k.size
    idx = np.arange(n).reshape(shape)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for ax in range(k.ndim):
        lo = [slice(None)] * k.ndim
        hi = [slice(None)] * k.ndim
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        ka, kb = k[tuple(lo)], k[tuple(hi)]
        w = (2 * ka * kb / (ka + kb)).ravel()
        ia, ib = idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()
        rows += [ia, ib]
        cols += [ib, ia]
        vals += [-w, -w]
        np.add.at(diag, ia, w)
        np.add.at(diag, ib, w)
        for end in (0, -1):
            face = [slice(None)] * k.ndim
            face[ax] = end
            np.add.at(diag, idx[tuple(face)].ravel(), 2 * k[tuple(face)].ravel())
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def shape_args(shape):
    if len(shape) == 2:
        return 2, (shape[1], shape[0], 1)
    return 3, (shape[2], shape[1], shape[0])


def test_normal_statistics_and_determinism():
    z = cfm.normal(7, 100001)
    assert abs(z.mean()) < 0.01 and abs(z.var() - 1) < 0.01
    assert abs((z ** 4).mean() - 3) < 0.05
    np.testing.assert_array_equal(z, cfm.normal(7, 100001))
    assert not np.array_equal(z[:1000], cfm.normal(7, 1000, stream=1))


def test_grf_unit_variance_and_gaussian_covariance():
    v, c16 = [], []
    for s in range(4):
        g = cfm.grf((384, 384), s)
        v.append(g.var())
        c16.append(np.mean(g * np.roll(g, 16, 1)))
    assert abs(np.mean(v) - 1) < 0.1
    assert abs(np.mean(c16) - np.exp(-0.5)) < 0.06
    g3 = cfm.grf((40, 48, 56), 1, sigma=2.0, corr_len=4.0)
    assert abs(g3.var() - 4) < 0.6


def test_varcoef_problem_is_lognormal_k_and_normal_f():
    k, f = cfm.varcoef_problem((128, 96), 11)
    assert k.shape == f.shape == (128, 96) and (k > 0).all()
    k2, f2 = cfm.varcoef_problem((128, 96), 11)
    np.testing.assert_array_equal(k, k2)
    np.testing.assert_array_equal(f, f2)
    np.testing.assert_allclose(np.log(k), cfm.grf((128, 96), 11), rtol=0, atol=1e-14)


@pytest.mark.parametrize("shape", [(9, 13), (1, 7), (64, 64), (5, 6, 7), (12, 9, 10)])
def test_stencil_coefficients_match_scipy_assembly(shape):
    k = np.exp(np.random.default_rng(len(shape)).normal(size=shape))
    A = fv_matrix(k)
    dims, grid = shape_args(shape)
    c = cfm.varcoef_coeffs(k)
    x = np.random.default_rng(1).uniform(-1, 1, k.size)
    y = oracle.stencil_apply(dims, grid, c, x)
    ref = A @ x
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    np.testing.assert_allclose(c[3], A.diagonal(), rtol=1e-15, atol=0)
    assert abs(A - A.T).max() == 0


@pytest.mark.parametrize("method", [oracle.STD, oracle.PIPELINED, oracle.MIXED])
@pytest.mark.parametrize("shape", [(48, 40), (14, 12, 10)])
def test_oracle_methods_solve_varcoef(method, shape):
    k, f = cfm.varcoef_problem(shape, 5)
    dims, grid = shape_args(shape)
    c = cfm.varcoef_coeffs(k)
    x, st, it, rs, rr = oracle.krylov_stencil(dims, grid, c, f, method, 20000, 1e-8)
    assert st == 0 and rr <= 1e-8 and it > 0
    xs = spla.spsolve(fv_matrix(k).tocsc(), f.ravel())
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
    if method == oracle.MIXED:
        assert rs >= 2  # FP64 reliable updates


def test_oracle_std_csr_equals_reference_restatement():
    """Method 0 on CSR is the same arithmetic as orc_cg (the restatement of
    CG/src/common.cu:399-538)."""
    rowptr, col, val = cfm.poisson3d(9)
    b = np.linspace(-1, 2, len(rowptr) - 1)
    x0, st0, it0, rr0 = oracle.cg(rowptr, col, val, b, 2000, 1e-10)
    x1, st1, it1, _, rr1 = oracle.krylov_csr(rowptr, col, val, b, oracle.STD, 2000, 1e-10)
    assert st0 == st1 == 0 and it0 == it1
    np.testing.assert_array_equal(x0, x1)
    x0, _, _, _ = oracle.cg(rowptr, col, val, None, 17, 0.0)
    x1, _, it1, _, _ = oracle.krylov_csr(rowptr, col, val, None, oracle.STD, 17, 0.0)
    assert it1 == 17
    np.testing.assert_array_equal(x0, x1)


def test_oracle_pipelined_fixed_count_matches_standard_in_exact_arithmetic():
    """Pipelined CG is CG: after a few steps both iterates agree closely (the
    reference's recurrence restarts once, at its second step)."""
    rowptr, col, val = cfm.poisson3d(8)
    b = np.ones(len(rowptr) - 1)
    xs, *_ = oracle.krylov_csr(rowptr, col, val, b, oracle.STD, 200, 1e-12)
    xp, st, it, _, rr = oracle.krylov_csr(rowptr, col, val, b, oracle.PIPELINED, 200, 1e-12)
    assert st == 0 and rr <= 1e-12
    assert np.linalg.norm(xs - xp) / np.linalg.norm(xs) < 1e-10
