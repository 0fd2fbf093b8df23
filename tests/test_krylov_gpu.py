"""Persistent Krylov solvers on the GPU through the C ABI, against the oracle:
the matrix-free variable-coefficient stencil operator and every solver
(host-controlled, standard persistent, pipelined persistent, FP32 with
FP64 reliable updates) on CSR and stencil operators give the oracle's x, iteration
count and status bit for bit (same reduction trees, same rounding)."""
import numpy as np
import pytest

import cfm
import oracle

pytestmark = pytest.mark.gpu

METHOD = {cfm.CG_DISCRETE: oracle.STD, cfm.CG_PERSISTENT: oracle.STD,
          cfm.CG_PERSISTENT_PIPELINED: oracle.PIPELINED, cfm.CG_MIXED: oracle.MIXED}
IMPLS = list(METHOD)


def grid_of(shape):
    if len(shape) == 2:
        return 2, (shape[1], shape[0], 1)
    return 3, (shape[2], shape[1], shape[0])


@pytest.mark.parametrize("shape", [(1, 5), (7, 9), (64, 64), (100, 37), (3, 4, 5), (17, 12, 9)])
def test_stencil_apply_bitexact(shape):
    k = np.exp(np.random.default_rng(2).normal(size=shape))
    S = cfm.Stencil(k)
    x = np.random.default_rng(3).uniform(-1, 1, k.size)
    dims, grid = grid_of(shape)
    np.testing.assert_array_equal(S.apply(x), oracle.stencil_apply(dims, grid, cfm.varcoef_coeffs(k), x))


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("shape", [(40, 33), (96, 96), (11, 13, 9), (24, 24, 24)])
def test_stencil_solvers_bitexact(impl, shape):
    k, f = cfm.varcoef_problem(shape, 21)
    S = cfm.Stencil(k)
    dims, grid = grid_of(shape)
    xo, st_o, it_o, rs_o, rr_o = oracle.krylov_stencil(dims, grid, cfm.varcoef_coeffs(k), f,
                                                       METHOD[impl], 20000, 1e-8)
    x, st = cfm.CG(S, impl, 20000, 1e-8).solve(f.ravel())
    assert st_o == 0 and st.status == cfm.OK
    assert st.iterations == it_o and st.refinements == rs_o
    np.testing.assert_array_equal(x, xo)
    assert st.residual <= 1e-8


@pytest.mark.parametrize("impl", [cfm.CG_PERSISTENT_PIPELINED, cfm.CG_MIXED])
@pytest.mark.parametrize("g", [3, 10, 21])
def test_csr_new_solvers_bitexact(impl, g):
    rowptr, col, val = cfm.poisson3d(g)
    A = cfm.CSR(rowptr, col, val)
    b = A.spmv(cfm.uniform(4, A.n))
    xo, st_o, it_o, rs_o, _ = oracle.krylov_csr(rowptr, col, val, b, METHOD[impl], 20000, 1e-8)
    x, st = cfm.CG(A, impl, 20000, 1e-8).solve(b)
    assert st_o == 0 and st.status == cfm.OK
    assert st.iterations == it_o and st.refinements == rs_o
    np.testing.assert_array_equal(x, xo)


def banded_spd(n, seed):
    """Symmetric, diagonally dominant band matrix whose half-bandwidth steps
    through 1..5 every 40 rows: row lengths 2..11, similar within a slice."""
    rng = np.random.default_rng(seed)
    h = 1 + (np.arange(n) // 40) % 5
    rows = [[] for _ in range(n)]
    for i in range(n):
        for j in range(i + 1, min(n, i + h[i] + 1)):
            v = -rng.uniform(0.1, 1.0)
            rows[i].append((j, v))
            rows[j].append((i, v))
    rowptr, col, val = [0], [], []
    for i in range(n):
        ent = sorted(rows[i] + [(i, 1.0 - sum(v for _, v in rows[i]))])
        col += [c for c, _ in ent]
        val += [v for _, v in ent]
        rowptr.append(len(col))
    return np.array(rowptr, np.int32), np.array(col, np.int32), np.array(val)


def arrow_spd(n):
    """Row and column 0 full (-1), tridiagonal -1 elsewhere: one row n
    entries long among rows of 2 and 3."""
    rowptr, col, val = [0], [], []
    for i in range(n):
        ent = {0: -1.0} if i else {j: -1.0 for j in range(n)}
        if i > 1:
            ent[i - 1] = -1.0
        if 0 < i < n - 1:
            ent[i + 1] = -1.0
        ent[i] = 2.0 * n if i == 0 else 4.0
        for c in sorted(ent):
            col.append(c)
            val.append(ent[c])
        rowptr.append(len(col))
    return np.array(rowptr, np.int32), np.array(col, np.int32), np.array(val)


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("kind", ["banded", "arrow", "poisson"])
def test_csr_uneven_rows_bitexact(impl, kind):
    """Uneven rows (2..11 entries, or one full row), n not a multiple of 32:
    every solver gives the oracle's SpMV, x, iteration count and
    refinements bit for bit."""
    rowptr, col, val = {"banded": lambda: banded_spd(1007, 5), "arrow": lambda: arrow_spd(301),
                        "poisson": lambda: cfm.poisson3d(11)}[kind]()
    A = cfm.CSR(rowptr, col, val)
    xs = cfm.uniform(6, A.n)
    np.testing.assert_array_equal(A.spmv(xs), oracle.spmv(rowptr, col, val, xs))
    b = oracle.spmv(rowptr, col, val, xs)
    xo, st_o, it_o, rs_o, _ = oracle.krylov_csr(rowptr, col, val, b, METHOD[impl], 20000, 1e-8)
    x, st = cfm.CG(A, impl, 20000, 1e-8).solve(b)
    assert st_o == 0 and st.status == cfm.OK
    assert st.iterations == it_o and st.refinements == rs_o
    np.testing.assert_array_equal(x, xo)


def test_pipelined_fixed_count_reference_mode():
    """-niter semantics: exactly maxiter pipelined iterations, b = ones."""
    rowptr, col, val = cfm.tridiag(3000)
    A = cfm.CSR(rowptr, col, val)
    xo, _, it_o, _, _ = oracle.krylov_csr(rowptr, col, val, None, oracle.PIPELINED, 30, 0.0)
    x, st = cfm.CG(A, cfm.CG_PERSISTENT_PIPELINED, 30, 0.0).solve(None)
    assert st.iterations == it_o == 30
    np.testing.assert_array_equal(x, xo)


def test_mixed_inner_parameters_and_launch_count():
    k, f = cfm.varcoef_problem((64, 48), 2)
    S = cfm.Stencil(k)
    c = cfm.varcoef_coeffs(k)
    xo, _, it_o, rs_o, _ = oracle.krylov_stencil(2, (48, 64, 1), c, f, oracle.MIXED, 20000, 1e-10,
                                                 inner_maxiter=25, inner_tol=1e-3)
    x, st = cfm.CG(S, cfm.CG_MIXED, 20000, 1e-10, inner_maxiter=25, inner_tol=1e-3).solve(f.ravel())
    assert st.status == cfm.OK and st.launches == 1
    assert (st.iterations, st.refinements) == (it_o, rs_o) and rs_o > 2
    np.testing.assert_array_equal(x, xo)


@pytest.mark.parametrize("maxiter", [1, 7, 30])
def test_mixed_iteration_cap_folds_the_correction(maxiter):
    """A cap below convergence: the FP32 steps taken so far are folded into
    x by a last FP64 update; x, the count and the updates equal the
    oracle's, and the status is NOT_CONVERGED."""
    rowptr, col, val = cfm.poisson3d(12)
    A = cfm.CSR(rowptr, col, val)
    b = A.spmv(cfm.uniform(9, A.n))
    xo, st_o, it_o, rs_o, _ = oracle.krylov_csr(rowptr, col, val, b, oracle.MIXED, maxiter, 1e-10)
    x, st = cfm.CG(A, cfm.CG_MIXED, maxiter, 1e-10).solve(b, allowed=(cfm.NOT_CONVERGED,))
    assert st_o == cfm.NOT_CONVERGED and st.status == cfm.NOT_CONVERGED
    assert st.iterations == it_o == maxiter and st.refinements == rs_o
    np.testing.assert_array_equal(x, xo)
    assert np.abs(x).max() > 0


@pytest.mark.parametrize("delta", [0.5, 0.1, 1e-3])
def test_mixed_update_threshold_bitexact(delta):
    """The reliable-update threshold changes when the FP64 updates happen
    (more of them for a larger delta); every setting equals the oracle and
    reaches the FP64 tolerance."""
    k, f = cfm.varcoef_problem((40, 56), 4)
    S = cfm.Stencil(k)
    xo, st_o, it_o, rs_o, _ = oracle.krylov_stencil(2, (56, 40, 1), cfm.varcoef_coeffs(k), f, oracle.MIXED,
                                                    20000, 1e-9, inner_tol=delta)
    x, st = cfm.CG(S, cfm.CG_MIXED, 20000, 1e-9, inner_tol=delta).solve(f.ravel())
    assert st_o == 0 and st.status == cfm.OK and st.residual <= 1e-9
    assert (st.iterations, st.refinements) == (it_o, rs_o)
    np.testing.assert_array_equal(x, xo)


def test_config4_varcoef_512_plain_and_pipelined_persistent():
    """The 512^2 variable-coefficient system (k = exp(GRF), f ~ N(0,1)) to
    1e-8: standard and pipelined persistent CG match the oracle exactly."""
    k, f = cfm.varcoef_problem((512, 512), 0)
    S = cfm.Stencil(k)
    c = cfm.varcoef_coeffs(k)
    for impl in (cfm.CG_PERSISTENT, cfm.CG_PERSISTENT_PIPELINED, cfm.CG_MIXED):
        xo, st_o, it_o, rs_o, rr_o = oracle.krylov_stencil(2, (512, 512, 1), c, f, METHOD[impl],
                                                           20000, 1e-8)
        x, st = cfm.CG(S, impl, 20000, 1e-8).solve(f.ravel())
        assert st_o == 0 and st.status == cfm.OK and st.launches == 1
        assert st.iterations == it_o
        np.testing.assert_array_equal(x, xo)
        assert st.residual <= 1e-8


def test_config3_poisson128_mixed_reaches_fp64_tolerance():
    """128^3 Poisson CSR, FP32 inner / FP64 refinement to a true relative
    residual of 1e-8, error against the FP64 oracle solution stated."""
    rowptr, col, val = cfm.poisson3d(128)
    A = cfm.CSR(rowptr, col, val)
    xs = cfm.uniform(0, A.n)
    b = A.spmv(xs)
    x64, st64 = cfm.CG(A, cfm.CG_PERSISTENT, 20000, 1e-8).solve(b)
    x, st = cfm.CG(A, cfm.CG_MIXED, 20000, 1e-8).solve(b)
    assert st.status == cfm.OK and st.residual <= 1e-8
    # both stop at a relative residual of 1e-8; their errors against x* are
    # bounded by cond(A) * 1e-8 (cond ~ 6.6e3 here) and must be alike
    err64 = np.linalg.norm(x64 - xs) / np.linalg.norm(xs)
    err = np.linalg.norm(x - xs) / np.linalg.norm(xs)
    assert err < 1e-5 and err < 3 * err64 + 1e-7, (err, err64)
    assert st.refinements >= 2
