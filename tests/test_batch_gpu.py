"""Batched uneven solves in one persistent launch: every system reaches its
FP64 true relative residual target, iteration counts and solutions match a
single-system solve with the same preconditioner (FPCG with the same
Jacobi polynomial on 2D members), the class plan and the autotuner keep
results unchanged, and the launch is one graph."""
import numpy as np
import pytest

import cfm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    systems = cfm.uneven_systems(24, 8, seed=3, side2d=(16, 160), side3d=(8, 40))
    return systems, cfm.Batch(systems)


def test_batch_converges_every_system(batch):
    systems, B = batch
    B.set_solver(smooth=4, maxiter=20000, tol=1e-8)
    it, stt, rr, st = B.solve()
    assert (stt == cfm.OK).all() and (rr <= 1e-8 * 1.5).all(), rr.max()
    assert st.launches == 2 and st.iterations == it.sum()
    # solutions agree with plain CG on the same system
    for i in (0, 5, len(systems) - 1):
        k, f = systems[i]
        x = B.solution(i)
        xs, sts = cfm.CG(cfm.Stencil(k), cfm.CG_PERSISTENT, 50000, 1e-10).solve(f.ravel())
        assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-5


def test_polynomial_preconditioner_beats_diagonal(batch):
    """The Jacobi-polynomial preconditioner (4 sweeps) needs fewer
    iterations than diagonal scaling on every member of the batch."""
    systems, B = batch
    B.set_solver(smooth=0, maxiter=50000, tol=1e-8)
    it0, stt0, rr0, _ = B.solve()
    B.set_solver(smooth=4, maxiter=50000, tol=1e-8)
    it4, stt4, rr4, _ = B.solve()
    assert (stt0 == cfm.OK).all() and (stt4 == cfm.OK).all()
    assert (it4 < it0).all()  # the polynomial preconditioner needs fewer iterations


def test_plans_and_autotune_do_not_change_results(batch):
    systems, B = batch
    B.set_solver(smooth=2, maxiter=20000, tol=1e-9)
    B.set_plan([1 << 12, 0], [4, 1])
    itA, _, rrA, _ = B.solve()
    xA = B.solution(3)
    B.set_plan([1 << 14, 1 << 10, 0], [8, 2, 1])
    itB, _, rrB, _ = B.solve()
    np.testing.assert_array_equal(itA, itB)  # fixed reduction order per system
    np.testing.assert_array_equal(xA, B.solution(3))
    ms = B.autotune()
    itC, _, _, st = B.solve()
    np.testing.assert_array_equal(itA, itC)
    assert ms > 0


def test_mixed_precision_batch_reaches_fp64_tolerance(batch):
    """FP32 PCG with FP64 reliable updates, in the same persistent launch:
    every system reaches the FP64 true relative residual target, each needs
    at least one update, the iteration counts stay within 25% of FP64 PCG
    (the search direction survives the updates) and the solutions agree with
    the FP64 batch to the tolerance's order."""
    systems, B = batch
    B.set_solver(smooth=4, maxiter=20000, tol=1e-8)
    B.set_precision(cfm.FP64)
    it64, stt64, rr64, _ = B.solve()
    x64 = [B.solution(i) for i in range(len(systems))]
    B.set_precision(cfm.FP32, 0, 0.1)
    it, stt, rr, st = B.solve()
    assert (stt == cfm.OK).all() and (rr <= 1e-8).all(), rr.max()
    assert st.refinements >= len(systems) and st.iterations == it.sum()
    assert it.sum() <= 1.25 * it64.sum(), (it.sum(), it64.sum())
    for i in range(len(systems)):
        x = B.solution(i)
        assert np.linalg.norm(x - x64[i]) / np.linalg.norm(x64[i]) < 1e-6
    # back to FP64: the same iterations and solutions as before, bit for bit
    B.set_precision(cfm.FP64)
    itB, _, _, stB = B.solve()
    np.testing.assert_array_equal(itB, it64)
    np.testing.assert_array_equal(B.solution(2), x64[2])
    assert stB.refinements == 0


def test_mixed_precision_plan_independent_and_inner_cap(batch):
    systems, B = batch
    B.set_solver(smooth=2, maxiter=20000, tol=1e-8)
    B.set_precision(cfm.FP32, 0, 0.1)
    B.set_plan([1 << 12, 0], [4, 1])
    itA, sttA, _, stA = B.solve()
    xA = B.solution(5)
    B.set_plan([1 << 14, 1 << 10, 0], [8, 2, 1])
    itB, _, _, stB = B.solve()
    np.testing.assert_array_equal(itA, itB)
    np.testing.assert_array_equal(xA, B.solution(5))
    assert stA.refinements == stB.refinements
    # an update at least every 5 steps still converges, with more updates
    B.set_precision(cfm.FP32, 5, 0.1)
    itC, sttC, rrC, stC = B.solve()
    assert (sttC == cfm.OK).all() and (rrC <= 1e-8).all()
    assert stC.refinements >= itC.sum() // 5 and stC.refinements > stA.refinements
    B.set_precision(cfm.FP64)
    with pytest.raises(cfm.CfmError):
        B.set_precision(7)


def test_mixed_precision_iteration_cap(batch):
    """maxiter below convergence: every unconverged system stops at the cap
    with NOT_CONVERGED, its FP32 steps folded into x by a last FP64 update
    (the true residual is below |b|), in both precisions."""
    systems, B = batch
    for prec in (cfm.FP32, cfm.FP64):
        B.set_precision(prec, 0, 0.1)
        B.set_solver(smooth=4, maxiter=12, tol=1e-12)
        it, stt, rr, st = B.solve(allowed=(cfm.OK, cfm.NOT_CONVERGED))
        assert (stt == cfm.NOT_CONVERGED).all() and (it == 12).all()
        assert np.isfinite(rr).all() and (rr < 1.0).all()
        assert all(np.abs(B.solution(i)).max() > 0 for i in (0, 9, len(systems) - 1))
        if prec == cfm.FP32:
            assert st.refinements >= len(systems)
    B.set_precision(cfm.FP64)
    B.set_solver(smooth=4, maxiter=20000, tol=1e-8)
