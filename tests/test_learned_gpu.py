"""The learned preconditioner end to end on the GPU: training pairs from
plain CG, training on the tensor cores, and flexible PCG in one device-side
loop.  The ablation: on a held-out system the trained network inside the
hybrid preconditioner needs fewer FPCG iterations than the same
preconditioner without it (Jacobi smoothing alone) and far fewer than plain
CG, and every solve reaches an FP64 true relative residual of 1e-8 with the
plain-CG solution's accuracy."""
import numpy as np
import pytest

import cfm

pytestmark = pytest.mark.gpu

N = 256
SMOOTH = 4


@pytest.fixture(scope="module")
def trained():
    net = cfm.UNet(N, N, max_batch=8, seed=11)
    info = net.train_varcoef(16, 9, 5000, 6, 8, 1e-3, smooth=SMOOTH)
    return net, info


@pytest.fixture(scope="module")
def system():
    k, f = cfm.varcoef_problem((N, N), 77)  # seed outside the training seeds
    return k, f, cfm.Stencil(k)


def test_training_reduces_loss(trained):
    _, info = trained
    assert info["loss_last"] < 0.8 * info["loss_first"], info


def test_identity_fpcg_is_plain_cg(system):
    """With no network and no smoothing the device loop is CG itself."""
    k, f, S = system
    _, st_cg = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-8).solve(f.ravel())
    x, st = cfm.FPCG(S, k, None, maxiter=50000, tol=1e-8, smooth=0).solve(f)
    assert st.refinements == 0 and st.residual <= 1e-8
    assert abs(st.iterations - st_cg.iterations) <= 0.05 * st_cg.iterations


def test_learned_preconditioner_ablation(trained, system):
    net, _ = trained
    k, f, S = system
    xs, st_cg = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-8).solve(f.ravel())
    x_j, st_j = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=SMOOTH).solve(f)
    fp = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8)
    x_n, st_n = fp.solve(f)
    h = fp.history()
    print(f"plain CG {st_cg.iterations} it; Jacobi-smoothed FPCG {st_j.iterations} it; "
          f"learned FPCG {st_n.iterations} it ({st_n.seconds * 1e3:.1f} ms)")
    for st in (st_j, st_n):
        assert st.status == cfm.OK and st.refinements == 0 and st.residual <= 1e-8
    assert st_n.iterations < 0.8 * st_j.iterations
    assert st_n.iterations < 0.1 * st_cg.iterations
    assert len(h) == st_n.iterations + 1 and h[-1] <= 1e-8 * np.linalg.norm(f)
    for x in (x_j, x_n):  # errors bounded like plain CG's (same residual target)
        assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-5


def test_fpcg_rejects_mismatched_smoothing(trained, system):
    net, _ = trained
    k, f, S = system
    with pytest.raises(cfm.CfmError):
        cfm.FPCG(S, k, net, smooth=SMOOTH + 1)


# ------------------------------------------- the two-level (coarse) network
NC = 512


@pytest.fixture(scope="module")
def coarse_trained():
    """A (NC/2)^2 network trained on plain-CG pairs of NC^2 systems: it sees
    the 2x-restricted residual and its output is prolongated."""
    net = cfm.UNet(NC // 2, NC // 2, max_batch=8, seed=5)
    info = net.train_varcoef(24, 9, 7000, 8, 8, 1e-3, smooth=SMOOTH, coarsen=2)
    return net, info


def test_coarse_network_preconditioner(coarse_trained):
    net, info = coarse_trained
    assert info["loss_last"] < info["loss_first"], info
    k, f = cfm.varcoef_problem((NC, NC), 78)
    S = cfm.Stencil(k)
    xs, st_cg = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-8).solve(f.ravel())
    _, st_j = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=SMOOTH).solve(f)
    x_n, st_n = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8).solve(f)  # FCG(8) by default
    print(f"plain CG {st_cg.iterations} it; Jacobi FPCG {st_j.iterations} it; "
          f"coarse learned FCG(8) {st_n.iterations} it ({st_n.seconds * 1e3:.1f} ms)")
    assert st_n.status == cfm.OK and st_n.refinements == 0 and st_n.residual <= 1e-8
    assert st_n.iterations < 0.85 * st_j.iterations
    assert np.linalg.norm(x_n - xs) / np.linalg.norm(xs) < 1e-5


def test_truncation_choices_converge(coarse_trained):
    """Every truncation reaches the tolerance and m can be changed between
    solves; the one-term recurrence may stall with the nonlinear network
    (the plain-CG fallback then finishes), the default FCG(8) does not."""
    net, _ = coarse_trained
    k, f = cfm.varcoef_problem((NC, NC), 79)
    S = cfm.Stencil(k)
    fp = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8)
    for m in (1, 2, 8):
        cfm.check("cfm_fpcg_set_truncation", cfm.lib.cfm_fpcg_set_truncation(fp.h, m))
        _, st = fp.solve(f)
        assert st.status == cfm.OK and st.residual <= 1e-8, m
        if m == 8:
            assert st.refinements == 0
    with pytest.raises(cfm.CfmError):
        cfm.check("cfm_fpcg_set_truncation", cfm.lib.cfm_fpcg_set_truncation(fp.h, 9))


def test_coarse_network_grid_must_match(coarse_trained):
    net, _ = coarse_trained
    k, _ = cfm.varcoef_problem((NC // 2, NC // 2), 1)
    with pytest.raises(cfm.CfmError):
        cfm.FPCG(cfm.Stencil(k), k, net)  # a factor-2 net needs the 2x grid


def test_restored_network_needs_training_info(coarse_trained):
    """Parameters saved from one net and restored into another give the same
    solve once the restored net is told what it was trained for."""
    net, _ = coarse_trained
    k, f = cfm.varcoef_problem((NC, NC), 80)
    S = cfm.Stencil(k)
    twin = cfm.UNet(NC // 2, NC // 2, max_batch=1, seed=99)
    twin.set_params(net.params())
    with pytest.raises(cfm.CfmError):
        cfm.FPCG(S, k, twin)  # not yet told its smoothing and coarsening
    twin.set_training_info(SMOOTH, 2)
    _, st_a = cfm.FPCG(S, k, net, maxiter=20000, tol=1e-8).solve(f)
    _, st_b = cfm.FPCG(S, k, twin, maxiter=20000, tol=1e-8).solve(f)
    assert st_b.status == cfm.OK and st_b.iterations == st_a.iterations


def test_validation_keeps_a_checkpoint():
    """Checkpoint selection: with a held-out system every 2 epochs, training
    keeps the parameters of an evaluated checkpoint (epoch 2 or 4) and
    reports its FPCG time; the kept network still solves that system."""
    net = cfm.UNet(64, 256, max_batch=4, seed=3)
    assert net.validation() == (-1, 0.0)
    net.set_validation(1000, 2)
    net.train_varcoef(6, 3, 40, 4, 4, 1e-3, smooth=4, coarsen=2)
    ep, ms = net.validation()
    assert ep in (2, 4) and ms > 0
    k, f = cfm.varcoef_problem((128, 512), 1000)
    x, st = cfm.FPCG(cfm.Stencil(k), k, net, maxiter=20000, tol=1e-8).solve(f)
    assert st.status == cfm.OK and st.residual <= 1e-8
    net.set_validation(0, 0)
    net.train_varcoef(6, 3, 40, 2, 4, 1e-3, smooth=4, coarsen=2)
    assert net.validation()[0] == -1


def test_training_is_deterministic():
    """Two trainings from the same seeds give bit-identical parameters, the
    same losses, the same kept checkpoint and the same FPCG iteration count:
    the weight gradients (tensor-core and thin layers), bias gradients, loss
    sums and training-data scalings all add their partial sums in a fixed
    order, and the checkpoint is chosen by iteration count."""
    runs = []
    for _ in range(2):
        net = cfm.UNet(64, 256, max_batch=4, seed=3)
        net.set_validation(1000, 1)
        info = net.train_varcoef(6, 3, 40, 3, 4, 1e-3, smooth=4, coarsen=2)
        k, f = cfm.varcoef_problem((128, 512), 1001)
        _, st = cfm.FPCG(cfm.Stencil(k), k, net, maxiter=20000, tol=1e-8).solve(f)
        runs.append((net.params(), info["loss_first"], info["loss_last"], net.validation()[0],
                     st.iterations, st.residual))
        net.close()
    a, b = runs
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1:] == b[1:]
