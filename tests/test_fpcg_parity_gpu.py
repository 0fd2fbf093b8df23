"""Flexible PCG parity on the GPU through the C ABI: with the identity in
place of the network (no network given), the device loop -- FP64, or FP32
Krylov vectors with FP64 reliable updates -- reproduces the oracle's
restatement (orc_fpcg2d) bit for bit: the same x, iteration count and
number of reliable updates, for several smoothing depths, truncations and
grid shapes (tiles cut at the edges included).  Then the learned
preconditioner in mixed precision: FP64 true residual 1e-8, plain CG's
accuracy, and about FP64 FPCG's iteration count."""
import numpy as np
import pytest

import cfm
import oracle

pytestmark = pytest.mark.gpu


def system(shape, seed):
    ny, nx = shape
    k, f = cfm.varcoef_problem((ny, nx), seed)
    return k, f, cfm.Stencil(k), cfm.varcoef_coeffs(k)


@pytest.mark.parametrize("shape", [(96, 64), (60, 100), (128, 128)])
@pytest.mark.parametrize("smooth,m", [(4, 1), (2, 3), (0, 1), (4, 8)])
@pytest.mark.parametrize("mixed", [False, True])
def test_fpcg_matches_oracle_bitexact(shape, smooth, m, mixed):
    k, f, S, c = system(shape, 31)
    ny, nx = shape
    x_o, it_o, up_o, done_o = oracle.fpcg2d((nx, ny), c, f, smooth, m, mixed)
    assert done_o == 1
    fp = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=smooth, truncation=m,
                  precision=cfm.FP32 if mixed else None)
    x, st = fp.solve(f)
    assert st.status == cfm.OK and st.refinements == 0 and st.residual <= 1e-8
    assert st.iterations == it_o
    assert fp.reliable_updates() == up_o
    np.testing.assert_array_equal(x, x_o)


def test_mixed_precision_switch_and_repeat():
    """FP64 -> FP32 -> FP64 on one handle: each solve equals the oracle's for
    its precision, and a repeated mixed solve gives the same bits."""
    k, f, S, c = system((96, 160), 32)
    fp = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=4)
    for mixed in (False, True, True, False):
        fp.set_precision(cfm.FP32 if mixed else cfm.FP64)
        x, st = fp.solve(f)
        x_o, it_o, up_o, _ = oracle.fpcg2d((160, 96), c, f, 4, 1, mixed)
        assert st.iterations == it_o and fp.reliable_updates() == up_o
        np.testing.assert_array_equal(x, x_o)
    with pytest.raises(cfm.CfmError):
        fp.set_precision(cfm.FP32, 1.5)


NC = 512


@pytest.fixture(scope="module")
def coarse_net():
    net = cfm.UNet(NC // 2, NC // 2, max_batch=8, seed=5)
    net.train_varcoef(24, 9, 7000, 8, 8, 1e-3, smooth=4, coarsen=2)
    return net


def test_learned_mixed_precision_fpcg(coarse_net):
    """Learned + mixed: the trained coarse network inside FCG(8) with FP32
    Krylov vectors and FP64 reliable updates reaches an FP64 true relative
    residual of 1e-8 without the fallback, agrees with plain FP64 CG's
    solution like the FP64 FPCG does, and needs about its iterations."""
    k, f = cfm.varcoef_problem((NC, NC), 81)
    S = cfm.Stencil(k)
    xs, _ = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-10).solve(f.ravel())
    x64, st64 = cfm.FPCG(S, k, coarse_net, maxiter=20000, tol=1e-8).solve(f)
    fpm = cfm.FPCG(S, k, coarse_net, maxiter=20000, tol=1e-8, precision=cfm.FP32)
    x32, st32 = fpm.solve(f)
    print(f"learned FPCG FP64 {st64.iterations} it {st64.seconds * 1e3:.1f} ms; "
          f"mixed {st32.iterations} it {st32.seconds * 1e3:.1f} ms, {fpm.reliable_updates()} updates")
    assert st32.status == cfm.OK and st32.refinements == 0 and st32.residual <= 1e-8
    assert fpm.reliable_updates() >= 1
    assert st32.iterations <= 1.25 * st64.iterations + 5
    for x in (x64, x32):
        assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-5
