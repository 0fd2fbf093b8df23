"""A batch of 2D systems in one FPCG device loop (cfm_fpcg_create_batch),
on the GPU through the C ABI.  With the identity in place of the network,
every member equals the oracle's FPCG restatement run on the member
embedded in the batch's frame (zero faces to the padding, unit diagonal,
zero right-hand side there) bit for bit, in FP64 and mixed precision.  With
the trained network on its 512^2 frame, members of uneven sizes all reach
the FP64 true residual 1e-8 with plain CG's accuracy, each at its own
iteration count."""
import numpy as np
import pytest

import cfm
import oracle

pytestmark = pytest.mark.gpu


def frame_coeffs(k, FX, FY):
    """The member's coefficients embedded at the origin of an FX x FY frame."""
    ny, nx = k.shape
    we, wn, wt, dg = cfm.varcoef_coeffs(k)
    F = [np.zeros((FY, FX)) for _ in range(4)]
    F[3][:] = 1.0
    we, wn, dg = we.reshape(ny, nx), wn.reshape(ny, nx), dg.reshape(ny, nx)
    F[0][:ny, :nx - 1] = we[:, :nx - 1]
    F[1][:ny - 1, :nx] = wn[:ny - 1, :]
    F[3][:ny, :nx] = dg
    return tuple(a.ravel() for a in F)


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("smooth,m", [(4, 1), (2, 3)])
def test_batch_members_match_oracle_on_their_frames(mixed, smooth, m):
    shapes = [(64, 64), (50, 70), (96, 96), (33, 17)]
    ks, fs = zip(*[cfm.varcoef_problem(sh, 40 + i) for i, sh in enumerate(shapes)])
    B = cfm.FPCGBatch(ks, None, maxiter=20000, tol=1e-8, smooth=smooth, truncation=m,
                      precision=cfm.FP32 if mixed else None)
    xs, its, stt, rr, st = B.solve(fs)
    assert (stt == cfm.OK).all() and (rr <= 1e-8).all()
    FY = max(sh[0] for sh in shapes)
    FX = max(sh[1] for sh in shapes)
    for k, f, x, it in zip(ks, fs, xs, its):
        ny, nx = k.shape
        bf = np.zeros((FY, FX))
        bf[:ny, :nx] = f
        x_o, it_o, _, done = oracle.fpcg2d((FX, FY), frame_coeffs(k, FX, FY), bf, smooth, m, mixed)
        assert done == 1 and it == it_o
        x_o = x_o.reshape(FY, FX)
        np.testing.assert_array_equal(x, x_o[:ny, :nx])
        assert not x_o[ny:, :].any() and not x_o[:, nx:].any()  # the padding stays zero


NC = 512


@pytest.fixture(scope="module")
def coarse_net():
    net = cfm.UNet(NC // 2, NC // 2, max_batch=4, seed=5)  # six members: two network chunks
    net.train_varcoef(24, 9, 7000, 8, 4, 1e-3, smooth=4, coarsen=2)
    return net


@pytest.mark.parametrize("mixed", [False, True])
def test_learned_batch_of_uneven_members(coarse_net, mixed):
    """Members of sides 256..512 (and one 300 x 450) in the 512^2 frame, the
    network in chunks of its batch of 4: all converge to 1e-8 without help,
    agree with plain CG, and take fewer iterations than Jacobi-smoothed FPCG."""
    shapes = [(512, 512), (300, 450), (256, 256), (384, 384), (420, 300), (512, 400)]
    ks, fs = zip(*[cfm.varcoef_problem(sh, 90 + i) for i, sh in enumerate(shapes)])
    B = cfm.FPCGBatch(ks, coarse_net, maxiter=20000, tol=1e-8, precision=cfm.FP32 if mixed else None)
    xs, its, stt, rr, st = B.solve(fs)
    print(f"learned batch ({'mixed' if mixed else 'FP64'}): iterations {list(its)}, "
          f"{st.seconds * 1e3:.1f} ms, {B.reliable_updates()} reliable updates")
    assert (stt == cfm.OK).all() and (rr <= 1e-8).all()
    for k, f, x, it in zip(ks, fs, xs, its):
        S = cfm.Stencil(k)
        xs_cg, _ = cfm.CG(S, cfm.CG_PERSISTENT, 50000, 1e-10).solve(f.ravel())
        assert np.linalg.norm(x.ravel() - xs_cg) / np.linalg.norm(xs_cg) < 1e-5
        _, st_j = cfm.FPCG(S, k, None, maxiter=20000, tol=1e-8, smooth=4).solve(f)
        assert it < st_j.iterations


def test_config5_shaped_subset_learned_split(coarse_net):
    """A config-5-shaped subset (2D sides 64..512, 3D sides 32..128, log-
    uniform, per-system seeds) solved as the bench does with the learned
    preconditioner: the 2D members of side >= 256 in the batched learned +
    mixed FPCG, the others in the persistent mixed polynomial kernel (its
    blocks per system from the autotuner).  Every member reaches the FP64
    true residual 1e-8, and the learned members take fewer iterations than
    the polynomial preconditioner gives them."""
    systems = cfm.uneven_systems(10, 4, seed=11)
    big = [i for i, (k, _) in enumerate(systems) if k.ndim == 2 and min(k.shape) >= 256]
    rest = [i for i in range(len(systems)) if i not in big]
    assert big and rest
    FB = cfm.FPCGBatch([systems[i][0] for i in big], coarse_net, maxiter=20000, tol=1e-8, precision=cfm.FP32)
    xs, it_l, st_l, rr_l, _ = FB.solve([systems[i][1] for i in big])
    B = cfm.Batch([systems[i] for i in rest])
    B.set_solver(smooth=4, maxiter=20000, tol=1e-8)
    B.set_precision(cfm.FP32, 0, 0.1)
    assert B.autotune() > 0
    it_p, st_p, rr_p, _ = B.solve()
    assert (st_l == cfm.OK).all() and (rr_l <= 1e-8).all()
    assert (st_p == cfm.OK).all() and (rr_p <= 1e-8 * 1.5).all()
    P = cfm.Batch([systems[i] for i in big])  # the same members with the polynomial
    P.set_solver(smooth=4, maxiter=20000, tol=1e-8)
    it_poly, st_poly, _, _ = P.solve()
    assert (st_poly == cfm.OK).all()
    print(f"learned {list(it_l)} vs polynomial {list(it_poly)}")
    assert (it_l < it_poly).all()
