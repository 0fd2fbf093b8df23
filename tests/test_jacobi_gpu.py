"""Jacobi parity on the GPU through the C ABI: every implementation must give
the oracle's grid bit-for-bit (FP64 and FP32), on random and problem inputs,
odd and tiny sizes, and the full 512^3 size."""
import os

import numpy as np
import pytest

import cfm
import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

IMPLS = [cfm.JACOBI_HOST_LOOP, cfm.JACOBI_HOST_LOOP_INKERNEL_HALO, cfm.JACOBI_PERSISTENT, cfm.JACOBI_RESIDENT]
PRECS = [cfm.FP64, cfm.FP32]


def rand_grid(shape, dtype, seed):
    return np.random.default_rng(seed).uniform(-1, 1, shape).astype(dtype)


def run_gpu(a, niter, impl, periodic_y=0, mirror=False):
    prec = cfm.FP64 if a.dtype == np.float64 else cfm.FP32
    if a.ndim == 2:
        ny, nx = a.shape
        j = cfm.Jacobi(2, nx, ny, 1, prec, 1, impl)
    else:
        nz, ny, nx = a.shape
        j = cfm.Jacobi(3, nx, ny, nz, prec, periodic_y, impl)
    with j:
        if mirror:
            j.set_boundary(cfm.BOUNDARY_MIRROR)
        j.upload(a)
        st = j.run(niter)
        assert st.iterations == niter
        return j.download(), st


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(3, 3), (9, 7), (17, 33), (70, 130), (1026, 100), (6, 4), (5, 64),
                                   (37, 128), (260, 256), (300, 1032)])
@pytest.mark.parametrize("niter", [0, 1, 2, 7])
def test_jacobi2d_random_bitexact(impl, prec, shape, niter):
    """Rows of a multiple of 16 bytes take the row-marching vector kernel,
    the others the warp-per-segment one; both equal the oracle."""
    a = rand_grid(shape, cfm.np_dtype(prec), 11)
    got, _ = run_gpu(a, niter, impl)
    np.testing.assert_array_equal(got, oracle.jacobi2d(a, niter))


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(3, 3), (9, 7), (17, 33), (70, 130), (1026, 100), (5, 64),
                                   (260, 256), (40, 2050)])
@pytest.mark.parametrize("niter", [0, 1, 2, 7])
def test_jacobi2d_mirror_random_bitexact(impl, prec, shape, niter):
    """The mirror x boundary (the reference's PERKS comparator,
    Stencil/jacobi2D/src/common.cu:44-66) on every implementation, edge
    columns and corner cells included."""
    a = rand_grid(shape, cfm.np_dtype(prec), 21)
    got, _ = run_gpu(a, niter, impl, mirror=True)
    np.testing.assert_array_equal(got, oracle.jacobi2d_mirror(a, niter))


def test_mirror_boundary_is_2d_only_and_switchable():
    a = rand_grid((34, 64), np.float64, 5)
    with cfm.Jacobi(2, 64, 34, 1, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        j.set_boundary(cfm.BOUNDARY_MIRROR)
        j.upload(a)
        j.run(3)
        np.testing.assert_array_equal(j.download(), oracle.jacobi2d_mirror(a, 3))
        j.set_boundary(cfm.BOUNDARY_DIRICHLET)
        j.upload(a)
        j.run(3)
        np.testing.assert_array_equal(j.download(), oracle.jacobi2d(a, 3))
    with cfm.Jacobi(3, 8, 8, 8, cfm.FP64, 0, cfm.JACOBI_PERSISTENT) as j:
        with pytest.raises(cfm.CfmError):
            j.set_boundary(cfm.BOUNDARY_MIRROR)


@pytest.mark.parametrize("impl", IMPLS)
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("py", [0, 1])
@pytest.mark.parametrize("shape", [(3, 3, 3), (5, 6, 7), (17, 9, 33), (16, 40, 64), (20, 11, 131),
                                   (7, 13, 128), (5, 3, 200), (33, 70, 96), (9, 10, 66)])
@pytest.mark.parametrize("niter", [1, 2, 5])
def test_jacobi3d_random_bitexact(impl, prec, py, shape, niter):
    a = rand_grid(shape, cfm.np_dtype(prec), 12)
    got, _ = run_gpu(a, niter, impl, py)
    np.testing.assert_array_equal(got, oracle.jacobi3d(a, niter, py))


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("dims,problem", [(2, 0), (3, 0), (3, 1)])
def test_device_problem_matches_host_problem(prec, dims, problem):
    shape = (37, 45) if dims == 2 else (11, 13, 37)
    ny, nx = shape[-2:]
    nz = shape[0] if dims == 3 else 1
    with cfm.Jacobi(dims, nx, ny, nz, prec, problem if dims == 3 else 1) as j:
        want = j.problem_host(problem)
        j.load_problem(problem)
        np.testing.assert_array_equal(j.download(), want)


def test_jacobi2d_config1_problem_1024():
    """Config 1 at its stated length: 1024^2 FP64, 1000 sweeps, persistent and
    resident against the oracle bit for bit."""
    a = oracle.jacobi2d_init(1024, 1024, np.float64)
    want = oracle.jacobi2d(a, 1000)
    with cfm.Jacobi(2, 1024, 1024, 1, cfm.FP64, 1, cfm.JACOBI_RESIDENT) as j:
        assert j.launch_shape()[1] == 1024  # the on-chip resident kernel
    for impl in (cfm.JACOBI_PERSISTENT, cfm.JACOBI_RESIDENT):
        got, st = run_gpu(a, 1000, impl)
        np.testing.assert_array_equal(got, want)
        assert st.launches <= 2


@pytest.fixture(scope="module")
def config2_fp64():
    """The 512^3 periodic config problem and the oracle's grid after config
    2's 100 sweeps (about 1.07 GB each)."""
    with cfm.Jacobi(3, 512, 512, 512, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        a = j.problem_host(cfm.PROBLEM_CONFIG)
    return a, oracle.jacobi3d(a, 100, 1)


def test_jacobi3d_config2_fp64_100_sweeps_bitexact(config2_fp64):
    """Config 2 at its stated size and length: 512^3 FP64, 100 sweeps, the
    persistent TMA pipeline equals the oracle bit for bit."""
    a, want = config2_fp64
    got, st = run_gpu(a, 100, cfm.JACOBI_PERSISTENT, 1)
    assert st.launches == 2
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("dataflow", [False, True])
@pytest.mark.parametrize("shape,py,niter", [((96, 40, 64), 1, 7), ((70, 33, 128), 0, 5), ((34, 130, 64), 1, 12),
                                            ((18, 9, 16), 1, 4)])
def test_jacobi3d_sweep_order_same_grid(dataflow, shape, py, niter):
    """The TMA pipeline with a grid barrier per sweep and with the units'
    neighbourhood order (no grid barrier) give the oracle's grid, including
    the periodic images across z chunks and y tiles."""
    for prec in PRECS:
        a = rand_grid(shape, cfm.np_dtype(prec), 17)
        nz, ny, nx = shape
        with cfm.Jacobi(3, nx, ny, nz, prec, py, cfm.JACOBI_PERSISTENT) as j:
            j.set_dataflow(dataflow)
            j.upload(a)
            st = j.run(niter)
            np.testing.assert_array_equal(j.download(), oracle.jacobi3d(a, niter, py))
            assert st.status == cfm.OK


def test_jacobi3d_config2_fp32_100_sweeps(config2_fp64):
    """Config 2's FP32 variant: 512^3, 100 sweeps, bit for bit against the FP32
    oracle, and within 1.5e-6 (max-abs and relative L2) of the FP64 grid."""
    a64, want64 = config2_fp64
    a32 = a64.astype(np.float32)
    got, _ = run_gpu(a32, 100, cfm.JACOBI_PERSISTENT, 1)
    np.testing.assert_array_equal(got, oracle.jacobi3d(a32, 100, 1))
    err = got.astype(np.float64) - want64
    assert np.abs(err).max() <= 1.5e-6
    assert np.linalg.norm(err) / np.linalg.norm(want64) <= 1.5e-6


def test_jacobi3d_512_fp64_bitexact_and_e2e():
    """Full-size 512^3 FP64 periodic problem: 3 sweeps equal the oracle; the
    end-to-end host-buffer call gives the same grid."""
    nx = ny = nz = 512
    with cfm.Jacobi(3, nx, ny, nz, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        assert j.launch_shape()[1] in (96, 160, 288)  # a TMA pipeline kernel (consumer warps + producer)
        a = j.problem_host(cfm.PROBLEM_CONFIG)
        want = oracle.jacobi3d(a, 3, 1)
        j.upload(a)
        st = j.run(3)
        np.testing.assert_array_equal(j.download(), want)
        assert st.launches == 2 and st.glups > 0
        out = np.empty_like(a)
        st2 = j.run_host(3, a, out)
        np.testing.assert_array_equal(out, want)
        assert st2.h2d_bytes == a.nbytes and st2.d2h_bytes == a.nbytes


def test_autotune_restores_grid_and_stays_bitexact():
    a = rand_grid((40, 36, 128), np.float64, 15)
    with cfm.Jacobi(3, 128, 36, 40, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        j.upload(a)
        best, rate = j.autotune(3)
        assert best >= 0 and rate > 0 and cfm.variant_info(best) is not None
        np.testing.assert_array_equal(j.download(), a)
        j.run(6)
        np.testing.assert_array_equal(j.download(), oracle.jacobi3d(a, 6, 1))
    with cfm.Jacobi(2, 64, 64, 1, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        assert j.autotune(2)[0] == -1  # nothing to tune outside the 3D TMA pipeline


NVARIANTS = 16  # pipeline shapes: 0-11 one sweep per pass, 12-15 two


@pytest.mark.parametrize("variant", range(NVARIANTS))
def test_every_pipeline_variant_bitexact(variant, monkeypatch):
    assert cfm.variant_info(variant) is not None and cfm.variant_info(NVARIANTS) is None
    assert cfm.variant_info(variant)[3] == (2 if variant >= 12 else 1)
    monkeypatch.setenv("CFM_J3D_TMA_VARIANT", str(variant))
    for prec, py, shape in ((cfm.FP64, 1, (21, 19, 128)), (cfm.FP32, 0, (13, 40, 136))):
        a = rand_grid(shape, cfm.np_dtype(prec), 16)
        got, _ = run_gpu(a, 5, cfm.JACOBI_PERSISTENT, py)
        np.testing.assert_array_equal(got, oracle.jacobi3d(a, 5, py))


@pytest.mark.parametrize("variant", range(12, NVARIANTS))
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("py", [0, 1])
@pytest.mark.parametrize("shape", [(3, 3, 64), (4, 5, 64), (5, 3, 130), (7, 36, 64), (40, 35, 192),
                                   (70, 9, 128)])
@pytest.mark.parametrize("niter", [1, 2, 3, 6])
def test_two_sweep_pipeline_bitexact(variant, prec, py, shape, niter, monkeypatch):
    """Two sweeps per pass: the periodic images (far rows and planes), tiny
    grids where one tile or one z-chunk touches both ends, odd counts."""
    monkeypatch.setenv("CFM_J3D_TMA_VARIANT", str(variant))
    a = rand_grid(shape, cfm.np_dtype(prec), 17)
    got, st = run_gpu(a, niter, cfm.JACOBI_PERSISTENT, py)
    np.testing.assert_array_equal(got, oracle.jacobi3d(a, niter, py))


@pytest.mark.parametrize("zc", [1, 2, 5, 64])
def test_two_sweep_pipeline_zchunks(zc, monkeypatch):
    monkeypatch.setenv("CFM_J3D_TMA_VARIANT", "13")
    monkeypatch.setenv("CFM_J3D_ZCHUNK", str(zc))
    a = rand_grid((23, 21, 128), np.float64, 18)
    got, _ = run_gpu(a, 4, cfm.JACOBI_PERSISTENT, 1)
    np.testing.assert_array_equal(got, oracle.jacobi3d(a, 4, 1))


def test_jacobi_run_twice_equals_one_long_run():
    a = rand_grid((13, 17, 19), np.float64, 13)
    with cfm.Jacobi(3, 19, 17, 13, cfm.FP64, 1, cfm.JACOBI_PERSISTENT) as j:
        j.upload(a)
        j.run(3)
        j.run(4)
        np.testing.assert_array_equal(j.download(), oracle.jacobi3d(a, 7, 1))


def test_fp32_variant_error_against_fp64_oracle():
    """The FP32 sweep of the 3D problem stays close to the FP64 oracle (the
    bound is loose: it documents the max-abs and L2 error, not a claim)."""
    n = 64
    a64 = oracle.jacobi3d_init(n, n, n, 1, np.float64)
    want = oracle.jacobi3d(a64, 100, 1)
    got, _ = run_gpu(a64.astype(np.float32), 100, cfm.JACOBI_PERSISTENT, 1)
    err = got.astype(np.float64) - want
    assert np.abs(err).max() < 1e-5
    assert np.linalg.norm(err) / np.linalg.norm(want) < 1e-5


# --------------------------------------------------- pin against the reference
def _ref_cases():
    import glob
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_jacobi*.npz")))


@pytest.mark.parametrize("path", _ref_cases(), ids=os.path.basename)
@pytest.mark.parametrize("impl", IMPLS)
def test_gpu_matches_reference_fixture(path, impl):
    """Our kernels reproduce grids written by the reference's own single_gpu()."""
    f = np.load(path)
    kind = str(f["kind"])
    out = f["out"]
    niter = int(f["niter"])
    if kind == "2d_mirror":
        # the mirror sweep updates the x edge columns, so it starts from the
        # initial state (the oracle's, pinned to these fixtures on the CPU)
        ny, nx = out.shape
        a = oracle.jacobi2d_init(nx, ny, np.float32)
        got, _ = run_gpu(a, niter, impl, mirror=True)
        np.testing.assert_array_equal(got, out)
        return
    if kind == "2d":
        ny, nx = out.shape
        # the reference computed its boundary columns with device sin; a sweep
        # never changes them (the corner cells it does change are never read)
        a = np.zeros((ny, nx), np.float32)
        a[:, 0] = out[:, 0]
        a[:, -1] = out[:, -1]
    else:
        nz, ny, nx = out.shape
        a = oracle.jacobi3d_init(nx, ny, nz, 0, np.float32)
    got, _ = run_gpu(a, niter, impl, 0)
    np.testing.assert_array_equal(got, out)


def test_barrier_timeout_returns_status_and_device_stays_usable():
    cfm.set_barrier_timeout_ms(300)
    try:
        st, ms = cfm.barrier_selftest(0, 3, 5)
        assert st == cfm.BARRIER_TIMEOUT
        assert 250 <= ms < 5000
        st, _ = cfm.barrier_selftest(0, 1000, -1)
        assert st == cfm.OK
        a = rand_grid((9, 10, 11), np.float64, 14)
        got, _ = run_gpu(a, 4, cfm.JACOBI_PERSISTENT, 1)
        np.testing.assert_array_equal(got, oracle.jacobi3d(a, 4, 1))
    finally:
        cfm.set_barrier_timeout_ms(2000)
