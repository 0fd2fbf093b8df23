"""The drop-in binaries on the GPU: every single-GPU version of jacobi2D,
jacobi3D and cg runs, passes its own -compare / -compare-single-gpu check,
prints the execution time as the first float, and writes (-out) the grid the
oracle computes for the same problem, bit for bit."""
import os
import re
import subprocess

import numpy as np
import pytest

import cfm
import oracle

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(cfm.__file__), "bin")


def run(name, *args):
    out = subprocess.run([os.path.join(BIN, name), *map(str, args)], capture_output=True, text=True,
                         timeout=300)
    return out.returncode, out.stdout, out.stderr


def first_float(text):
    return float(re.search(r"[-+]?\d+\.\d+", text).group(0))


@pytest.mark.parametrize("version", range(6))
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_jacobi2d_versions_compare_and_match_oracle(version, prec, tmp_path):
    nx, ny, niter = 68, 37, 9
    path = tmp_path / "grid.bin"
    rc, out, err = run("jacobi2D", "-v", version, "-s", "-nx", nx, "-ny", ny, "-niter", niter,
                       "-precision", prec, "-compare", "-out", path)
    assert rc == 0 and "ERROR" not in err, err
    assert out.lstrip().startswith("Execution time:") and first_float(out) >= 0
    dt = np.float32 if prec == "fp32" else np.float64
    got = np.fromfile(path, dt).reshape(ny, nx)
    a = oracle.jacobi2d_init(nx, ny, dt)
    # PERKS (-v 5) runs the mirror x boundary, as the reference's PERKS version
    # is checked against jacobi_kernel_single_gpu_mirror
    want = oracle.jacobi2d_mirror(a, niter) if version == 5 else oracle.jacobi2d(a, niter)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("version,boundary", [(3, "mirror"), (5, "dirichlet"), (0, "mirror")])
def test_jacobi2d_boundary_flag(version, boundary, tmp_path):
    nx, ny, niter = 64, 30, 11
    path = tmp_path / "grid.bin"
    rc, out, err = run("jacobi2D", "-v", version, "-s", "-nx", nx, "-ny", ny, "-niter", niter,
                       "-boundary", boundary, "-compare", "-out", path)
    assert rc == 0 and "ERROR" not in err, err
    got = np.fromfile(path, np.float32).reshape(ny, nx)
    a = oracle.jacobi2d_init(nx, ny, np.float32)
    want = oracle.jacobi2d_mirror(a, niter) if boundary == "mirror" else oracle.jacobi2d(a, niter)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("version", [3, 5])
def test_jacobi2d_config1_full_length_and_norm(version, tmp_path):
    """Config 1 at its stated size and length: 1024^2 FP64, 1000 sweeps
    (Dirichlet columns), Design 1 and PERKS; the -out grid equals the oracle
    bit for bit and the printed final L2 norm is the oracle grid's."""
    nx = ny = 1024
    niter = 1000
    path = tmp_path / "grid.bin"
    rc, out, err = run("jacobi2D", "-v", version, "-s", "-nx", nx, "-ny", ny, "-niter", niter,
                       "-precision", "fp64", "-boundary", "dirichlet", "-out", path)
    assert rc == 0 and "ERROR" not in err, err
    got = np.fromfile(path, np.float64).reshape(ny, nx)
    want = oracle.jacobi2d(oracle.jacobi2d_init(nx, ny, np.float64), niter)
    np.testing.assert_array_equal(got, want)
    norm = float(re.search(r"Final grid L2 norm: (\S+)", out).group(1))
    want_norm = float(np.sqrt(np.sum(want.astype(np.longdouble) ** 2)))
    assert abs(norm - want_norm) <= 1e-14 * want_norm


@pytest.mark.parametrize("version", range(6))
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_jacobi3d_versions_compare_and_match_oracle(version, prec, tmp_path):
    nx, ny, nz, niter = 40, 19, 13, 5
    path = tmp_path / "grid.bin"
    rc, out, err = run("jacobi3D", "-v", version, "-s", "-nx", nx, "-ny", ny, "-nz", nz, "-niter", niter,
                       "-precision", prec, "-problem", "config", "-compare", "-out", path)
    assert rc == 0 and "ERROR" not in err, err
    assert out.lstrip().startswith("Execution time:")
    dt = np.float32 if prec == "fp32" else np.float64
    got = np.fromfile(path, dt).reshape(nz, ny, nx)
    want = oracle.jacobi3d(oracle.jacobi3d_init(nx, ny, nz, 1, dt), niter, 1)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("version", range(10))
def test_cg_versions_compare_single_gpu(version):
    rc, out, err = run("cg", "-v", version, "-s", "-problem", "poisson", "-grid", 14, "-tol", "1e-8",
                       "-compare-single-gpu")
    assert rc == 0 and "ERROR" not in err, err
    assert out.lstrip().startswith("Execution time:")
    assert "speedup" in out
    its = int(re.search(r"Iterations: (\d+)", out).group(1))
    assert 0 < its < 200
