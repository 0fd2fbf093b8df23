"""ctypes binding of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline and
--impl reference legs, always as the checker or the timed host baseline,
never as the thing measured.  See cfm_oracle.h for the reference lines each
function restates.  Also exposes the reference's own single-GPU Jacobi and CG
runs (oracle/_ref, built from the reference sources) when they were built.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF2D_PATH = os.path.join(HERE, "_ref", "libref_jacobi2d.so")
REF3D_PATH = os.path.join(HERE, "_ref", "libref_jacobi3d.so")
REFCG_PATH = os.path.join(HERE, "_ref", "libref_cg.so")

_vp = ctypes.c_void_p
_i = ctypes.c_int


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: run `make -C oracle`")
    lib = ctypes.CDLL(LIB_PATH)
    sigs = {
        "orc_jacobi2d_init_f64": [_i, _i, _vp],
        "orc_jacobi2d_init_f32": [_i, _i, _vp],
        "orc_jacobi3d_init_f64": [_i, _i, _i, _i, _vp],
        "orc_jacobi3d_init_f32": [_i, _i, _i, _i, _vp],
        "orc_jacobi2d_f64": [_i, _i, _i, _vp, _vp, _i],
        "orc_jacobi2d_f32": [_i, _i, _i, _vp, _vp, _i],
        "orc_jacobi3d_f64": [_i, _i, _i, _i, _i, _vp, _vp, _i],
        "orc_jacobi3d_f32": [_i, _i, _i, _i, _i, _vp, _vp, _i],
        "orc_jacobi2d_mirror_f32": [_i, _i, _i, _vp, _vp, _i],
        "orc_jacobi2d_mirror_f64": [_i, _i, _i, _vp, _vp, _i],
        "orc_cg": [_i, _vp, _vp, _vp, _vp, _i, ctypes.c_double, _vp, _vp, _vp, _i],
        "orc_spmv": [_i, _vp, _vp, _vp, _vp, _vp, _i],
        "orc_max_threads": [],
        "orc_krylov_csr": [_i, _vp, _vp, _vp, _i, _vp, _i, ctypes.c_double, _i, ctypes.c_double,
                           _vp, _vp, _vp, _vp, _i],
        "orc_stencil_apply": [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i],
        "orc_krylov_stencil": [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp, _i, ctypes.c_double, _i,
                               ctypes.c_double, _vp, _vp, _vp, _vp, _i],
    }
    for name, args in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.orc_fpcg2d.argtypes = [_i, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _i, ctypes.c_double, _i,
                               ctypes.c_double, _vp, _vp, _vp, _vp]
    lib.orc_fpcg2d.restype = _i
    lib.orc_dot.argtypes = [ctypes.c_longlong, _vp, _vp, _i]
    lib.orc_dot.restype = ctypes.c_double
    lib.orc_jacobi3d_bench_f64.argtypes = [_i, _i, _i, _i, _i]
    lib.orc_jacobi3d_bench_f64.restype = ctypes.c_double
    return lib


lib = _load()


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _suffix(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def max_threads():
    return lib.orc_max_threads()


def jacobi2d_init(nx, ny, dtype=np.float64):
    a = np.empty((ny, nx), dtype)
    assert getattr(lib, f"orc_jacobi2d_init_{_suffix(dtype)}")(nx, ny, _p(a)) == 0
    return a


def jacobi3d_init(nx, ny, nz, problem, dtype=np.float64):
    a = np.empty((nz, ny, nx), dtype)
    assert getattr(lib, f"orc_jacobi3d_init_{_suffix(dtype)}")(nx, ny, nz, problem, _p(a)) == 0
    return a


def jacobi2d(a, niter, threads=0):
    a = np.ascontiguousarray(a)
    ny, nx = a.shape
    out = np.empty_like(a)
    assert getattr(lib, f"orc_jacobi2d_{_suffix(a.dtype)}")(nx, ny, niter, _p(a), _p(out), threads) == 0
    return out


def jacobi2d_mirror(a, niter, threads=0):
    a = np.ascontiguousarray(a)
    if a.dtype != np.float64:
        a = np.ascontiguousarray(a, np.float32)
    ny, nx = a.shape
    out = np.empty_like(a)
    assert getattr(lib, f"orc_jacobi2d_mirror_{_suffix(a.dtype)}")(nx, ny, niter, _p(a), _p(out),
                                                                  threads) == 0
    return out


def jacobi3d(a, niter, periodic_y=0, threads=0):
    a = np.ascontiguousarray(a)
    nz, ny, nx = a.shape
    out = np.empty_like(a)
    fn = getattr(lib, f"orc_jacobi3d_{_suffix(a.dtype)}")
    assert fn(nx, ny, nz, niter, periodic_y, _p(a), _p(out), threads) == 0
    return out


def jacobi3d_bench(n, niter, threads=0):
    """Seconds of `niter` FP64 sweeps of the n^3 periodic config problem (loop only)."""
    return lib.orc_jacobi3d_bench_f64(n, n, n, niter, threads)


def dot(a, b, threads=0):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return lib.orc_dot(len(a), _p(a), _p(b), threads)


def spmv(rowptr, col, val, x, threads=0):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(len(rowptr) - 1)
    assert lib.orc_spmv(len(y), _p(rowptr), _p(col), _p(val), _p(x), _p(y), threads) == 0
    return y


def cg(rowptr, col, val, b, maxiter, tol, threads=0):
    """Returns (x, status, iterations, true relative residual)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    n = len(rowptr) - 1
    x = np.empty(n)
    it = ctypes.c_longlong()
    rr = ctypes.c_double()
    bb = None if b is None else np.ascontiguousarray(b, np.float64)
    st = lib.orc_cg(n, _p(rowptr), _p(col), _p(val), None if bb is None else _p(bb), maxiter, tol,
                    _p(x), ctypes.byref(it), ctypes.byref(rr), threads)
    return x, st, it.value, rr.value


STD, PIPELINED, MIXED = 0, 1, 2


def krylov_csr(rowptr, col, val, b, method, maxiter, tol, inner_maxiter=0, inner_tol=0.0, threads=0):
    """Persistent-solver restatement on a CSR matrix.
    Returns (x, status, iterations, restarts or FP64 updates, true relative residual)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    n = len(rowptr) - 1
    x = np.empty(n)
    it, rs, rr = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_double()
    bb = None if b is None else np.ascontiguousarray(b, np.float64)
    st = lib.orc_krylov_csr(n, _p(rowptr), _p(col), _p(val), method, None if bb is None else _p(bb),
                            maxiter, tol, inner_maxiter, inner_tol, _p(x), ctypes.byref(it),
                            ctypes.byref(rs), ctypes.byref(rr), threads)
    return x, st, it.value, rs.value, rr.value


def _coeffs(c):
    """c = (we, wn, wt, dg) as cfm.varcoef_coeffs returns them."""
    we, wn, wt, dg = (np.ascontiguousarray(a, np.float64) for a in c)
    return we, wn, wt, dg


def stencil_apply(dims, shape, c, x, threads=0):
    we, wn, wt, dg = _coeffs(c)
    nx, ny, nz = shape
    x = np.ascontiguousarray(x, np.float64).reshape(-1)
    y = np.empty_like(x)
    assert lib.orc_stencil_apply(dims, nx, ny, nz, _p(we), _p(wn), _p(wt), _p(dg), _p(x), _p(y),
                                 threads) == 0
    return y


def krylov_stencil(dims, shape, c, b, method, maxiter, tol, inner_maxiter=0, inner_tol=0.0,
                   threads=0):
    we, wn, wt, dg = _coeffs(c)
    nx, ny, nz = shape
    x = np.empty(len(dg))
    it, rs, rr = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_double()
    bb = None if b is None else np.ascontiguousarray(b, np.float64).reshape(-1)
    st = lib.orc_krylov_stencil(dims, nx, ny, nz, _p(we), _p(wn), _p(wt), _p(dg), method,
                                None if bb is None else _p(bb), maxiter, tol, inner_maxiter,
                                inner_tol, _p(x), ctypes.byref(it), ctypes.byref(rs),
                                ctypes.byref(rr), threads)
    return x, st, it.value, rs.value, rr.value


def fpcg2d(shape, c, b, smooth, m, mixed=False, delta=0.1, maxiter=20000, tol=1e-8, f=1):
    """FPCG restatement (identity in place of the network) on the 2D stencil
    with coefficients c = (we, wn, wt, dg).  Returns (x, iterations,
    reliable updates, done)."""
    we, wn, _, dg = _coeffs(c)
    nx, ny = shape
    bb = np.ascontiguousarray(b, np.float64).reshape(-1)
    x = np.empty(nx * ny)
    it, up, dn = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
    assert lib.orc_fpcg2d(nx, ny, _p(we), _p(wn), _p(dg), _p(bb), f, smooth, m, int(mixed), delta,
                          maxiter, tol, _p(x), ctypes.byref(it), ctypes.byref(up), ctypes.byref(dn)) == 0
    return x, it.value, up.value, dn.value


# ------------------------------------------------------ the reference itself
def ref_available():
    return os.path.exists(REF2D_PATH) and os.path.exists(REF3D_PATH)


def _ref_lib(path, names):
    lib = ctypes.CDLL(path)
    for name, args in names.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_double
    return lib


def ref_jacobi2d(nx, ny, niter, mirror=False):
    """The reference's single_gpu() (FP32, its own init) on the current GPU."""
    lib = _ref_lib(REF2D_PATH, {"ref_jacobi2d_single_gpu": [_i, _i, _i, _vp],
                                "ref_jacobi2d_single_gpu_mirror": [_i, _i, _i, _vp]})
    out = np.empty((ny, nx), np.float32)
    fn = lib.ref_jacobi2d_single_gpu_mirror if mirror else lib.ref_jacobi2d_single_gpu
    fn(nx, ny, niter, _p(out))
    return out


def ref_jacobi3d(nx, ny, nz, niter):
    lib = _ref_lib(REF3D_PATH, {"ref_jacobi3d_single_gpu": [_i, _i, _i, _i, _vp]})
    out = np.empty((nz, ny, nx), np.float32)
    lib.ref_jacobi3d_single_gpu(nx, ny, nz, niter, _p(out))
    return out


def ref_cg_available():
    return os.path.exists(REFCG_PATH)


def _ref_cg_lib():
    lib = ctypes.CDLL(REFCG_PATH)
    lib.ref_cg_standard.argtypes = [_i, _i, _vp, _vp, _vp, _i, _i, _vp]
    lib.ref_cg_standard.restype = ctypes.c_double
    lib.ref_gen_tridiag.argtypes = [_i, _vp, _vp, _vp]
    lib.ref_gen_tridiag.restype = _i
    return lib


def ref_cg(rowptr, col, val, niter):
    """The reference's SingleGPUDiscreteStandard::run_single_gpu() on the
    current GPU: b = ones, x0 = 0, exactly `niter` iterations.  The index base
    is taken from rowptr[0], as the reference's main() does.  Returns x."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    n = len(rowptr) - 1
    x = np.empty(n)
    t = _ref_cg_lib().ref_cg_standard(n, len(val), _p(rowptr), _p(col), _p(val),
                                       int(rowptr[0] == 0), niter, _p(x))
    assert t >= 0, "reference CG run failed"
    return x


def ref_tridiag(n):
    """The reference's genTridiag() from libc rand()'s unseeded start state."""
    nnz = 3 * (n - 2) + 4
    rowptr = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz)
    assert _ref_cg_lib().ref_gen_tridiag(n, _p(rowptr), _p(col), _p(val)) == 0
    return rowptr, col, val
