"""ctypes binding of libcfm.so (declared in include/cfm.h).

Used by the tests and bench.py to drive the C ABI exactly as a foreign host
(cgo / JNI / ctypes) would: plain pointers and sizes, integer status codes.
There is no fallback: if lib/libcfm.so is missing the import of this module
raises, and every call goes to the CUDA library.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcfm.so")

OK, BAD_ARG, CUDA_ERROR, BARRIER_TIMEOUT, BREAKDOWN, NOT_CONVERGED, NO_DEVICE, UNSUPPORTED, OOM = range(9)
FP64, FP32 = 0, 1
PROBLEM_REF, PROBLEM_CONFIG = 0, 1
JACOBI_HOST_LOOP, JACOBI_HOST_LOOP_INKERNEL_HALO, JACOBI_PERSISTENT, JACOBI_RESIDENT = range(4)
BOUNDARY_DIRICHLET, BOUNDARY_MIRROR = 0, 1
CG_DISCRETE, CG_PERSISTENT, CG_PERSISTENT_PIPELINED, CG_MIXED = range(4)

# Every function include/cfm.h declares, with (restype, argtypes).
_c = ctypes
_vp = _c.c_void_p
_SIGS = {
    "cfm_api_version": (_c.c_int, []),
    "cfm_status_string": (_c.c_char_p, [_c.c_int]),
    "cfm_last_error": (_c.c_char_p, []),
    "cfm_set_barrier_timeout_ms": (_c.c_int, [_c.c_double]),
    "cfm_device_info": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_jacobi_problem_host": (_c.c_int, [_vp, _c.c_int, _vp]),
    "cfm_jacobi_create": (_c.c_int, [_vp, _vp]),
    "cfm_jacobi_destroy": (None, [_vp]),
    "cfm_jacobi_set_stream": (_c.c_int, [_vp, _vp]),
    "cfm_jacobi_set_boundary": (_c.c_int, [_vp, _c.c_int]),
    "cfm_jacobi_set_dataflow": (_c.c_int, [_vp, _c.c_int]),
    "cfm_jacobi_load_problem": (_c.c_int, [_vp, _c.c_int]),
    "cfm_jacobi_upload": (_c.c_int, [_vp, _vp]),
    "cfm_jacobi_download": (_c.c_int, [_vp, _vp]),
    "cfm_jacobi_run": (_c.c_int, [_vp, _c.c_int, _vp]),
    "cfm_jacobi_run_host": (_c.c_int, [_vp, _c.c_int, _vp, _vp, _vp]),
    "cfm_jacobi_device_grid": (_vp, [_vp]),
    "cfm_jacobi_launch_shape": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_jacobi_autotune": (_c.c_int, [_vp, _c.c_int, _vp, _vp]),
    "cfm_jacobi_variant_info": (_c.c_int, [_c.c_int, _vp, _vp, _vp]),
    "cfm_jacobi_variant_sweeps": (_c.c_int, [_c.c_int]),
    "cfm_mm_read": (_c.c_int, [_c.c_char_p, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cfm_jacobi_zchunk": (_c.c_int, [_vp]),
    "cfm_csr_create": (_c.c_int, [_c.c_int, _c.c_longlong, _vp, _vp, _vp, _vp]),
    "cfm_csr_destroy": (None, [_vp]),
    "cfm_csr_spmv_host": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_cg_create": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_cg_destroy": (None, [_vp]),
    "cfm_cg_set_stream": (_c.c_int, [_vp, _vp]),
    "cfm_cg_solve": (_c.c_int, [_vp, _vp, _vp, _vp]),
    "cfm_cg_solve_device": (_c.c_int, [_vp, _vp, _vp, _vp]),
    "cfm_cg_solve_noalloc": (_c.c_int, [_c.c_int, _c.c_longlong, _vp, _vp, _vp, _vp, _vp, _c.c_int,
                                        _c.c_double, _vp, _vp]),
    "cfm_stencil_create": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _vp, _vp]),
    "cfm_stencil_destroy": (None, [_vp]),
    "cfm_stencil_apply_host": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_cg_create_stencil": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_normal": (_c.c_int, [_c.c_ulonglong, _c.c_uint, _c.c_longlong, _vp]),
    "cfm_grf": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_ulonglong, _c.c_double,
                           _c.c_double, _vp]),
    "cfm_varcoef_problem": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_ulonglong, _vp, _vp]),
    "cfm_varcoef_coeffs": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp]),
    "cfm_tc_conv3x3": (_c.c_int, [_c.c_int] * 5 + [_vp, _vp, _vp, _c.c_int, _vp]),
    "cfm_tc_conv3x3_wgrad": (_c.c_int, [_c.c_int] * 5 + [_vp, _vp, _vp]),
    "cfm_unet_num_params": (_c.c_longlong, []),
    "cfm_unet_create": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_ulonglong, _vp]),
    "cfm_unet_destroy": (None, [_vp]),
    "cfm_unet_get_params": (_c.c_int, [_vp, _vp]),
    "cfm_unet_set_params": (_c.c_int, [_vp, _vp]),
    "cfm_unet_forward_host": (_c.c_int, [_vp, _c.c_int, _vp, _vp]),
    "cfm_unet_set_training_info": (_c.c_int, [_vp, _c.c_int, _c.c_int]),
    "cfm_unet_gradient_host": (_c.c_int, [_vp, _c.c_int, _vp, _vp, _vp]),
    "cfm_unet_activation_host": (_c.c_int, [_vp, _c.c_int, _c.c_int, _vp]),
    "cfm_unet_time_forward": (_c.c_int, [_vp, _c.c_int, _c.c_int, _vp]),
    "cfm_unet_set_forward_mode": (_c.c_int, [_vp, _c.c_int]),
    "cfm_unet_time_train_step": (_c.c_int, [_vp, _c.c_int, _c.c_int, _vp]),
    "cfm_unet_train_varcoef": (_c.c_int, [_vp, _c.c_int, _c.c_int, _c.c_ulonglong, _c.c_int, _c.c_int,
                                          _c.c_float, _c.c_int, _c.c_int, _vp, _vp, _vp, _vp]),
    "cfm_unet_set_validation": (_c.c_int, [_vp, _c.c_ulonglong, _c.c_int]),
    "cfm_unet_validation": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_fpcg_create": (_c.c_int, [_vp, _vp, _vp, _c.c_int, _c.c_int, _c.c_double, _vp]),
    "cfm_fpcg_destroy": (None, [_vp]),
    "cfm_fpcg_set_truncation": (_c.c_int, [_vp, _c.c_int]),
    "cfm_fpcg_set_network_period": (_c.c_int, [_vp, _c.c_int]),
    "cfm_fpcg_solve": (_c.c_int, [_vp, _vp, _vp, _vp]),
    "cfm_fpcg_history": (_c.c_int, [_vp, _vp, _c.c_longlong, _vp]),
    "cfm_fpcg_set_precision": (_c.c_int, [_vp, _c.c_int, _c.c_double]),
    "cfm_fpcg_set_device_loop": (_c.c_int, [_vp, _c.c_int]),
    "cfm_fpcg_reliable_updates": (_c.c_int, [_vp]),
    "cfm_fpcg_create_batch": (_c.c_int, [_c.c_int, _vp, _vp, _vp, _vp, _c.c_int, _c.c_int, _c.c_double, _vp]),
    "cfm_fpcg_solve_batch": (_c.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cfm_batch_create": (_c.c_int, [_c.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cfm_batch_destroy": (None, [_vp]),
    "cfm_batch_set_plan": (_c.c_int, [_vp, _c.c_int, _vp, _vp]),
    "cfm_batch_set_solver": (_c.c_int, [_vp, _c.c_int, _c.c_int, _c.c_double]),
    "cfm_batch_set_precision": (_c.c_int, [_vp, _c.c_int, _c.c_int, _c.c_double]),
    "cfm_batch_solve": (_c.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "cfm_batch_solution": (_c.c_int, [_vp, _c.c_int, _vp]),
    "cfm_batch_autotune": (_c.c_int, [_vp, _vp]),
    "cfm_poisson3d_nnz": (_c.c_longlong, [_c.c_int, _c.c_int, _c.c_int]),
    "cfm_poisson3d_csr": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _vp, _vp, _vp]),
    "cfm_tridiag_csr": (_c.c_int, [_c.c_int, _vp, _vp, _vp]),
    "cfm_uniform": (_c.c_int, [_c.c_ulonglong, _c.c_longlong, _c.c_double, _c.c_double, _vp]),
    "cfm_philox4x32_10": (_c.c_int, [_vp, _vp, _vp]),
    "cfm_barrier_selftest": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _vp]),
}


class Stats(ctypes.Structure):
    _fields_ = [
        ("seconds", ctypes.c_double),
        ("iterations", ctypes.c_longlong),
        ("lups", ctypes.c_double),
        ("glups", ctypes.c_double),
        ("bytes", ctypes.c_double),
        ("gbs", ctypes.c_double),
        ("residual", ctypes.c_double),
        ("h2d_bytes", ctypes.c_double),
        ("d2h_bytes", ctypes.c_double),
        ("launches", ctypes.c_int),
        ("status", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("pad", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class JacobiParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("dims", "nx", "ny", "nz", "precision", "periodic_y", "impl")]


class CGParams(ctypes.Structure):
    _fields_ = [
        ("impl", ctypes.c_int),
        ("maxiter", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("inner_maxiter", ctypes.c_int),
        ("inner_tol", ctypes.c_double),
    ]


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C cpu-free-model_b200` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load_library()


class CfmError(RuntimeError):
    def __init__(self, what, status):
        self.status = status
        msg = lib.cfm_last_error().decode(errors="replace")
        super().__init__(f"{what}: {lib.cfm_status_string(status).decode()} ({msg})")


def check(what, status, allowed=(OK,)):
    if status not in allowed:
        raise CfmError(what, status)
    return status


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def np_dtype(precision):
    return np.float64 if precision == FP64 else np.float32


class Jacobi:
    """One device grid pair; mirrors cfm_jacobi_* (and the reference's init(argc, argv))."""

    def __init__(self, dims, nx, ny, nz=1, precision=FP64, periodic_y=0, impl=JACOBI_PERSISTENT):
        self.p = JacobiParams(dims, nx, ny, nz if dims == 3 else 1, precision, periodic_y, impl)
        self.shape = (nz, ny, nx) if dims == 3 else (ny, nx)
        self.dtype = np_dtype(precision)
        h = ctypes.c_void_p()
        check("cfm_jacobi_create", lib.cfm_jacobi_create(ctypes.byref(self.p), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_jacobi_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def problem_host(self, problem):
        a = np.empty(self.shape, self.dtype)
        check("cfm_jacobi_problem_host", lib.cfm_jacobi_problem_host(ctypes.byref(self.p), problem, _ptr(a)))
        return a

    def load_problem(self, problem):
        check("cfm_jacobi_load_problem", lib.cfm_jacobi_load_problem(self.h, problem))

    def upload(self, a):
        a = np.ascontiguousarray(a, self.dtype)
        assert a.shape == self.shape
        check("cfm_jacobi_upload", lib.cfm_jacobi_upload(self.h, _ptr(a)))

    def download(self):
        a = np.empty(self.shape, self.dtype)
        check("cfm_jacobi_download", lib.cfm_jacobi_download(self.h, _ptr(a)))
        return a

    def run(self, niter, allowed=(OK,)):
        st = Stats()
        check("cfm_jacobi_run", lib.cfm_jacobi_run(self.h, niter, ctypes.byref(st)), allowed)
        return st

    def run_host(self, niter, host_in, host_out):
        """End-to-end call with caller-owned host buffers (numpy or pinned torch memory)."""
        st = Stats()
        pin = host_in.ctypes.data if isinstance(host_in, np.ndarray) else host_in.data_ptr()
        pout = host_out.ctypes.data if isinstance(host_out, np.ndarray) else host_out.data_ptr()
        check("cfm_jacobi_run_host",
              lib.cfm_jacobi_run_host(self.h, niter, ctypes.c_void_p(pin), ctypes.c_void_p(pout), ctypes.byref(st)))
        return st

    def set_stream(self, stream_handle):
        check("cfm_jacobi_set_stream", lib.cfm_jacobi_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def set_dataflow(self, on):
        """3D TMA pipeline: order sweeps by unit neighbourhoods (True) or by a
        grid barrier per sweep (False)."""
        check("cfm_jacobi_set_dataflow", lib.cfm_jacobi_set_dataflow(self.h, int(on)))

    def set_boundary(self, boundary):
        """BOUNDARY_DIRICHLET (fixed x columns) or, 2D only, BOUNDARY_MIRROR
        (the reference's PERKS comparator sweep)."""
        check("cfm_jacobi_set_boundary", lib.cfm_jacobi_set_boundary(self.h, boundary))

    def device_grid(self):
        return lib.cfm_jacobi_device_grid(self.h)

    def launch_shape(self):
        b, t = ctypes.c_int(), ctypes.c_int()
        check("cfm_jacobi_launch_shape", lib.cfm_jacobi_launch_shape(self.h, ctypes.byref(b), ctypes.byref(t)))
        return b.value, t.value

    def autotune(self, sweeps=20):
        v, r = ctypes.c_int(), ctypes.c_double()
        check("cfm_jacobi_autotune", lib.cfm_jacobi_autotune(self.h, sweeps, ctypes.byref(v), ctypes.byref(r)))
        return v.value, r.value


def mm_read(path):
    """MatrixMarket coordinate file -> (rowptr, col, val, m, n) with the file's
    index base kept in rowptr[0] (cfm_mm_read)."""
    m, n, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    p = os.fsencode(path)
    check("cfm_mm_read", lib.cfm_mm_read(p, ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz), None, None, None))
    rowptr = np.empty(m.value + 1, np.int32)
    col = np.empty(nnz.value, np.int32)
    val = np.empty(nnz.value, np.float64)
    check("cfm_mm_read", lib.cfm_mm_read(p, ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz), _ptr(rowptr),
                                         _ptr(col), _ptr(val)))
    return rowptr, col, val, m.value, n.value


def variant_info(i):
    """(consumer warps, rows per warp, stages, sweeps per pass) of pipeline shape i, or None."""
    cw, rpw, st = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    s = lib.cfm_jacobi_variant_info(i, ctypes.byref(cw), ctypes.byref(rpw), ctypes.byref(st))
    return None if s != OK else (cw.value, rpw.value, st.value, lib.cfm_jacobi_variant_sweeps(i))


class CSR:
    def __init__(self, rowptr, col, val):
        self.rowptr = np.ascontiguousarray(rowptr, np.int32)
        self.col = np.ascontiguousarray(col, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        self.n = len(self.rowptr) - 1
        h = ctypes.c_void_p()
        check("cfm_csr_create", lib.cfm_csr_create(self.n, len(self.val), _ptr(self.rowptr), _ptr(self.col),
                                                   _ptr(self.val), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_csr_destroy(self.h)
            self.h = None

    __del__ = close

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.n)
        check("cfm_csr_spmv_host", lib.cfm_csr_spmv_host(self.h, _ptr(x), _ptr(y)))
        return y


class Stencil:
    """Matrix-free variable-coefficient operator (cfm_stencil) built from k."""

    def __init__(self, k):
        k = np.ascontiguousarray(k, np.float64)
        self.dims = k.ndim
        self.shape = k.shape
        nz = k.shape[0] if k.ndim == 3 else 1
        ny, nx = k.shape[-2], k.shape[-1]
        self.grid = (nx, ny, nz)
        self.n = k.size
        h = ctypes.c_void_p()
        check("cfm_stencil_create", lib.cfm_stencil_create(self.dims, nx, ny, nz, _ptr(k), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_stencil_destroy(self.h)
            self.h = None

    __del__ = close

    def apply(self, x):
        x = np.ascontiguousarray(x, np.float64).reshape(-1)
        y = np.empty(self.n)
        check("cfm_stencil_apply_host", lib.cfm_stencil_apply_host(self.h, _ptr(x), _ptr(y)))
        return y


class CG:
    def __init__(self, A, impl=CG_PERSISTENT, maxiter=20000, tol=1e-8, inner_maxiter=0, inner_tol=0.0):
        self.A = A
        self.p = CGParams(impl, maxiter, tol, inner_maxiter, inner_tol)
        h = ctypes.c_void_p()
        if isinstance(A, Stencil):
            check("cfm_cg_create_stencil", lib.cfm_cg_create_stencil(A.h, ctypes.byref(self.p), ctypes.byref(h)))
        else:
            check("cfm_cg_create", lib.cfm_cg_create(A.h, ctypes.byref(self.p), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_cg_destroy(self.h)
            self.h = None

    __del__ = close

    def solve(self, b=None, allowed=(OK, NOT_CONVERGED)):
        x = np.empty(self.A.n)
        st = Stats()
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        check("cfm_cg_solve", lib.cfm_cg_solve(self.h, _ptr(bb), _ptr(x), ctypes.byref(st)), allowed)
        return x, st

    def solve_device(self, b_dev_ptr, x_dev_ptr, allowed=(OK, NOT_CONVERGED)):
        st = Stats()
        check("cfm_cg_solve_device", lib.cfm_cg_solve_device(self.h, ctypes.c_void_p(b_dev_ptr),
                                                              ctypes.c_void_p(x_dev_ptr), ctypes.byref(st)), allowed)
        return st

    def set_stream(self, stream_handle):
        check("cfm_cg_set_stream", lib.cfm_cg_set_stream(self.h, ctypes.c_void_p(stream_handle)))


def poisson3d(g):
    nnz = lib.cfm_poisson3d_nnz(g, g, g)
    n = g * g * g
    rowptr = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz, np.float64)
    check("cfm_poisson3d_csr", lib.cfm_poisson3d_csr(g, g, g, _ptr(rowptr), _ptr(col), _ptr(val)))
    return rowptr, col, val


def tridiag(n):
    nnz = 3 * n - 2
    rowptr = np.empty(n + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz, np.float64)
    check("cfm_tridiag_csr", lib.cfm_tridiag_csr(n, _ptr(rowptr), _ptr(col), _ptr(val)))
    return rowptr, col, val


def uniform(seed, n, lo=-1.0, hi=1.0):
    out = np.empty(n)
    check("cfm_uniform", lib.cfm_uniform(seed, n, lo, hi, _ptr(out)))
    return out


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.empty(4, np.uint32)
    check("cfm_philox4x32_10", lib.cfm_philox4x32_10(_ptr(c), _ptr(k), _ptr(o)))
    return o


def device_info():
    sms, ma, mi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = lib.cfm_device_info(ctypes.byref(sms), ctypes.byref(ma), ctypes.byref(mi))
    return st, sms.value, ma.value, mi.value


def barrier_selftest(blocks=0, rounds=4, drop_block=-1):
    ms = ctypes.c_double()
    st = lib.cfm_barrier_selftest(blocks, rounds, drop_block, ctypes.byref(ms))
    return st, ms.value


def set_barrier_timeout_ms(ms):
    check("cfm_set_barrier_timeout_ms", lib.cfm_set_barrier_timeout_ms(ms))


def normal(seed, n, stream=0):
    out = np.empty(n)
    check("cfm_normal", lib.cfm_normal(seed, stream, n, _ptr(out)))
    return out


def _grid_args(shape):
    if len(shape) == 2:
        return 2, shape[1], shape[0], 1
    return 3, shape[2], shape[1], shape[0]


def grf(shape, seed, sigma=1.0, corr_len=16.0):
    dims, nx, ny, nz = _grid_args(shape)
    out = np.empty(shape)
    check("cfm_grf", lib.cfm_grf(dims, nx, ny, nz, seed, sigma, corr_len, _ptr(out)))
    return out


def varcoef_problem(shape, seed):
    """(k, f) of the variable-coefficient diffusion problem on a grid of `shape` (y, x) or (z, y, x)."""
    dims, nx, ny, nz = _grid_args(shape)
    k = np.empty(shape)
    f = np.empty(shape)
    check("cfm_varcoef_problem", lib.cfm_varcoef_problem(dims, nx, ny, nz, seed, _ptr(k), _ptr(f)))
    return k, f


def varcoef_coeffs(k):
    """(we, wn, wt, dg) face coefficients of the stencil operator for k."""
    k = np.ascontiguousarray(k, np.float64)
    dims, nx, ny, nz = _grid_args(k.shape)
    we, wn, wt, dg = (np.zeros(k.size) for _ in range(4))
    check("cfm_varcoef_coeffs", lib.cfm_varcoef_coeffs(dims, nx, ny, nz, _ptr(k), _ptr(we), _ptr(wn),
                                                       _ptr(wt), _ptr(dg)))
    return we, wn, wt, dg


def to_bf16_bits(a):
    """float array -> uint16 BF16 patterns, round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b):
    return (np.ascontiguousarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def tc_conv3x3(x_bits, w_bits, bias=None, relu=False):
    """x [B,H,W,Cin] and w [9,Cout,Cin] as BF16 patterns -> out [B,H,W,Cout] BF16 patterns."""
    B, H, W, Cin = x_bits.shape
    Cout = w_bits.shape[1]
    x_bits = np.ascontiguousarray(x_bits, np.uint16)
    w_bits = np.ascontiguousarray(w_bits, np.uint16)
    out = np.empty((B, H, W, Cout), np.uint16)
    bb = None if bias is None else np.ascontiguousarray(bias, np.float32)
    check("cfm_tc_conv3x3", lib.cfm_tc_conv3x3(B, H, W, Cin, Cout, _ptr(x_bits), _ptr(w_bits), _ptr(bb),
                                               int(relu), _ptr(out)))
    return out


def tc_conv3x3_wgrad(x_bits, dz_bits):
    B, H, W, Cin = x_bits.shape
    Cout = dz_bits.shape[3]
    x_bits = np.ascontiguousarray(x_bits, np.uint16)
    dz_bits = np.ascontiguousarray(dz_bits, np.uint16)
    dw = np.empty((9, Cout, Cin), np.float32)
    check("cfm_tc_conv3x3_wgrad", lib.cfm_tc_conv3x3_wgrad(B, H, W, Cin, Cout, _ptr(x_bits), _ptr(dz_bits),
                                                           _ptr(dw)))
    return dw


# U-Net forward pass (cfm_unet_set_forward_mode)
UNET_FORWARD_AUTO, UNET_FORWARD_LAYERS, UNET_FORWARD_PERSISTENT = 0, 1, 2


class UNet:
    """The learned preconditioner's network (cfm_unet)."""

    def __init__(self, H, W, max_batch=1, seed=0):
        self.H, self.W, self.max_batch = H, W, max_batch
        self.smooth = 0
        self.coarsen = 1
        self.n = lib.cfm_unet_num_params()
        h = ctypes.c_void_p()
        check("cfm_unet_create", lib.cfm_unet_create(H, W, max_batch, seed, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_unet_destroy(self.h)
            self.h = None

    __del__ = close

    def params(self):
        t = np.empty(self.n, np.float32)
        check("cfm_unet_get_params", lib.cfm_unet_get_params(self.h, _ptr(t)))
        return t

    def set_params(self, t):
        t = np.ascontiguousarray(t, np.float32)
        assert t.size == self.n
        check("cfm_unet_set_params", lib.cfm_unet_set_params(self.h, _ptr(t)))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        B = x.shape[0]
        out = np.empty((B, self.H, self.W), np.float32)
        check("cfm_unet_forward_host", lib.cfm_unet_forward_host(self.h, B, _ptr(x), _ptr(out)))
        return out

    ACTIVATIONS = [("h0", 0, 32), ("p1", 1, 32), ("h1", 1, 64), ("p2", 2, 64), ("h2", 2, 128),
                   ("p3", 3, 128), ("h3", 3, 256), ("g3", 3, 128), ("u2", 2, 128), ("g2", 2, 64),
                   ("u1", 1, 64), ("g1", 1, 32), ("u0", 0, 32), ("g0", 0, 32)]

    def activations(self, B):
        """The last forward pass's activations as float32 arrays, by name."""
        out = {}
        for i, (name, lev, ch) in enumerate(self.ACTIVATIONS):
            a = np.empty((B, self.H >> lev, self.W >> lev, ch), np.uint16)
            check("cfm_unet_activation_host", lib.cfm_unet_activation_host(self.h, i, B, _ptr(a)))
            out[name] = from_bf16_bits(a)
        return out

    def train_varcoef(self, nsys, snaps, seed0, epochs, batch, lr=1e-3, smooth=0, coarsen=1):
        """Plain-CG training pairs + Adam on systems of (coarsen H) x (coarsen W);
        returns dict(loss_first, loss_last, data_s, train_s)."""
        v = [ctypes.c_double() for _ in range(4)]
        self.smooth, self.coarsen = smooth, coarsen
        check("cfm_unet_train_varcoef",
              lib.cfm_unet_train_varcoef(self.h, nsys, snaps, seed0, epochs, batch, lr, smooth, coarsen,
                                         *[ctypes.byref(x) for x in v]))
        return dict(zip(("loss_first", "loss_last", "data_s", "train_s"), (x.value for x in v)))

    def set_validation(self, seed, every):
        """Keep the checkpoint whose FPCG solve of a held-out system takes the
        fewest iterations (ties: the earlier epoch)."""
        check("cfm_unet_set_validation", lib.cfm_unet_set_validation(self.h, seed, every))

    def validation(self):
        """(epochs of the kept checkpoint or -1, its validation solve in ms)."""
        ep, ms = ctypes.c_int(), ctypes.c_double()
        check("cfm_unet_validation", lib.cfm_unet_validation(self.h, ctypes.byref(ep), ctypes.byref(ms)))
        return ep.value, ms.value

    def set_training_info(self, smooth, coarsen=1):
        """What a network restored with set_params was trained for."""
        check("cfm_unet_set_training_info", lib.cfm_unet_set_training_info(self.h, smooth, coarsen))
        self.smooth, self.coarsen = smooth, coarsen

    def set_forward_mode(self, mode):
        """UNET_FORWARD_LAYERS (one kernel per layer), UNET_FORWARD_PERSISTENT
        (one persistent kernel) or UNET_FORWARD_AUTO (per layer, the faster);
        same outputs bit for bit."""
        check("cfm_unet_set_forward_mode", lib.cfm_unet_set_forward_mode(self.h, mode))

    def time_forward(self, B=1, iters=20):
        ms = ctypes.c_double()
        check("cfm_unet_time_forward", lib.cfm_unet_time_forward(self.h, B, iters, ctypes.byref(ms)))
        return ms.value

    def time_train_step(self, B=8, iters=10):
        """ms per training step (forward, backward, Adam) on synthetic inputs;
        it changes the weights: use a scratch network."""
        ms = ctypes.c_double()
        check("cfm_unet_time_train_step", lib.cfm_unet_time_train_step(self.h, B, iters, ctypes.byref(ms)))
        return ms.value

    def gradient(self, x, dout):
        x = np.ascontiguousarray(x, np.float32)
        dout = np.ascontiguousarray(dout, np.float32)
        g = np.empty(self.n, np.float32)
        check("cfm_unet_gradient_host", lib.cfm_unet_gradient_host(self.h, x.shape[0], _ptr(x), _ptr(dout), _ptr(g)))
        return g


class FPCG:
    """Flexible PCG with the network as preconditioner (cfm_fpcg)."""

    def __init__(self, S, k, net, maxiter=5000, tol=1e-8, smooth=None, truncation=None, net_period=None,
                 precision=None, delta=0.1):
        self.S, self.net = S, net
        self.k = np.ascontiguousarray(k, np.float64)
        h = ctypes.c_void_p()
        self.maxiter = maxiter
        if smooth is None:
            smooth = getattr(net, "smooth", 0) if net is not None else 0
        check("cfm_fpcg_create", lib.cfm_fpcg_create(S.h, _ptr(self.k), None if net is None else net.h,
                                                     smooth, maxiter, tol, ctypes.byref(h)))
        self.h = h
        if truncation is not None:
            check("cfm_fpcg_set_truncation", lib.cfm_fpcg_set_truncation(self.h, truncation))
        if net_period is not None:
            check("cfm_fpcg_set_network_period", lib.cfm_fpcg_set_network_period(self.h, net_period))
        if precision is not None:
            self.set_precision(precision, delta)

    def set_precision(self, precision, delta=0.1):
        """FP64, or FP32 Krylov vectors with FP64 reliable updates (delta: the
        residual drop that triggers one)."""
        check("cfm_fpcg_set_precision", lib.cfm_fpcg_set_precision(self.h, precision, delta))

    def set_device_loop(self, on):
        """0 (default): one kernel per phase; 1: a single system's iterations
        between network applications in one persistent launch (same values)."""
        check("cfm_fpcg_set_device_loop", lib.cfm_fpcg_set_device_loop(self.h, int(on)))

    def reliable_updates(self):
        """FP64 reliable updates of the last solve (mixed precision)."""
        return lib.cfm_fpcg_reliable_updates(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_fpcg_destroy(self.h)
            self.h = None

    __del__ = close

    def history(self):
        out = np.empty(self.maxiter + 1)
        n = ctypes.c_longlong()
        check("cfm_fpcg_history", lib.cfm_fpcg_history(self.h, _ptr(out), len(out), ctypes.byref(n)))
        return out[:n.value]

    def solve(self, b, allowed=(OK, NOT_CONVERGED)):
        b = np.ascontiguousarray(b, np.float64).reshape(-1)
        x = np.empty_like(b)
        st = Stats()
        check("cfm_fpcg_solve", lib.cfm_fpcg_solve(self.h, _ptr(b), _ptr(x), ctypes.byref(st)), allowed)
        return x, st


class FPCGBatch(FPCG):
    """A batch of 2D systems [(k, b) or k] solved together by the FPCG device
    loop (cfm_fpcg_create_batch): each member embedded in the network's frame
    (or, without a network, the largest member's), its own scalars and stop."""

    def __init__(self, ks, net, maxiter=5000, tol=1e-8, smooth=None, truncation=None, net_period=None,
                 precision=None, delta=0.1):
        self.net, self.maxiter = net, maxiter
        self.ks = [np.ascontiguousarray(k, np.float64) for k in ks]
        self.shapes = [k.shape for k in self.ks]
        nx = np.array([sh[1] for sh in self.shapes], np.int32)
        ny = np.array([sh[0] for sh in self.shapes], np.int32)
        kp = (ctypes.c_void_p * len(self.ks))(*[k.ctypes.data for k in self.ks])
        if smooth is None:
            smooth = getattr(net, "smooth", 0) if net is not None else 0
        h = ctypes.c_void_p()
        check("cfm_fpcg_create_batch", lib.cfm_fpcg_create_batch(len(self.ks), _ptr(nx), _ptr(ny), kp,
                                                                 None if net is None else net.h, smooth,
                                                                 maxiter, tol, ctypes.byref(h)))
        self.h = h
        if truncation is not None:
            check("cfm_fpcg_set_truncation", lib.cfm_fpcg_set_truncation(self.h, truncation))
        if net_period is not None:
            check("cfm_fpcg_set_network_period", lib.cfm_fpcg_set_network_period(self.h, net_period))
        if precision is not None:
            self.set_precision(precision, delta)

    def solve(self, bs, allowed=(OK, NOT_CONVERGED)):
        """bs: one right-hand side per member (its shape).  Returns (xs,
        iterations, status, true relative residuals, stats)."""
        M = len(self.ks)
        bs = [np.ascontiguousarray(b, np.float64).reshape(sh) for b, sh in zip(bs, self.shapes)]
        xs = [np.empty(sh) for sh in self.shapes]
        bp = (ctypes.c_void_p * M)(*[b.ctypes.data for b in bs])
        xp = (ctypes.c_void_p * M)(*[x.ctypes.data for x in xs])
        it = np.empty(M, np.int64)
        stt = np.empty(M, np.int32)
        rr = np.empty(M)
        st = Stats()
        check("cfm_fpcg_solve_batch", lib.cfm_fpcg_solve_batch(self.h, bp, xp, _ptr(it), _ptr(stt), _ptr(rr),
                                                               ctypes.byref(st)), allowed)
        return xs, it, stt, rr, st


class Batch:
    """Many variable-coefficient systems in one persistent launch (cfm_batch).
    systems: list of (k, b) with k of shape (ny, nx) or (nz, ny, nx)."""

    def __init__(self, systems):
        self.n = len(systems)
        dims, nx, ny, nz = [], [], [], []
        self._keep = []
        for k, b in systems:
            k = np.ascontiguousarray(k, np.float64)
            b = np.ascontiguousarray(b, np.float64).reshape(-1)
            assert b.size == k.size
            self._keep += [k, b]
            dims.append(k.ndim)
            nx.append(k.shape[-1])
            ny.append(k.shape[-2])
            nz.append(k.shape[0] if k.ndim == 3 else 1)
        arr = lambda v: np.ascontiguousarray(v, np.int32)
        self.dims, self.nx, self.ny, self.nz = arr(dims), arr(nx), arr(ny), arr(nz)
        kp = (ctypes.c_void_p * self.n)(*[a.ctypes.data for a in self._keep[0::2]])
        bp = (ctypes.c_void_p * self.n)(*[a.ctypes.data for a in self._keep[1::2]])
        h = ctypes.c_void_p()
        check("cfm_batch_create", lib.cfm_batch_create(self.n, _ptr(self.dims), _ptr(self.nx), _ptr(self.ny),
                                                       _ptr(self.nz), kp, bp, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib.cfm_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def set_solver(self, smooth=4, maxiter=20000, tol=1e-8):
        check("cfm_batch_set_solver", lib.cfm_batch_set_solver(self.h, smooth, maxiter, tol))

    def set_precision(self, precision, inner_maxiter=0, inner_tol=0.1):
        """FP64, or FP32 (FP32 PCG with FP64 reliable updates: inner_tol is
        the residual drop that triggers one, inner_maxiter caps the steps
        between two)."""
        check("cfm_batch_set_precision", lib.cfm_batch_set_precision(self.h, precision, inner_maxiter,
                                                                     inner_tol))

    def set_plan(self, thresholds, teams):
        t = np.ascontiguousarray(thresholds, np.int64)
        m = np.ascontiguousarray(teams, np.int32)
        check("cfm_batch_set_plan", lib.cfm_batch_set_plan(self.h, len(t), _ptr(t), _ptr(m)))

    def autotune(self):
        ms = ctypes.c_double()
        check("cfm_batch_autotune", lib.cfm_batch_autotune(self.h, ctypes.byref(ms)))
        return ms.value

    def solve(self, allowed=(OK, NOT_CONVERGED)):
        it = np.empty(self.n, np.int64)
        stt = np.empty(self.n, np.int32)
        rr = np.empty(self.n)
        st = Stats()
        check("cfm_batch_solve", lib.cfm_batch_solve(self.h, _ptr(it), _ptr(stt), _ptr(rr), ctypes.byref(st)),
              allowed)
        return it, stt, rr, st

    def solution(self, i):
        n = int(self.nx[i]) * int(self.ny[i]) * int(self.nz[i])
        x = np.empty(n)
        check("cfm_batch_solution", lib.cfm_batch_solution(self.h, i, _ptr(x)))
        return x


def uneven_systems(n2d, n3d, seed=0, side2d=(64, 512), side3d=(32, 128)):
    """Sizes log-uniform in the given ranges (Philox draws from `seed`) and
    the variable-coefficient problem of each with its own seed."""
    u = uniform(seed, n2d + n3d, 0.0, 1.0)
    out = []
    for i in range(n2d + n3d):
        lo, hi = side2d if i < n2d else side3d
        side = int(round(lo * (hi / lo) ** u[i]))
        shape = (side, side) if i < n2d else (side, side, side)
        k, f = varcoef_problem(shape, seed * 100000 + 1 + i)
        out.append((k, f))
    return out
