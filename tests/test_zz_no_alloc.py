"""cfm_cg_solve_noalloc: CG for callers that cannot allocate device memory.

Some hosts of this library cannot call cudaMalloc at solve time: a framework
that owns the device memory through its own pool or allocator, a process
that reserves all of its memory up front, or a caller for whom an
allocation (which can synchronise the device) is not allowed at that point.
cfm_cg_solve_noalloc serves them: the caller passes its own device matrix
and vectors, and the solver's working vectors live in a fixed array inside
the library (CFM_CG_NOALLOC_MAX_N rows at most).

The GPU test checks, through the C ABI, that two calls in a row give the
same x and iteration count as the allocating entry point (cfm_cg_solve with
the persistent kernel): bit-for-bit, the tolerance every CG parity test here
uses, because both run the same kernel and reduction tree.  The file is
named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import cfm

MAX_N = 262144  # CFM_CG_NOALLOC_MAX_N in include/cfm.h


def _call(n, nnz, rowptr, col, val, b, x, maxiter, tol, stream=None):
    st = cfm.Stats()
    s = cfm.lib.cfm_cg_solve_noalloc(n, nnz, ctypes.c_void_p(rowptr), ctypes.c_void_p(col),
                                     ctypes.c_void_p(val), ctypes.c_void_p(b), ctypes.c_void_p(x),
                                     maxiter, tol, ctypes.c_void_p(stream), ctypes.byref(st))
    return s, st


def test_noalloc_rejects_sizes_beyond_the_fixed_array():
    # argument checks come before any CUDA call, so this runs without a GPU
    s, _ = _call(MAX_N + 1, 7 * (MAX_N + 1), 16, 16, 16, None, 16, 10, 1e-8)
    assert s == cfm.BAD_ARG
    assert b"CFM_CG_NOALLOC_MAX_N" in cfm.lib.cfm_last_error()
    s, _ = _call(0, 0, 16, 16, 16, None, 16, 10, 1e-8)
    assert s == cfm.BAD_ARG


def test_noalloc_rejects_b_aliasing_x():
    # the solve zeroes x before it reads b again, so b == x is refused up
    # front (before any CUDA call: no GPU needed)
    s, _ = _call(1000, 7000, 16, 16, 16, 32, 32, 10, 1e-8)
    assert s == cfm.BAD_ARG
    assert b"b and x" in cfm.lib.cfm_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("g", [24, 64])
def test_noalloc_matches_allocating_cg_two_calls(g):
    import torch

    rowptr, col, val = cfm.poisson3d(g)
    n, nnz = len(rowptr) - 1, len(val)
    assert n <= MAX_N
    A = cfm.CSR(rowptr, col, val)
    b1 = A.spmv(cfm.uniform(0, n))
    b2 = A.spmv(cfm.uniform(1, n))
    want = [cfm.CG(A, cfm.CG_PERSISTENT, 20000, 1e-8).solve(b) for b in (b1, b2)]

    dev = torch.device("cuda", 0)
    d_rowptr = torch.from_numpy(rowptr).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    for b, (x_want, st_want) in zip((b1, b2), want):
        d_b = torch.from_numpy(b).to(dev)
        d_x = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        s, st = _call(n, nnz, d_rowptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                      d_b.data_ptr(), d_x.data_ptr(), 20000, 1e-8, stream.cuda_stream)
        assert s == cfm.OK, cfm.lib.cfm_last_error()
        assert st.status == cfm.OK == st_want.status
        assert st.iterations == st_want.iterations
        np.testing.assert_array_equal(d_x.cpu().numpy(), x_want)
        assert st.residual <= 1e-8
        assert st.residual == pytest.approx(st_want.residual, rel=1e-12, abs=1e-20)
