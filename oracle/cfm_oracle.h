/*
 * cfm_oracle.h -- CPU oracle for the solver hot path.  TEST INFRASTRUCTURE
 * ONLY: used by tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py as the checker and the timed host
 * baseline.  The product library (libcfm.so) never links or calls it.
 *
 * Each function restates the reference's single-GPU arithmetic in plain C
 * (OpenMP over rows/planes, which does not change any result):
 *  - Jacobi: Stencil/jacobi2D/src/common.cu:28-42,154-273 and
 *    Stencil/jacobi3D/src/common.cu:31-57,110-239 (compute interior,
 *    copy the periodic halo rows/planes, swap).
 *  - CG: CG/src/common.cu:399-538 (standard CG, alpha = gamma0/delta,
 *    beta = gamma1/gamma0) with CG/src/common.cu:150-184 for SpMV/axpy and
 *    CG/src/common.cu:357-389 for the dot products, reduced in a fixed tree
 *    (tiles of 1024, warp-xor trees) instead of the reference's atomicAdd.
 *
 * Parity pin: the Jacobi FP32 restatement is checked bit-for-bit against
 * grids written by the reference's own single_gpu() (oracle/ref/, fixtures
 * in tests/golden/ref_jacobi*.npz).  The CG restatement is checked against x
 * written by the reference's own SingleGPUDiscreteStandard::run_single_gpu()
 * (CG/src/common.cu compiled unmodified with oracle/ref/shim standing in for
 * the NVSHMEM calls of its multi-GPU kernels; fixtures
 * tests/golden/ref_cg_*.npz) to 1e-12 relative -- not bit for bit, since the
 * reference sums its dots with atomicAdd in arrival order -- and cross-
 * checked against SciPy and manufactured solutions.
 */
#ifndef CFM_ORACLE_H
#define CFM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Initial grids (problem 0 = reference, 1 = config), see cfm.h. */
int orc_jacobi2d_init_f64(int nx, int ny, double *a);
int orc_jacobi2d_init_f32(int nx, int ny, float *a);
int orc_jacobi3d_init_f64(int nx, int ny, int nz, int problem, double *a);
int orc_jacobi3d_init_f32(int nx, int ny, int nz, int problem, float *a);

/* niter reference sweeps from grid `in` (not modified); result into `out`.
 * threads <= 0: OpenMP default. */
int orc_jacobi2d_f64(int nx, int ny, int niter, const double *in, double *out, int threads);
int orc_jacobi2d_f32(int nx, int ny, int niter, const float *in, float *out, int threads);
int orc_jacobi3d_f64(int nx, int ny, int nz, int niter, int periodic_y, const double *in,
                     double *out, int threads);
int orc_jacobi3d_f32(int nx, int ny, int nz, int niter, int periodic_y, const float *in,
                     float *out, int threads);
/* Timed host baseline: niter FP64 sweeps of the 3D config problem; returns
 * the seconds of the sweep loop alone (-1 on bad arguments). */
double orc_jacobi3d_bench_f64(int nx, int ny, int nz, int niter, int threads);
/* The reference's PERKS mirror-boundary sweep (Stencil/jacobi2D/src/common.cu:44-66),
 * FP32 (and its FP64 twin), all x columns updated with clamped east/west neighbours. */
int orc_jacobi2d_mirror_f32(int nx, int ny, int niter, const float *in, float *out, int threads);
int orc_jacobi2d_mirror_f64(int nx, int ny, int niter, const double *in, double *out, int threads);

/* Deterministic dot product (the tile tree the GPU uses). */
double orc_dot(long long n, const double *a, const double *b, int threads);

/* Standard CG.  b == NULL -> ones.  x0 = 0.  tol <= 0: exactly maxiter
 * iterations (reference).  Returns 0 converged / fixed count done,
 * 4 breakdown, 5 not converged.  iters, relres (true FP64 relative residual)
 * optional. */
int orc_cg(int n, const int *rowptr, const int *col, const double *val, const double *b,
           int maxiter, double tol, double *x, long long *iters, double *relres, int threads);

/* y = A x (index base from rowptr[0], fma accumulation in row order). */
int orc_spmv(int n, const int *rowptr, const int *col, const double *val, const double *x,
             double *y, int threads);

/* Operator-generic persistent-solver restatements (csrc/krylov.cuh):
 * method 0 standard CG, 1 pipelined CG, 2 FP32 CG with FP64 reliable
 * updates (inner_maxiter 0 -> no cap between updates, inner_tol 0 -> 0.1,
 * the residual drop that triggers one).  b == NULL -> ones, x0 = 0.
 * Returns 0 / 4 breakdown / 5 not converged; iters, restarts (FP64 updates
 * for method 2), relres (true FP64 relative residual) optional. */
int orc_krylov_csr(int n, const int *rowptr, const int *col, const double *val, int method,
                   const double *b, int maxiter, double tol, int inner_maxiter, double inner_tol,
                   double *x, long long *iters, int *restarts, double *relres, int threads);
/* Variable-coefficient stencil (coefficients as cfm_varcoef_coeffs gives them). */
int orc_stencil_apply(int dims, int nx, int ny, int nz, const double *we, const double *wn,
                      const double *wt, const double *dg, const double *x, double *y,
                      int threads);
int orc_krylov_stencil(int dims, int nx, int ny, int nz, const double *we, const double *wn,
                       const double *wt, const double *dg, int method, const double *b,
                       int maxiter, double tol, int inner_maxiter, double inner_tol, double *x,
                       long long *iters, int *restarts, double *relres, int threads);

/* Flexible PCG on the 2D variable-coefficient stencil (the learned-
 * preconditioner solver's device loop, csrc/fpcg.cu) with the identity in
 * place of the network: truncated FCG(m), z = J(z0 + c P R r1) with `smooth`
 * FP32 Jacobi sweeps and f x f coarse cells (f = 1 or 2); FP64 Krylov
 * vectors (mixed = 0) or FP32 ones with FP64 reliable updates at residual
 * drop `delta` (mixed = 1).  x0 = 0.  Returns 0 / 1 bad arguments; iters,
 * updates (FP64 reliable updates) and done (1 converged, 2 stalled / capped)
 * optional. */
int orc_fpcg2d(int nx, int ny, const double *we, const double *wn, const double *dg,
               const double *b, int f, int smooth, int m, int mixed, double delta, int maxiter,
               double tol, double *x, long long *iters, int *updates, int *done);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
