/*
 * cfm_oracle.c -- CPU oracle (test infrastructure only; see cfm_oracle.h).
 *
 * Built with -O2 -ffp-contract=off and no fast-math so that every sum is
 * evaluated in source order; fused multiply-adds appear only where they are
 * written as fma(), mirroring the contracted forms of the reference's CUDA
 * expressions (CG/src/common.cu:160-168 `output += alpha * val * x`,
 * :175 `y = a * x + y`).
 */
#include "cfm_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TILE 1024

int orc_max_threads(void) { return omp_get_max_threads(); }

static int nthreads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

/* ------------------------------------------------------------ Jacobi init */

/* Stencil/jacobi2D/src/common.cu:15-26: columns x=0 and x=nx-1 get
 * sin(2.0 * pi * iy / (ny - 1)) with pi rounded to the grid's precision;
 * everything else 0 (cudaMemset at :190-191). */
int orc_jacobi2d_init_f64(int nx, int ny, double *a) {
    if (nx < 3 || ny < 3 || !a) return 1;
    const double pi = 2.0 * asin(1.0);
    memset(a, 0, sizeof(double) * (size_t)nx * ny);
    for (int iy = 0; iy < ny; ++iy) {
        const double y0 = sin(2.0 * pi * (double)iy / (double)(ny - 1));
        a[(size_t)iy * nx] = y0;
        a[(size_t)iy * nx + nx - 1] = y0;
    }
    return 0;
}

int orc_jacobi2d_init_f32(int nx, int ny, float *a) {
    if (nx < 3 || ny < 3 || !a) return 1;
    const float pi = (float)(2.0 * asin(1.0));
    memset(a, 0, sizeof(float) * (size_t)nx * ny);
    for (int iy = 0; iy < ny; ++iy) {
        const float y0 = (float)sin(2.0 * (double)pi * (double)iy / (double)(ny - 1));
        a[(size_t)iy * nx] = y0;
        a[(size_t)iy * nx + nx - 1] = y0;
    }
    return 0;
}

/* problem 0: Stencil/jacobi3D/src/common.cu:15-29 -- only the x=0 face is
 * set, and the ix loop's last write wins: a[z][y][0] = z - y - (nx-1).
 * problem 1: both x faces = sin(2 pi y/(ny-1)) * sin(2 pi z/(nz-1)). */
#define ORC_J3_INIT(T, NAME)                                                               \
    int NAME(int nx, int ny, int nz, int problem, T *a) {                                  \
        if (nx < 3 || ny < 3 || nz < 3 || !a) return 1;                                    \
        const double pi = 2.0 * asin(1.0);                                                 \
        memset(a, 0, sizeof(T) * (size_t)nx * ny * nz);                                    \
        for (int iz = 0; iz < nz; ++iz)                                                    \
            for (int iy = 0; iy < ny; ++iy) {                                              \
                size_t row = ((size_t)iz * ny + iy) * nx;                                  \
                if (problem == 0) {                                                        \
                    a[row] = (T)((T)iz - (T)iy) - (T)(nx - 1);                             \
                } else {                                                                   \
                    double v = sin(2.0 * pi * (double)iy / (double)(ny - 1)) *             \
                               sin(2.0 * pi * (double)iz / (double)(nz - 1));              \
                    a[row] = (T)v;                                                         \
                    a[row + nx - 1] = (T)v;                                                \
                }                                                                          \
            }                                                                              \
        return 0;                                                                          \
    }
ORC_J3_INIT(double, orc_jacobi3d_init_f64)
ORC_J3_INIT(float, orc_jacobi3d_init_f32)

/* ---------------------------------------------------------- Jacobi sweeps */

/* 2D sweep, Stencil/jacobi2D/src/common.cu:28-42: 0.25 (a double literal)
 * times (((E + W) + N) + S) in the grid type; then the periodic halo copies of
 * :234-242 (row 0 <- row ny-2, row ny-1 <- row 1, full rows), then swap. */
#define ORC_J2(T, NAME, SCALE)                                                             \
    int NAME(int nx, int ny, int niter, const T *in, T *out, int threads) {               \
        if (nx < 3 || ny < 3 || niter < 0 || !in || !out) return 1;                        \
        size_t N = (size_t)nx * ny;                                                        \
        T *a = (T *)malloc(sizeof(T) * N), *b = (T *)malloc(sizeof(T) * N);                \
        if (!a || !b) { free(a); free(b); return 1; }                                      \
        memcpy(a, in, sizeof(T) * N);                                                      \
        memcpy(b, in, sizeof(T) * N);                                                      \
        for (int it = 0; it < niter; ++it) {                                               \
            _Pragma("omp parallel for num_threads(nthreads(threads)) schedule(static)")     \
            for (int iy = 1; iy < ny - 1; ++iy) {                                          \
                const T *r = a + (size_t)iy * nx;                                          \
                T *w = b + (size_t)iy * nx;                                                \
                for (int ix = 1; ix < nx - 1; ++ix) {                                      \
                    T s = r[ix + 1] + r[ix - 1];                                           \
                    s = s + r[ix + nx];                                                    \
                    s = s + r[ix - nx];                                                    \
                    w[ix] = SCALE(s);                                                      \
                }                                                                          \
            }                                                                              \
            memcpy(b, b + (size_t)(ny - 2) * nx, sizeof(T) * nx);                          \
            memcpy(b + (size_t)(ny - 1) * nx, b + (size_t)nx, sizeof(T) * nx);             \
            T *t = a; a = b; b = t;                                                        \
        }                                                                                  \
        memcpy(out, a, sizeof(T) * N);                                                     \
        free(a); free(b);                                                                  \
        return 0;                                                                          \
    }
#define ORC_SCALE_Q64(s) (0.25 * (s))
#define ORC_SCALE_Q32(s) ((float)(0.25 * (double)(s)))
ORC_J2(double, orc_jacobi2d_f64, ORC_SCALE_Q64)
ORC_J2(float, orc_jacobi2d_f32, ORC_SCALE_Q32)

/* 3D sweep, Stencil/jacobi3D/src/common.cu:31-57: (real(1)/real(6)) times
 * ((((( E + W) + N) + S) + T) + B), neighbours in the order ix+1, ix-1, iy+1,
 * iy-1, iz+1, iz-1; then the halo-plane copies of :198-207 (plane 0 <- plane
 * nz-2, plane nz-1 <- plane 1, full planes).  With periodic_y the rows
 * y=0 <- y=ny-2 and y=ny-1 <- y=1 of every interior plane are copied first
 * (full rows), so the plane copies carry the y halos into the z halos. */
#define ORC_J3(T, NAME)                                                                    \
    int NAME(int nx, int ny, int nz, int niter, int periodic_y, const T *in, T *out,      \
             int threads) {                                                                \
        if (nx < 3 || ny < 3 || nz < 3 || niter < 0 || !in || !out) return 1;              \
        const size_t P = (size_t)nx * ny, N = P * nz;                                      \
        const T c6 = (T)1 / (T)6;                                                          \
        T *a = (T *)malloc(sizeof(T) * N), *b = (T *)malloc(sizeof(T) * N);                \
        if (!a || !b) { free(a); free(b); return 1; }                                      \
        memcpy(a, in, sizeof(T) * N);                                                      \
        memcpy(b, in, sizeof(T) * N);                                                      \
        for (int it = 0; it < niter; ++it) {                                               \
            _Pragma("omp parallel for num_threads(nthreads(threads)) schedule(static)")     \
            for (int iz = 1; iz < nz - 1; ++iz) {                                          \
                for (int iy = 1; iy < ny - 1; ++iy) {                                      \
                    const T *r = a + (size_t)iz * P + (size_t)iy * nx;                     \
                    T *w = b + (size_t)iz * P + (size_t)iy * nx;                           \
                    for (int ix = 1; ix < nx - 1; ++ix) {                                  \
                        T s = r[ix + 1] + r[ix - 1];                                       \
                        s = s + r[ix + nx];                                                \
                        s = s + r[ix - nx];                                                \
                        s = s + r[ix + P];                                                 \
                        s = s + r[ix - P];                                                 \
                        w[ix] = c6 * s;                                                    \
                    }                                                                      \
                }                                                                          \
                if (periodic_y) {                                                          \
                    T *pl = b + (size_t)iz * P;                                            \
                    memcpy(pl, pl + (size_t)(ny - 2) * nx, sizeof(T) * nx);                \
                    memcpy(pl + (size_t)(ny - 1) * nx, pl + (size_t)nx, sizeof(T) * nx);   \
                }                                                                          \
            }                                                                              \
            memcpy(b, b + (size_t)(nz - 2) * P, sizeof(T) * P);                            \
            memcpy(b + (size_t)(nz - 1) * P, b + P, sizeof(T) * P);                        \
            T *t = a; a = b; b = t;                                                        \
        }                                                                                  \
        memcpy(out, a, sizeof(T) * N);                                                     \
        free(a); free(b);                                                                  \
        return 0;                                                                          \
    }
ORC_J3(double, orc_jacobi3d_f64)
ORC_J3(float, orc_jacobi3d_f32)

/* Timed host baseline: the FP64 3D sweep loop above on the config problem
 * (periodic y and z), timed around the iteration loop only (allocation and
 * initialisation excluded).  Returns loop seconds, or -1 on bad arguments. */
double orc_jacobi3d_bench_f64(int nx, int ny, int nz, int niter, int threads) {
    if (nx < 3 || ny < 3 || nz < 3 || niter < 1) return -1.0;
    const size_t P = (size_t)nx * ny, N = P * nz;
    double *a = (double *)malloc(sizeof(double) * N), *b = (double *)malloc(sizeof(double) * N);
    if (!a || !b) { free(a); free(b); return -1.0; }
    orc_jacobi3d_init_f64(nx, ny, nz, 1, a);
    const int nt = nthreads(threads);
    /* first-touch b with the same static schedule as the sweeps */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int iz = 0; iz < nz; ++iz) memcpy(b + (size_t)iz * P, a + (size_t)iz * P, sizeof(double) * P);
    const double c6 = 1.0 / 6.0;
    const double t0 = omp_get_wtime();
    for (int it = 0; it < niter; ++it) {
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int iz = 1; iz < nz - 1; ++iz) {
            for (int iy = 1; iy < ny - 1; ++iy) {
                const double *r = a + (size_t)iz * P + (size_t)iy * nx;
                double *w = b + (size_t)iz * P + (size_t)iy * nx;
                for (int ix = 1; ix < nx - 1; ++ix) {
                    double s = r[ix + 1] + r[ix - 1];
                    s = s + r[ix + nx];
                    s = s + r[ix - nx];
                    s = s + r[ix + P];
                    s = s + r[ix - P];
                    w[ix] = c6 * s;
                }
            }
            double *pl = b + (size_t)iz * P;
            memcpy(pl, pl + (size_t)(ny - 2) * nx, sizeof(double) * nx);
            memcpy(pl + (size_t)(ny - 1) * nx, pl + (size_t)nx, sizeof(double) * nx);
        }
        memcpy(b, b + (size_t)(nz - 2) * P, sizeof(double) * P);
        memcpy(b + (size_t)(nz - 1) * P, b + P, sizeof(double) * P);
        double *t = a; a = b; b = t;
    }
    const double t1 = omp_get_wtime();
    free(a); free(b);
    return t1 - t0;
}

/* Stencil/jacobi2D/src/common.cu:44-66: rows 1..ny-2, every column, east and
 * west clamped at the x edges, 0.25f * (N + S + E + W), then the same halo
 * rows copies as single_gpu().  The reference is FP32; the FP64 twin runs the
 * same steps in double. */
#define ORC_MIRROR2D(NAME, T)                                                         \
    int NAME(int nx, int ny, int niter, const T *in, T *out, int threads) {           \
        if (nx < 2 || ny < 3 || niter < 0 || !in || !out) return 1;                   \
        size_t N = (size_t)nx * ny;                                                   \
        T *a = (T *)malloc(sizeof(T) * N), *b = (T *)malloc(sizeof(T) * N);           \
        if (!a || !b) { free(a); free(b); return 1; }                                 \
        memcpy(a, in, sizeof(T) * N);                                                 \
        memcpy(b, in, sizeof(T) * N);                                                 \
        for (int it = 0; it < niter; ++it) {                                          \
            _Pragma("omp parallel for num_threads(nthreads(threads)) schedule(static)") \
            for (int iy = 1; iy < ny - 1; ++iy) {                                     \
                const T *r = a + (size_t)iy * nx;                                     \
                T *w = b + (size_t)iy * nx;                                           \
                for (int ix = 0; ix < nx; ++ix) {                                     \
                    T e = r[ix + (ix < nx - 1)];                                      \
                    T wv = r[ix - (ix > 0)];                                          \
                    T s = r[ix + nx] + r[ix - nx];                                    \
                    s = s + e;                                                        \
                    s = s + wv;                                                       \
                    w[ix] = (T)0.25 * s;                                              \
                }                                                                     \
            }                                                                         \
            memcpy(b, b + (size_t)(ny - 2) * nx, sizeof(T) * nx);                     \
            memcpy(b + (size_t)(ny - 1) * nx, b + (size_t)nx, sizeof(T) * nx);        \
            T *t = a; a = b; b = t;                                                   \
        }                                                                             \
        memcpy(out, a, sizeof(T) * N);                                                \
        free(a); free(b);                                                             \
        return 0;                                                                     \
    }
ORC_MIRROR2D(orc_jacobi2d_mirror_f32, float)
ORC_MIRROR2D(orc_jacobi2d_mirror_f64, double)

/* -------------------------------------------------------------------- CG */

/* Reduction tree shared with the GPU kernels: values of one tile of 1024
 * consecutive entries are summed per 32-lane warp by an xor butterfly
 * (offsets 16, 8, 4, 2, 1), the 32 warp sums by the same butterfly.
 * Entries past n contribute +0.0. */
static double tree32(double *v) {
    for (int off = 16; off >= 1; off >>= 1) {
        double t[32];
        for (int l = 0; l < 32; ++l) t[l] = v[l] + v[l ^ off];
        memcpy(v, t, sizeof(t));
    }
    return v[0];
}

static double tile_sum(const double *prod /* 1024 values */) {
    double ws[32];
    for (int w = 0; w < 32; ++w) {
        double v[32];
        memcpy(v, prod + 32 * w, sizeof(v));
        ws[w] = tree32(v);
    }
    return tree32(ws);
}

/* Sum of tile partials: lane t (of 1024) adds partial[t], partial[t+1024], ...
 * in order starting from 0.0, then the 1024 lane values go through tile_sum. */
static double partials_sum(const double *part, long long ntiles) {
    double *lane = (double *)calloc(ORC_TILE, sizeof(double));
    for (int t = 0; t < ORC_TILE; ++t) {
        double acc = 0.0;
        for (long long i = t; i < ntiles; i += ORC_TILE) acc = acc + part[i];
        lane[t] = acc;
    }
    double s = tile_sum(lane);
    free(lane);
    return s;
}

double orc_dot(long long n, const double *a, const double *b, int threads) {
    long long ntiles = (n + ORC_TILE - 1) / ORC_TILE;
    double *part = (double *)malloc(sizeof(double) * (ntiles > 0 ? ntiles : 1));
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (long long t = 0; t < ntiles; ++t) {
        double prod[ORC_TILE];
        for (int l = 0; l < ORC_TILE; ++l) {
            long long i = t * ORC_TILE + l;
            prod[l] = i < n ? a[i] * b[i] : 0.0;
        }
        part[t] = tile_sum(prod);
    }
    double s = partials_sum(part, ntiles);
    free(part);
    return s;
}

/* CG/src/common.cu:150-168 with alpha = 1: output += val * x[col] in row
 * order, contracted to one fma per nonzero; index base subtracted as the
 * reference does for 1-based matrices. */
int orc_spmv(int n, const int *rowptr, const int *col, const double *val, const double *x,
             double *y, int threads) {
    if (n < 0 || !rowptr || !x || !y) return 1;
    const int base = rowptr[0];
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
    for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int j = rowptr[i] - base; j < rowptr[i + 1] - base; ++j)
            acc = fma(val[j], x[col[j] - base], acc);
        y[i] = acc;
    }
    return 0;
}

int orc_cg(int n, const int *rowptr, const int *col, const double *val, const double *b,
           int maxiter, double tol, double *x, long long *iters, double *relres, int threads) {
    if (n <= 0 || !rowptr || !col || !val || !x || maxiter < 0) return 1;
    const int nt = nthreads(threads);
    double *bb = (double *)malloc(sizeof(double) * n);
    double *r = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n);
    double *s = (double *)malloc(sizeof(double) * n);
    double *t = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
        bb[i] = b ? b[i] : 1.0;
        x[i] = 0.0;
    }
    /* r0 = b - A x0 (CG/src/common.cu:448-456): the saxpy r = -1 * ax0 + r */
    orc_spmv(n, rowptr, col, val, x, s, nt);
    for (int i = 0; i < n; ++i) {
        r[i] = fma(-1.0, s[i], bb[i]);
        p[i] = r[i];
    }
    const double bnorm = sqrt(orc_dot(n, bb, bb, nt));
    double gamma0 = orc_dot(n, r, r, nt);
    long long k = 0;
    int status = tol > 0 ? 5 : 0;
    double res = NAN;
    if (tol > 0 && sqrt(gamma0) <= tol * bnorm) status = 0; /* x0 already solves it */
    while (k < maxiter && !(tol > 0 && status == 0)) {
        orc_spmv(n, rowptr, col, val, p, s, nt);
        const double delta = orc_dot(n, p, s, nt);
        const double alpha = gamma0 / delta;
        if (tol > 0 && !(delta > 0.0 && isfinite(alpha))) { status = 4; break; }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) {
            x[i] = fma(alpha, p[i], x[i]);
            r[i] = fma(-alpha, s[i], r[i]);
        }
        double gamma1 = orc_dot(n, r, r, nt);
        ++k;
        if (tol > 0 && sqrt(gamma1) <= tol * bnorm) {
            /* recursive residual says converged: confirm with the true one */
            orc_spmv(n, rowptr, col, val, x, s, nt);
            for (int i = 0; i < n; ++i) t[i] = bb[i] - s[i];
            const double tt = orc_dot(n, t, t, nt);
            if (sqrt(tt) <= tol * bnorm) { status = 0; break; }
            /* drifted: restart from the true residual */
            memcpy(r, t, sizeof(double) * n);
            memcpy(p, t, sizeof(double) * n);
            gamma0 = tt;
            continue;
        }
        const double beta = gamma1 / gamma0;
        if (tol > 0 && !isfinite(beta)) { status = 4; break; }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) p[i] = fma(beta, p[i], r[i]);
        gamma0 = gamma1;
    }
    /* final true relative residual */
    orc_spmv(n, rowptr, col, val, x, s, nt);
    for (int i = 0; i < n; ++i) t[i] = bb[i] - s[i];
    res = sqrt(orc_dot(n, t, t, nt)) / bnorm;
    if (iters) *iters = k;
    if (relres) *relres = res;
    free(bb); free(r); free(p); free(s); free(t);
    return status;
}

/* ------------------------------------------------ operator-generic Krylov */

/* Operator: CSR (kind 0, index base from rowptr[0]) or the matrix-free
 * variable-coefficient stencil (kind 2 / 3) whose row i gives
 *   t = dg[i] x[i]; then t = fma(-w, x_nb, t) for x-1, x+1, y-1, y+1, z-1, z+1
 * with w = we[i-1], we[i], wn[i-nx], wn[i], wt[i-P], wt[i] (neighbours that
 * exist only).  FP32 copies (fp32 = 1) apply the same in float with fmaf. */
typedef struct {
    int kind, n;
    const int *rowptr, *col;
    const double *val;
    int nx, ny, nz;
    const double *we, *wn, *wt, *dg;
    float *val32, *we32, *wn32, *wt32, *dg32;
} orc_op;

static void op_apply(const orc_op *A, const double *x, double *y, int nt) {
    const int n = A->n;
    if (A->kind == 0) {
        orc_spmv(n, A->rowptr, A->col, A->val, x, y, nt);
        return;
    }
    const int nx = A->nx, ny = A->ny, nz = A->nz, P = nx * ny;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < n; ++i) {
        const int ix = i % nx, q = i / nx, iy = q % ny, iz = q / ny;
        double t = A->dg[i] * x[i];
        if (ix > 0) t = fma(-A->we[i - 1], x[i - 1], t);
        if (ix < nx - 1) t = fma(-A->we[i], x[i + 1], t);
        if (iy > 0) t = fma(-A->wn[i - nx], x[i - nx], t);
        if (iy < ny - 1) t = fma(-A->wn[i], x[i + nx], t);
        if (A->kind == 3) {
            if (iz > 0) t = fma(-A->wt[i - P], x[i - P], t);
            if (iz < nz - 1) t = fma(-A->wt[i], x[i + P], t);
        }
        y[i] = t;
    }
}

static void op_apply32(const orc_op *A, const float *x, float *y, int nt) {
    const int n = A->n;
    if (A->kind == 0) {
        const int base = A->rowptr[0];
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) {
            float acc = 0.f;
            for (int j = A->rowptr[i] - base; j < A->rowptr[i + 1] - base; ++j)
                acc = fmaf(A->val32[j], x[A->col[j] - base], acc);
            y[i] = acc;
        }
        return;
    }
    const int nx = A->nx, ny = A->ny, nz = A->nz, P = nx * ny;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < n; ++i) {
        const int ix = i % nx, q = i / nx, iy = q % ny, iz = q / ny;
        float t = A->dg32[i] * x[i];
        if (ix > 0) t = fmaf(-A->we32[i - 1], x[i - 1], t);
        if (ix < nx - 1) t = fmaf(-A->we32[i], x[i + 1], t);
        if (iy > 0) t = fmaf(-A->wn32[i - nx], x[i - nx], t);
        if (iy < ny - 1) t = fmaf(-A->wn32[i], x[i + nx], t);
        if (A->kind == 3) {
            if (iz > 0) t = fmaf(-A->wt32[i - P], x[i - P], t);
            if (iz < nz - 1) t = fmaf(-A->wt32[i], x[i + P], t);
        }
        y[i] = t;
    }
}

/* Tree sum (tiles, then partials) of n precomputed products. */
static double tree_sum(long long n, const double *prod, int nt) {
    long long ntiles = (n + ORC_TILE - 1) / ORC_TILE;
    double *part = (double *)malloc(sizeof(double) * (ntiles > 0 ? ntiles : 1));
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long long t = 0; t < ntiles; ++t) {
        double pr[ORC_TILE];
        for (int l = 0; l < ORC_TILE; ++l) {
            long long i = t * ORC_TILE + l;
            pr[l] = i < n ? prod[i] : 0.0;
        }
        part[t] = tile_sum(pr);
    }
    double s = partials_sum(part, ntiles);
    free(part);
    return s;
}

/* <a, b> of FP32 vectors: FP64 sums of the exact FP32 products. */
static double dot32(int n, const float *a, const float *b, double *scr, int nt) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < n; ++i) scr[i] = (double)a[i] * (double)b[i];
    return tree_sum(n, scr, nt);
}

/* t = b - A x; returns <t, t>. */
static double true_res(const orc_op *A, const double *b, const double *x, double *t, double *s,
                       int nt) {
    op_apply(A, x, s, nt);
    for (int i = 0; i < A->n; ++i) t[i] = b[i] - s[i];
    return orc_dot(A->n, t, t, nt);
}

/* Standard CG: the arithmetic of cg_std_kernel (csrc/krylov.cuh). */
static int krylov_std(const orc_op *A, const double *b, int maxiter, double tol, double *x,
                      long long *iters, int *restarts_out, int nt) {
    const int n = A->n;
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
    double *s = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
        x[i] = 0.0;
        r[i] = fma(-1.0, 0.0, b[i]);
        p[i] = r[i];
    }
    double gamma0 = orc_dot(n, r, r, nt);
    const double bnorm = sqrt(orc_dot(n, b, b, nt));
    const int use_tol = tol > 0;
    const double target = tol * bnorm;
    int status = use_tol ? 5 : 0, restarts = 0;
    long long k = 0;
    if (use_tol && sqrt(gamma0) <= target) status = 0;
    while (k < maxiter && !(use_tol && status == 0)) {
        op_apply(A, p, s, nt);
        const double delta = orc_dot(n, p, s, nt);
        const double alpha = gamma0 / delta;
        if (use_tol && !(delta > 0.0 && isfinite(alpha))) { status = 4; break; }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) {
            x[i] = fma(alpha, p[i], x[i]);
            r[i] = fma(-alpha, s[i], r[i]);
        }
        const double gamma1 = orc_dot(n, r, r, nt);
        ++k;
        if (use_tol && sqrt(gamma1) <= target) {
            const double tt = true_res(A, b, x, t, s, nt);
            if (sqrt(tt) <= target) { status = 0; break; }
            memcpy(r, t, sizeof(double) * n);
            memcpy(p, t, sizeof(double) * n);
            ++restarts;
            gamma0 = tt;
            continue;
        }
        const double beta = gamma1 / gamma0;
        if (use_tol && !isfinite(beta)) { status = 4; break; }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) p[i] = fma(beta, p[i], r[i]);
        gamma0 = gamma1;
    }
    *iters = k;
    *restarts_out = restarts;
    free(r); free(p); free(s); free(t);
    return status;
}

/* Iterations between residual replacements (PIPE_REPLACE in csrc/krylov.cuh). */
#define ORC_PIPE_REPLACE 50

/* Pipelined CG: the arithmetic of cg_pipe_kernel (csrc/krylov.cuh), whose
 * scalar recurrence is the reference's (CG/src/single-stream/pipelined.cu:262-272). */
static int krylov_pipe(const orc_op *A, const double *b, int maxiter, double tol, double *x,
                       long long *iters, int *restarts_out, int nt) {
    const int n = A->n;
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
    double *s = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
    double *z = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n);
    double *wn = malloc(sizeof(double) * n), *q = malloc(sizeof(double) * n);
    double *scr = malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
        x[i] = 0.0;
        t[i] = fma(-1.0, 0.0, b[i]);
    }
    const double bnorm = sqrt(orc_dot(n, b, b, nt));
    double rr, wr;
#define ORC_PIPE_START()                                                   \
    do {                                                                   \
        memcpy(r, t, sizeof(double) * n);                                  \
        op_apply(A, t, w, nt);                                             \
        memset(z, 0, sizeof(double) * n);                                  \
        memset(s, 0, sizeof(double) * n);                                  \
        memset(p, 0, sizeof(double) * n);                                  \
        rr = orc_dot(n, r, r, nt);                                         \
        for (int i_ = 0; i_ < n; ++i_) scr[i_] = w[i_] * r[i_];            \
        wr = tree_sum(n, scr, nt);                                         \
    } while (0)
    ORC_PIPE_START();
    const int use_tol = tol > 0;
    const double target = tol * bnorm;
    int status = use_tol ? 5 : 0, restarts = 0;
    long long k = 0, kk = 0;
    double rr_prev = 0.0, alpha = 0.0;
    for (;;) {
        if (use_tol && sqrt(rr) <= target) {
            const double tt = true_res(A, b, x, t, q, nt);
            if (sqrt(tt) <= target) { status = 0; break; }
            ORC_PIPE_START();
            ++restarts;
            kk = 0;
            continue;
        }
        if (k >= maxiter) break;
        double beta;
        if (kk > 1) {
            beta = rr / rr_prev;
            const double c = (beta / alpha) * rr;
            alpha = rr / (wr - c);
        } else {
            beta = 0.0;
            alpha = rr / wr;
        }
        if (use_tol && !(isfinite(alpha) && alpha > 0.0 && isfinite(beta))) { status = 4; break; }
        op_apply(A, w, q, nt);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int i = 0; i < n; ++i) {
            const double zi = fma(beta, z[i], q[i]);
            const double si = fma(beta, s[i], w[i]);
            const double pi = fma(beta, p[i], r[i]);
            x[i] = fma(alpha, pi, x[i]);
            r[i] = fma(-alpha, si, r[i]);
            wn[i] = fma(-alpha, zi, w[i]);
            z[i] = zi;
            s[i] = si;
            p[i] = pi;
        }
        rr_prev = rr;
        rr = orc_dot(n, r, r, nt);
        for (int i = 0; i < n; ++i) scr[i] = wn[i] * r[i];
        wr = tree_sum(n, scr, nt);
        double *tmp = w; w = wn; wn = tmp;
        ++k;
        ++kk;
        if (use_tol && k < maxiter && k % ORC_PIPE_REPLACE == 0 && !(sqrt(rr) <= target)) {
            /* residual replacement: r = b - A x, w = A r, s = A p, z = A s */
            true_res(A, b, x, t, q, nt);
            op_apply(A, p, s, nt);
            memcpy(r, t, sizeof(double) * n);
            op_apply(A, t, w, nt);
            op_apply(A, s, z, nt);
            rr = orc_dot(n, r, r, nt);
            for (int i = 0; i < n; ++i) scr[i] = w[i] * r[i];
            wr = tree_sum(n, scr, nt);
            ++restarts;
        }
    }
#undef ORC_PIPE_START
    *iters = k;
    *restarts_out = restarts;
    free(r); free(p); free(s); free(t); free(z); free(w); free(wn); free(q); free(scr);
    return status;
}

/* FP32 CG with FP64 reliable updates: the arithmetic of cg_mixed_kernel
 * (csrc/krylov.cuh).  r32 = fl32(r / |b|); the FP32 steps gather in d32;
 * an update (when <r32, r32> <= tol^2, < inner_tol^2 times its largest value
 * since the last update, after inner_maxiter steps, or at maxiter) adds
 * |b| d32 to x in FP64 and replaces r32 by fl32((b - A x) / |b|), keeping
 * p32; beta comes from the replaced residual. */
static int krylov_mixed(const orc_op *A, const double *b, int maxiter, double tol,
                        int inner_maxiter, double inner_tol, double *x, long long *iters,
                        int *updates_out, int nt) {
    const int n = A->n;
    double *t = malloc(sizeof(double) * n), *s = malloc(sizeof(double) * n);
    double *scr = malloc(sizeof(double) * n);
    float *r32 = malloc(sizeof(float) * n), *p32 = malloc(sizeof(float) * n);
    float *s32 = malloc(sizeof(float) * n), *d32 = malloc(sizeof(float) * n);
    for (int i = 0; i < n; ++i) {
        x[i] = 0.0;
        t[i] = fma(-1.0, 0.0, b[i]);
    }
    double tt = orc_dot(n, t, t, nt);
    const double bnorm = sqrt(orc_dot(n, b, b, nt));
    const double target = tol * bnorm;
    int status = 5, updates = 0, since = 0;
    long long k = 0;
    if (sqrt(tt) <= target || bnorm == 0.0) {
        status = sqrt(tt) <= target ? 0 : 5;
    } else {
        const double scale = 1.0 / bnorm, tol2 = tol * tol, delta2 = inner_tol * inner_tol;
        for (int i = 0; i < n; ++i) {
            r32[i] = (float)(t[i] * scale);
            p32[i] = r32[i];
            d32[i] = 0.f;
        }
        double g0 = dot32(n, r32, r32, scr, nt), gmax = g0;
        while (k < maxiter) {
            op_apply32(A, p32, s32, nt);
            const double delta = dot32(n, p32, s32, scr, nt);
            const double alpha = g0 / delta;
            if (!(delta > 0.0 && isfinite(alpha))) { status = 4; break; }
            const float af = (float)alpha;
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int i = 0; i < n; ++i) {
                d32[i] = fmaf(af, p32[i], d32[i]);
                r32[i] = fmaf(-af, s32[i], r32[i]);
            }
            double g1 = dot32(n, r32, r32, scr, nt);
            ++k;
            ++since;
            if (g1 <= tol2 || g1 < delta2 * gmax || k >= maxiter ||
                (inner_maxiter > 0 && since >= inner_maxiter)) {
#pragma omp parallel for num_threads(nt) schedule(static)
                for (int i = 0; i < n; ++i) {
                    x[i] = fma(bnorm, (double)d32[i], x[i]);
                    d32[i] = 0.f;
                }
                tt = true_res(A, b, x, t, s, nt);
                for (int i = 0; i < n; ++i) r32[i] = (float)(t[i] * scale);
                g1 = dot32(n, r32, r32, scr, nt);
                ++updates;
                since = 0;
                gmax = g1;
                if (sqrt(tt) <= target) { status = 0; break; }
                if (k >= maxiter) break;
            } else if (g1 > gmax) {
                gmax = g1;
            }
            const float bf = (float)(g1 / g0);
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int i = 0; i < n; ++i) p32[i] = fmaf(bf, p32[i], r32[i]);
            g0 = g1;
        }
        if (since > 0)
            for (int i = 0; i < n; ++i) x[i] = fma(bnorm, (double)d32[i], x[i]);
    }
    *iters = k;
    *updates_out = updates;
    free(t); free(s); free(scr); free(r32); free(p32); free(s32); free(d32);
    return status;
}

static int krylov_run(orc_op *A, int method, const double *b_in, int maxiter, double tol,
                      int inner_maxiter, double inner_tol, double *x, long long *iters,
                      int *restarts, double *relres, int threads) {
    const int nt = nthreads(threads), n = A->n;
    double *b = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
    double *s = malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) b[i] = b_in ? b_in[i] : 1.0;
    long long k = 0;
    int rs = 0, status;
    if (method == 1) {
        status = krylov_pipe(A, b, maxiter, tol, x, &k, &rs, nt);
    } else if (method == 2) {
        status = krylov_mixed(A, b, maxiter, tol, inner_maxiter,
                              inner_tol > 0 ? inner_tol : 0.1, x, &k, &rs, nt);
    } else {
        status = krylov_std(A, b, maxiter, tol, x, &k, &rs, nt);
    }
    const double bnorm = sqrt(orc_dot(n, b, b, nt));
    const double tt = true_res(A, b, x, t, s, nt);
    if (iters) *iters = k;
    if (restarts) *restarts = rs;
    if (relres) *relres = bnorm > 0 ? sqrt(tt) / bnorm : sqrt(tt);
    free(b); free(t); free(s);
    return status;
}

static float *to_f32(const double *a, size_t n) {
    float *o = malloc(sizeof(float) * (n ? n : 1));
    for (size_t i = 0; i < n; ++i) o[i] = (float)a[i];
    return o;
}

int orc_krylov_csr(int n, const int *rowptr, const int *col, const double *val, int method,
                   const double *b, int maxiter, double tol, int inner_maxiter, double inner_tol,
                   double *x, long long *iters, int *restarts, double *relres, int threads) {
    if (n <= 0 || !rowptr || !col || !val || !x || maxiter < 0 || method < 0 || method > 2) return 1;
    orc_op A;
    memset(&A, 0, sizeof(A));
    A.kind = 0;
    A.n = n;
    A.rowptr = rowptr;
    A.col = col;
    A.val = val;
    const long long nnz = rowptr[n] - rowptr[0];
    A.val32 = to_f32(val, (size_t)nnz);
    const int st = krylov_run(&A, method, b, maxiter, tol, inner_maxiter, inner_tol, x, iters,
                              restarts, relres, threads);
    free(A.val32);
    return st;
}

static void stencil_op(orc_op *A, int dims, int nx, int ny, int nz, const double *we,
                       const double *wn, const double *wt, const double *dg) {
    memset(A, 0, sizeof(*A));
    A->kind = dims;
    A->nx = nx;
    A->ny = ny;
    A->nz = dims == 3 ? nz : 1;
    A->n = nx * ny * A->nz;
    A->we = we;
    A->wn = wn;
    A->wt = wt;
    A->dg = dg;
}

int orc_stencil_apply(int dims, int nx, int ny, int nz, const double *we, const double *wn,
                      const double *wt, const double *dg, const double *x, double *y,
                      int threads) {
    if ((dims != 2 && dims != 3) || nx < 1 || ny < 1 || !x || !y) return 1;
    orc_op A;
    stencil_op(&A, dims, nx, ny, nz, we, wn, wt, dg);
    op_apply(&A, x, y, nthreads(threads));
    return 0;
}

int orc_krylov_stencil(int dims, int nx, int ny, int nz, const double *we, const double *wn,
                       const double *wt, const double *dg, int method, const double *b,
                       int maxiter, double tol, int inner_maxiter, double inner_tol, double *x,
                       long long *iters, int *restarts, double *relres, int threads) {
    if ((dims != 2 && dims != 3) || nx < 1 || ny < 1 || !x || maxiter < 0 || method < 0 ||
        method > 2)
        return 1;
    orc_op A;
    stencil_op(&A, dims, nx, ny, nz, we, wn, wt, dg);
    const size_t n = (size_t)A.n;
    A.we32 = to_f32(we, n);
    A.wn32 = to_f32(wn, n);
    A.wt32 = dims == 3 ? to_f32(wt, n) : NULL;
    A.dg32 = to_f32(dg, n);
    const int st = krylov_run(&A, method, b, maxiter, tol, inner_maxiter, inner_tol, x, iters,
                              restarts, relres, threads);
    free(A.we32); free(A.wn32); free(A.wt32); free(A.dg32);
    return st;
}

/* ------------------------------------------------------------------ FPCG */

/* Flexible PCG on the 2D variable-coefficient stencil, the device loop of
 * the learned-preconditioner solver (csrc/fpcg.cu) with the identity in
 * place of the network, step for step: truncated FCG(m), the preconditioner
 * z = J(z0 + c P R r1) (z0 = J(0) by `smooth` damped Jacobi sweeps in FP32,
 * r1 = r - A z0, R the f x f block mean, P its piecewise-constant
 * prolongation, c = <P y, r1> / <P y, A P y>), FP64 Krylov vectors or
 * (mixed) FP32 ones with FP64 reliable updates.  Dots are the GPU's trees:
 * rows in 1024-row tiles, the smoothing kernels' dots in 32 x 32-cell tiles.
 * Has no reference counterpart (the reference's CG is unpreconditioned). */
#define FPO_TILE 32
#define FPO_STALL 200
#define FPO_OMEGA 0.8

typedef struct {
    int nx, ny, n, f, ncx, nc, smooth, m, ring, mixed, tx2, nt1, nt2;
    const double *we, *wn, *dg, *b;
    orc_op A;  /* FP64 and FP32 operator */
    float *wd;
    double delta2, *scr, *part1, *part2;
} fpo_ctx;

/* 1024-row tile partials of v, summed as the GPU's partial slots. */
static double fpo_sum1(fpo_ctx *c, const double *v) {
    for (int t = 0; t < c->nt1; ++t) {
        double pr[ORC_TILE];
        for (int l = 0; l < ORC_TILE; ++l) {
            const long long i = (long long)t * ORC_TILE + l;
            pr[l] = i < c->n ? v[i] : 0.0;
        }
        c->part1[t] = tile_sum(pr);
    }
    return partials_sum(c->part1, c->nt1);
}

/* 32 x 32-cell tile partials of v (cells in row-major order within a tile,
 * tiles row-major), summed as the GPU's partial slots. */
static double fpo_sum2(fpo_ctx *c, const double *v) {
    for (int t = 0; t < c->nt2; ++t) {
        const int x0 = (t % c->tx2) * FPO_TILE, y0 = (t / c->tx2) * FPO_TILE;
        double pr[ORC_TILE];
        for (int ly = 0; ly < FPO_TILE; ++ly)
            for (int lx = 0; lx < FPO_TILE; ++lx) {
                const int gx = x0 + lx, gy = y0 + ly;
                pr[ly * FPO_TILE + lx] = (gx < c->nx && gy < c->ny) ? v[(size_t)gy * c->nx + gx] : 0.0;
            }
        c->part2[t] = tile_sum(pr);
    }
    return partials_sum(c->part2, c->nt2);
}

/* `sweeps` damped Jacobi sweeps in FP32 on A z = r from z (in place). */
static void fpo_sweeps(fpo_ctx *c, const float *r, float *z, float *tmp, int sweeps) {
    for (int s = 0; s < sweeps; ++s) {
        op_apply32(&c->A, z, tmp, 1);
        for (int i = 0; i < c->n; ++i) tmp[i] = fmaf(c->wd[i], r[i] - tmp[i], z[i]);
        memcpy(z, tmp, sizeof(float) * c->n);
    }
}

typedef struct {
    double ps[9], target, best_rr, gmax;
    long long k, best_k;
    int done, par, pending, updates;
} fpo_state;

int orc_fpcg2d(int nx, int ny, const double *we, const double *wn, const double *dg,
               const double *b, int f, int smooth, int m, int mixed, double delta, int maxiter,
               double tol, double *x, long long *iters, int *updates, int *done_out) {
    if (nx < 1 || ny < 1 || !we || !wn || !dg || !b || !x || (f != 1 && f != 2) || nx % f ||
        ny % f || smooth < 0 || smooth > 8 || m < 1 || m > 8 || maxiter < 1)
        return 1;
    fpo_ctx c;
    memset(&c, 0, sizeof(c));
    c.nx = nx; c.ny = ny; c.n = nx * ny; c.f = f; c.ncx = nx / f; c.nc = c.n / (f * f);
    c.smooth = smooth; c.m = m; c.ring = m + 1; c.mixed = mixed;
    c.we = we; c.wn = wn; c.dg = dg; c.b = b;
    c.delta2 = delta * delta;
    c.tx2 = (nx + FPO_TILE - 1) / FPO_TILE;
    c.nt1 = (c.n + ORC_TILE - 1) / ORC_TILE;
    c.nt2 = c.tx2 * ((ny + FPO_TILE - 1) / FPO_TILE);
    const size_t n = (size_t)c.n;
    stencil_op(&c.A, 2, nx, ny, 1, we, wn, NULL, dg);
    c.A.we32 = to_f32(we, n);
    c.A.wn32 = to_f32(wn, n);
    c.A.dg32 = to_f32(dg, n);
    c.wd = (float *)malloc(sizeof(float) * n);
    for (size_t i = 0; i < n; ++i) c.wd[i] = (float)(FPO_OMEGA / (double)c.A.dg32[i]);
    c.scr = (double *)malloc(sizeof(double) * n * 3);
    c.part1 = (double *)malloc(sizeof(double) * c.nt1);
    c.part2 = (double *)malloc(sizeof(double) * c.nt2);
    double *r = (double *)calloc(n, sizeof(double)), *z = (double *)calloc(n, sizeof(double));
    double *za = (double *)calloc(n, sizeof(double)), *r1 = (double *)calloc(n, sizeof(double));
    double *pring = (double *)calloc(n * c.ring, sizeof(double));
    double *sring = (double *)calloc(n * c.ring, sizeof(double));
    float *r32 = (float *)calloc(n, sizeof(float)), *z32 = (float *)calloc(n, sizeof(float));
    float *p32 = (float *)calloc(n * c.ring, sizeof(float)), *s32 = (float *)calloc(n * c.ring, sizeof(float));
    float *d32[2] = {(float *)calloc(n, sizeof(float)), (float *)calloc(n, sizeof(float))};
    double *xm[2] = {(double *)calloc(n, sizeof(double)), (double *)calloc(n, sizeof(double))};
    float *rf = (float *)malloc(sizeof(float) * n), *zf = (float *)malloc(sizeof(float) * n);
    float *tf = (float *)malloc(sizeof(float) * n), *yv = (float *)malloc(sizeof(float) * c.nc);
    double *v1 = c.scr, *v2 = c.scr + n, *v3 = c.scr + 2 * n;
    fpo_state S;
    memset(&S, 0, sizeof(S));
    double RR, BB, TT = 0.0, PR = 0.0;
    double ZS[8];

    /* init (k_fp_init / k_fpm_init) */
    for (size_t i = 0; i < n; ++i) {
        x[i] = 0.0;
        v1[i] = b[i] * b[i];
        if (mixed) {
            r32[i] = (float)b[i];
            v2[i] = (double)r32[i] * (double)r32[i];
        } else {
            r[i] = b[i];
            v2[i] = v1[i];
        }
    }
    BB = fpo_sum1(&c, v1);
    RR = fpo_sum1(&c, v2);
    S.best_rr = 1e300;
    S.target = -tol;

    int first = 1;
    for (;;) {
        if (!first) {
            /* s = A p; <p, s> (k_fp_spmv / k_fpm_spmv) */
            const int slot = (int)(S.k % c.ring);
            double *p = pring + (size_t)slot * n, *sv = sring + (size_t)slot * n;
            float *pf = p32 + (size_t)slot * n, *sf = s32 + (size_t)slot * n;
            if (mixed) {
                op_apply32(&c.A, pf, sf, 1);
                for (size_t i = 0; i < n; ++i) v1[i] = (double)pf[i] * (double)sf[i];
            } else {
                op_apply(&c.A, p, sv, 1);
                for (size_t i = 0; i < n; ++i) v1[i] = p[i] * sv[i];
            }
            const double ps = fpo_sum1(&c, v1);
            /* alpha = <p, r> / <p, s>; updates (k_fp_update / k_fpm_update) */
            const double alpha = ps != 0.0 ? PR / ps : 0.0;
            if (mixed) {
                const float af = (float)alpha;
                float *d = d32[S.par];
                for (size_t i = 0; i < n; ++i) {
                    d[i] = fmaf(af, pf[i], d[i]);
                    r32[i] = fmaf(-af, sf[i], r32[i]);
                    v1[i] = (double)r32[i] * (double)r32[i];
                }
            } else {
                for (size_t i = 0; i < n; ++i) {
                    x[i] = fma(alpha, p[i], x[i]);
                    r[i] = fma(-alpha, sv[i], r[i]);
                    v1[i] = r[i] * r[i];
                }
            }
            RR = fpo_sum1(&c, v1);
            S.ps[slot] = ps;
            /* reliable update (k_fpm_reliable) */
            if (mixed && (RR <= S.target * S.target || RR < c.delta2 * S.gmax)) {
                const double *xo = xm[S.par];
                const float *d = d32[S.par];
                for (size_t i = 0; i < n; ++i) v3[i] = xo[i] + (double)d[i];
                op_apply(&c.A, v3, v2, 1);
                for (size_t i = 0; i < n; ++i) {
                    const double ti = b[i] - v2[i];
                    r32[i] = (float)ti;
                    xm[S.par ^ 1][i] = v3[i];
                    d32[S.par ^ 1][i] = 0.f;
                    v1[i] = ti * ti;
                    v2[i] = (double)r32[i] * (double)r32[i];
                }
                TT = fpo_sum1(&c, v1);
                RR = fpo_sum1(&c, v2);
                S.pending = 1;
            }
        }
        /* k_fp_pre: state, z0 = J(0), r1 = r - A z0, R r1 */
        if (!first) S.k += 1;
        if (S.target < 0) S.target = -S.target * sqrt(BB);
        if (!mixed) {
            if (sqrt(RR) <= S.target) S.done = 1;
        } else if (S.pending) {
            S.par ^= 1;
            S.pending = 0;
            S.updates += 1;
            S.gmax = RR;
            if (sqrt(TT) <= S.target) S.done = 1;
        } else if (RR > S.gmax) {
            S.gmax = RR;
        }
        if (RR < S.best_rr) {
            S.best_rr = RR;
            S.best_k = S.k;
        } else if (S.k - S.best_k > FPO_STALL) {
            S.done = 2;
        }
        if (S.k >= maxiter && !S.done) S.done = 2;
        for (size_t i = 0; i < n; ++i) {
            rf[i] = mixed ? r32[i] : (float)r[i];
            zf[i] = smooth > 0 ? c.wd[i] * rf[i] : 0.f;
        }
        if (smooth > 1) fpo_sweeps(&c, rf, zf, tf, smooth - 1);
        op_apply32(&c.A, zf, tf, 1);
        for (size_t i = 0; i < n; ++i) {
            r1[i] = (double)(rf[i] - tf[i]);
            za[i] = (double)zf[i];
        }
        for (int ic = 0; ic < c.nc; ++ic) {  /* R r1 (the identity in place of the network) */
            const int cx = ic % c.ncx, cy = ic / c.ncx;
            double sum = 0;
            for (int dy = 0; dy < f; ++dy)
                for (int dx = 0; dx < f; ++dx) sum += r1[(size_t)(cy * f + dy) * nx + cx * f + dx];
            yv[ic] = (float)(sum / (f * f));
        }
        /* k_fp_ydots: <P y, r1>, <P y, A P y> */
        for (int i = 0; i < c.n; ++i) {
            const int ix = i % nx, iy = i / nx, cx = ix / f, cy = iy / f;
            const double zi = (double)yv[cy * c.ncx + cx];
            double t = dg[i] * zi;
            if (ix > 0) t = fma(-we[i - 1], (double)yv[cy * c.ncx + (ix - 1) / f], t);
            if (ix < nx - 1) t = fma(-we[i], (double)yv[cy * c.ncx + (ix + 1) / f], t);
            if (iy > 0) t = fma(-wn[i - nx], (double)yv[((iy - 1) / f) * c.ncx + cx], t);
            if (iy < ny - 1) t = fma(-wn[i], (double)yv[((iy + 1) / f) * c.ncx + cx], t);
            v1[i] = zi * r1[i];
            v2[i] = zi * t;
        }
        const double yr = fpo_sum1(&c, v1), yay = fpo_sum1(&c, v2);
        /* k_fp_post: z = J(z0 + c P y); <z, s_j> */
        const double cc = yay > 0 ? yr / yay : 0.0;
        for (int i = 0; i < c.n; ++i) {
            const int ix = i % nx, iy = i / nx;
            const double yi = (double)yv[(iy / f) * c.ncx + ix / f];
            zf[i] = (float)(cc != 0.0 ? fma(cc, yi, za[i]) : za[i]);
        }
        fpo_sweeps(&c, rf, zf, tf, smooth);
        for (size_t i = 0; i < n; ++i) {
            z[i] = (double)zf[i];
            z32[i] = zf[i];
        }
        const int k = (int)S.k, nj = k < m ? k : m;
        for (int j = 0; j < nj; ++j) {
            const size_t off = (size_t)((k - 1 - j) % c.ring) * n;
            for (size_t i = 0; i < n; ++i)
                v1[i] = mixed ? (double)z32[i] * (double)s32[off + i] : z[i] * sring[off + i];
            ZS[j] = fpo_sum2(&c, v1);
        }
        /* k_fp_dir: p_k = z - sum_j beta_j p_{k-1-j}; <p, r> */
        double beta[8];
        for (int j = 0; j < nj; ++j) {
            const double ps = S.ps[(k - 1 - j) % c.ring];
            beta[j] = ps != 0.0 ? ZS[j] / ps : 0.0;
        }
        const size_t out = (size_t)(k % c.ring) * n;
        for (size_t i = 0; i < n; ++i) {
            if (mixed) {
                float pi = z32[i];
                for (int j = 0; j < nj; ++j)
                    pi = fmaf(-(float)beta[j], p32[(size_t)((k - 1 - j) % c.ring) * n + i], pi);
                p32[out + i] = pi;
                v1[i] = (double)pi * (double)r32[i];
            } else {
                double pi = z[i];
                for (int j = 0; j < nj; ++j) pi = fma(-beta[j], pring[(size_t)((k - 1 - j) % c.ring) * n + i], pi);
                pring[out + i] = pi;
                v1[i] = pi * r[i];
            }
        }
        PR = fpo_sum1(&c, v1);
        if (!first && S.done) break;
        first = 0;
    }
    if (mixed)
        for (size_t i = 0; i < n; ++i) x[i] = xm[S.par][i] + (double)d32[S.par][i];
    if (iters) *iters = S.k;
    if (updates) *updates = S.updates;
    if (done_out) *done_out = S.done;
    free(c.A.we32); free(c.A.wn32); free(c.A.dg32); free(c.wd); free(c.scr); free(c.part1);
    free(c.part2); free(r); free(z); free(za); free(r1); free(pring); free(sring); free(r32);
    free(z32); free(p32); free(s32); free(d32[0]); free(d32[1]); free(xm[0]); free(xm[1]);
    free(rf); free(zf); free(tf); free(yv);
    return 0;
}
