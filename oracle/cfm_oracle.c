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
 * rows copies as single_gpu(). */
int orc_jacobi2d_mirror_f32(int nx, int ny, int niter, const float *in, float *out, int threads) {
    if (nx < 2 || ny < 3 || niter < 0 || !in || !out) return 1;
    size_t N = (size_t)nx * ny;
    float *a = (float *)malloc(sizeof(float) * N), *b = (float *)malloc(sizeof(float) * N);
    if (!a || !b) { free(a); free(b); return 1; }
    memcpy(a, in, sizeof(float) * N);
    memcpy(b, in, sizeof(float) * N);
    for (int it = 0; it < niter; ++it) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
        for (int iy = 1; iy < ny - 1; ++iy) {
            const float *r = a + (size_t)iy * nx;
            float *w = b + (size_t)iy * nx;
            for (int ix = 0; ix < nx; ++ix) {
                float e = r[ix + (ix < nx - 1)];
                float wv = r[ix - (ix > 0)];
                float s = r[ix + nx] + r[ix - nx];
                s = s + e;
                s = s + wv;
                w[ix] = 0.25f * s;
            }
        }
        memcpy(b, b + (size_t)(ny - 2) * nx, sizeof(float) * nx);
        memcpy(b + (size_t)(ny - 1) * nx, b + (size_t)nx, sizeof(float) * nx);
        float *t = a; a = b; b = t;
    }
    memcpy(out, a, sizeof(float) * N);
    free(a); free(b);
    return 0;
}

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
