// Host-side problem generators exported through the C ABI.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cfm.h"
#include "cfm_internal.h"

namespace {

// Philox-4x32-10 (Salmon et al., "Parallel random numbers: as easy as 1, 2,
// 3", SC'11): 10 rounds of the 4x32 S-P network with the published
// multipliers and Weyl key increments.
struct Philox4x32 {
    static constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    static constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    static void round(uint32_t c[4], const uint32_t k[2]) {
        const uint64_t p0 = (uint64_t)M0 * c[0];
        const uint64_t p1 = (uint64_t)M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k[0];
        const uint32_t n2 = hi0 ^ c[3] ^ k[1];
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
    static void block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
        uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
        uint32_t k[2] = {key[0], key[1]};
        for (int r = 0; r < 10; ++r) {
            if (r) {
                k[0] += W0;
                k[1] += W1;
            }
            round(c, k);
        }
        std::memcpy(out, c, sizeof(c));
    }
};

}  // namespace

extern "C" {

// Exposed for the known-answer test of the generator.
int cfm_philox4x32_10(const unsigned int ctr[4], const unsigned int key[2], unsigned int out[4]) {
    CFM_ARG_CHECK(ctr && key && out, "null argument");
    Philox4x32::block(ctr, key, out);
    return CFM_OK;
}

// Entry i uses counter (i / 2, 0, 0, 0) under key (seed lo, seed hi); the
// even entry takes words 0-1, the odd entry words 2-3, as a 53-bit fraction.
int cfm_uniform(unsigned long long seed, long long n, double lo, double hi, double *out) {
    CFM_ARG_CHECK(out || n == 0, "out is null");
    CFM_ARG_CHECK(n >= 0, "n");
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const double span = hi - lo;
    for (long long i = 0; i < n; i += 2) {
        const uint64_t c = (uint64_t)(i / 2);
        const uint32_t ctr[4] = {(uint32_t)c, (uint32_t)(c >> 32), 0u, 0u};
        uint32_t w[4];
        Philox4x32::block(ctr, key, w);
        for (int h = 0; h < 2 && i + h < n; ++h) {
            const uint64_t bits = ((uint64_t)w[2 * h + 1] << 32) | w[2 * h];
            const double u = (double)(bits >> 11) * 0x1.0p-53;
            out[i + h] = lo + u * span;
        }
    }
    return CFM_OK;
}

// Entry i uses counter (i / 2, stream, 0x4e4f524d) under key (seed lo, seed
// hi): words 0-1 give u1 in (0, 1], words 2-3 give u2 in [0, 1), and the
// Box-Muller pair sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2) supplies the
// even and the odd entry.
int cfm_normal(unsigned long long seed, unsigned int stream, long long n, double *out) {
    CFM_ARG_CHECK(out || n == 0, "out is null");
    CFM_ARG_CHECK(n >= 0, "n");
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    const double two_pi = 4.0 * std::asin(1.0);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; i += 2) {
        const uint64_t c = (uint64_t)(i / 2);
        const uint32_t ctr[4] = {(uint32_t)c, (uint32_t)(c >> 32), stream, 0x4e4f524du};
        uint32_t w[4];
        Philox4x32::block(ctr, key, w);
        const uint64_t b1 = ((uint64_t)w[1] << 32) | w[0];
        const uint64_t b2 = ((uint64_t)w[3] << 32) | w[2];
        const double u1 = (double)((b1 >> 11) + 1) * 0x1.0p-53;
        const double u2 = (double)(b2 >> 11) * 0x1.0p-53;
        const double rad = std::sqrt(-2.0 * std::log(u1));
        out[i] = rad * std::cos(two_pi * u2);
        if (i + 1 < n) out[i + 1] = rad * std::sin(two_pi * u2);
    }
    return CFM_OK;
}

// Gaussian random field: white noise (cfm_normal, stream 0) convolved, with
// periodic wrap, by a separable Gaussian kernel h(d) = exp(-d^2 / (2 l^2)),
// l = corr_len / sqrt(2), truncated at |d| <= ceil(3 l), normalised so that
// sum h^2 = 1 per axis.  The field then has unit variance and covariance
// exp(-r^2 / (2 corr_len^2)); it is scaled by sigma.
int cfm_grf(int dims, int nx, int ny, int nz, unsigned long long seed, double sigma,
            double corr_len, double *g) {
    CFM_ARG_CHECK(dims == 2 || dims == 3, "dims must be 2 or 3");
    CFM_ARG_CHECK(nx >= 1 && ny >= 1 && (dims == 2 || nz >= 1), "sizes");
    CFM_ARG_CHECK(g, "g is null");
    CFM_ARG_CHECK(corr_len > 0 && sigma >= 0, "sigma, corr_len");
    if (dims == 2) nz = 1;
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> a(n), b(n);
    int st = cfm_normal(seed, 0u, (long long)n, a.data());
    if (st) return st;
    const double l = corr_len / std::sqrt(2.0);
    const int R = (int)std::ceil(3.0 * l);
    std::vector<double> h(2 * R + 1);
    double s2 = 0;
    for (int d = -R; d <= R; ++d) {
        h[d + R] = std::exp(-(double)d * d / (2.0 * l * l));
        s2 += h[d + R] * h[d + R];
    }
    for (auto &v : h) v /= std::sqrt(s2);
    auto wrap = [](long long i, int m) { return (int)(((i % m) + m) % m); };
    // x pass a -> b, y pass b -> a, z pass a -> b (3D)
#pragma omp parallel for schedule(static)
    for (long long row = 0; row < (long long)ny * nz; ++row) {
        const double *src = a.data() + row * nx;
        double *dst = b.data() + row * nx;
        for (int x = 0; x < nx; ++x) {
            double acc = 0;
            for (int d = -R; d <= R; ++d) acc += h[d + R] * src[wrap(x + d, nx)];
            dst[x] = acc;
        }
    }
#pragma omp parallel for schedule(static)
    for (long long zx = 0; zx < (long long)nz * nx; ++zx) {
        const long long z = zx / nx, x = zx % nx;
        const size_t base = (size_t)z * nx * ny + x;
        for (int y = 0; y < ny; ++y) {
            double acc = 0;
            for (int d = -R; d <= R; ++d) acc += h[d + R] * b[base + (size_t)wrap(y + d, ny) * nx];
            a[base + (size_t)y * nx] = acc;
        }
    }
    if (dims == 3) {
        const size_t P = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
        for (long long yx = 0; yx < (long long)P; ++yx) {
            for (int z = 0; z < nz; ++z) {
                double acc = 0;
                for (int d = -R; d <= R; ++d) acc += h[d + R] * a[(size_t)wrap(z + d, nz) * P + yx];
                b[(size_t)z * P + yx] = acc;
            }
        }
    }
    const std::vector<double> &res = dims == 3 ? b : a;
    for (size_t i = 0; i < n; ++i) g[i] = sigma * res[i];
    return CFM_OK;
}

// The variable-coefficient diffusion problem -div(k grad u) = f of the
// learned-preconditioner and batched workloads: k = exp(g) with g =
// cfm_grf(seed, sigma = 1, correlation length 16 cells); f ~ N(0, 1) per
// cell from cfm_normal(seed, stream 1).
int cfm_varcoef_problem(int dims, int nx, int ny, int nz, unsigned long long seed, double *k,
                        double *f) {
    CFM_ARG_CHECK(k && f, "null argument");
    int st = cfm_grf(dims, nx, ny, nz, seed, 1.0, 16.0, k);
    if (st) return st;
    const size_t n = (size_t)nx * ny * (dims == 3 ? nz : 1);
    for (size_t i = 0; i < n; ++i) k[i] = std::exp(k[i]);
    return cfm_normal(seed, 1u, (long long)n, f);
}

// Cell-centred finite-volume coefficients of -div(k grad u) on an nx x ny
// (x nz) grid of unit cells with u = 0 on the domain boundary:
//   interior face between cells i, j: w = 2 k_i k_j / (k_i + k_j)
//   boundary face of cell i:          w = 2 k_i (half-cell distance)
// w_e[i], w_n[i], w_t[i] hold the faces to x+1, y+1, z+1 (0 on the last
// column / row / plane); diag[i] is the sum of the cell's 4 (6) face
// weights in the order x-, x+, y-, y+, z-, z+.
int cfm_varcoef_coeffs(int dims, int nx, int ny, int nz, const double *k, double *w_e,
                       double *w_n, double *w_t, double *diag) {
    CFM_ARG_CHECK(dims == 2 || dims == 3, "dims must be 2 or 3");
    CFM_ARG_CHECK(nx >= 1 && ny >= 1 && (dims == 2 || nz >= 1), "sizes");
    CFM_ARG_CHECK(k && w_e && w_n && diag && (dims == 2 || w_t), "null argument");
    if (dims == 2) nz = 1;
    const size_t P = (size_t)nx * ny;
    auto harm = [](double a, double b) { return 2.0 * a * b / (a + b); };
#pragma omp parallel for schedule(static)
    for (long long zz = 0; zz < (long long)nz; ++zz) {
        const int z = (int)zz;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const size_t i = (size_t)z * P + (size_t)y * nx + x;
                const double ki = k[i];
                const double bnd = 2.0 * ki;
                const double wxm = x > 0 ? harm(k[i - 1], ki) : bnd;
                const double wxp = x < nx - 1 ? harm(ki, k[i + 1]) : bnd;
                const double wym = y > 0 ? harm(k[i - nx], ki) : bnd;
                const double wyp = y < ny - 1 ? harm(ki, k[i + nx]) : bnd;
                w_e[i] = x < nx - 1 ? wxp : 0.0;
                w_n[i] = y < ny - 1 ? wyp : 0.0;
                double d = wxm + wxp;
                d = d + wym;
                d = d + wyp;
                if (dims == 3) {
                    const double wzm = z > 0 ? harm(k[i - P], ki) : bnd;
                    const double wzp = z < nz - 1 ? harm(ki, k[i + P]) : bnd;
                    w_t[i] = z < nz - 1 ? wzp : 0.0;
                    d = d + wzm;
                    d = d + wzp;
                }
                diag[i] = d;
            }
    }
    return CFM_OK;
}

long long cfm_poisson3d_nnz(int gx, int gy, int gz) {
    if (gx < 1 || gy < 1 || gz < 1) return -1;
    const long long n = (long long)gx * gy * gz;
    return 7 * n - 2LL * ((long long)gy * gz + (long long)gx * gz + (long long)gx * gy);
}

// Row (i, j, k) = i + gx (j + gy k); columns in increasing order:
// k-1, j-1, i-1, diagonal, i+1, j+1, k+1.
int cfm_poisson3d_csr(int gx, int gy, int gz, int *rowptr, int *col, double *val) {
    CFM_ARG_CHECK(gx >= 1 && gy >= 1 && gz >= 1, "grid sizes");
    CFM_ARG_CHECK(rowptr && col && val, "null argument");
    const long long n = (long long)gx * gy * gz;
    CFM_ARG_CHECK(cfm_poisson3d_nnz(gx, gy, gz) < 2147483647LL && n < 2147483647LL,
                  "matrix too large for int32 indices");
    long long e = 0;
    for (int k = 0; k < gz; ++k)
        for (int j = 0; j < gy; ++j)
            for (int i = 0; i < gx; ++i) {
                const long long r = i + (long long)gx * (j + (long long)gy * k);
                rowptr[r] = (int)e;
                auto put = [&](long long c, double v) {
                    col[e] = (int)c;
                    val[e] = v;
                    ++e;
                };
                if (k > 0) put(r - (long long)gx * gy, -1.0);
                if (j > 0) put(r - gx, -1.0);
                if (i > 0) put(r - 1, -1.0);
                put(r, 6.0);
                if (i < gx - 1) put(r + 1, -1.0);
                if (j < gy - 1) put(r + gx, -1.0);
                if (k < gz - 1) put(r + (long long)gx * gy, -1.0);
            }
    rowptr[n] = (int)e;
    return CFM_OK;
}

// Restates genTridiag (CG/src/common.cu:46-76): symmetric tridiagonal,
// diagonal rand()/RAND_MAX + 10, off-diagonal rand()/RAND_MAX, the sub-
// diagonal copied from the previous row's super-diagonal, values drawn from
// libc rand() in its current state (the reference never seeds it).
int cfm_tridiag_csr(int n, int *rowptr, int *col, double *val) {
    CFM_ARG_CHECK(n >= 2, "n must be >= 2");
    CFM_ARG_CHECK(rowptr && col && val, "null argument");
    const int nnz = (n - 2) * 3 + 4;
    rowptr[0] = 0;
    col[0] = 0;
    col[1] = 1;
    val[0] = (double)rand() / RAND_MAX + 10.0;
    val[1] = (double)rand() / RAND_MAX;
    for (int i = 1; i < n; ++i) {
        rowptr[i] = (i > 1) ? rowptr[i - 1] + 3 : 2;
        const int start = (i - 1) * 3 + 2;
        col[start] = i - 1;
        col[start + 1] = i;
        if (i < n - 1) col[start + 2] = i + 1;
        val[start] = val[start - 1];
        val[start + 1] = (double)rand() / RAND_MAX + 10.0;
        if (i < n - 1) val[start + 2] = (double)rand() / RAND_MAX;
    }
    rowptr[n] = nnz;
    return CFM_OK;
}

}  // extern "C"
