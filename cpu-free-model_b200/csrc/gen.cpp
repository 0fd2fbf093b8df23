// Host-side problem generators exported through the C ABI.
#include <cstdint>
#include <cstdlib>
#include <cstring>

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
