// Persistent Krylov solvers on one GPU, templated on the operator.
//
// Operators (one row per thread, tiles of CG_TILE consecutive rows):
//   CsrOp        CSR SpMV, row order, one fma per nonzero (CG/src/common.cu:150-168)
//   StencilOp<D> matrix-free cell-centred -div(k grad u), 5-point (D = 2) or
//                7-point (D = 3): t = d_i u_i, then one fma(-w, u_nb, t) per
//                neighbour in the order x-1, x+1, y-1, y+1, z-1, z+1
// Each operator also applies in FP32 (apply32) from FP32 copies of its
// coefficients, for the inner solve of the mixed-precision method.
//
// Solvers, each one cooperative launch for the whole solve:
//   cg_std_kernel    standard CG, 3 grid barriers per iteration
//                    (CG/src/common.cu:399-538, CG/src/single-stream/standard.cu:158-299)
//   cg_pipe_kernel   pipelined CG (CG/src/single-stream/pipelined.cu:176-330): the
//                    SpMV q = A w and every vector recurrence of an iteration fused
//                    into one pass, double-buffered w and dot partials, 1 grid
//                    barrier per iteration
//   cg_mixed_kernel  FP32 CG with FP64 reliable updates: the true residual, the
//                    correction x += |b| d and the dot reductions (FP64 sums of
//                    exact FP32 products) stay FP64
// Every dot is a fixed tree (1024-row tiles, xor butterflies, then the tile
// partials in lane order), so results do not depend on the launch shape and
// the CPU oracle reproduces them bit for bit.  Scalar arithmetic is written
// with explicit-rounding intrinsics where the compiler could otherwise fuse a
// multiply into an add.
#pragma once

#include "barrier.cuh"

namespace cfm {

constexpr int CG_TILE = 1024;  // rows per tile == threads per block
constexpr unsigned CG_FULL = 0xffffffffu;

// Partial-sum slots (each ntiles doubles) in KArgs::part.
enum : int { SL_G0 = 0, SL_D0 = 1, SL_TT = 2, SL_B = 3, SL_G1 = 4, SL_D1 = 5, NSLOTS = 6 };

struct CgResult {
    long long iters;
    int status;
    int restarts;  // restarts (standard, pipelined) or FP64 reliable updates (mixed)
    double gamma;
    double bnorm;
};

__device__ __forceinline__ double warp_xor_sum(double v) {
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) v = __dadd_rn(v, __shfl_xor_sync(CG_FULL, v, off));
    return v;
}

// Tree sum over the 1024 threads of the block; every thread gets the result.
__device__ __forceinline__ double block_sum(double v, double *sm /* 33 doubles */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_xor_sum(v);
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = warp_xor_sum(sm[lane]);
        if (lane == 0) sm[32] = w;
    }
    __syncthreads();
    const double out = sm[32];
    __syncthreads();
    return out;
}

// Sum of tile partials in the fixed order: thread t adds part[t], part[t+1024], ...
__device__ __forceinline__ double sum_partials(const double *part, int ntiles, double *sm) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < ntiles; i += CG_TILE) acc = __dadd_rn(acc, part[i]);
    return block_sum(acc, sm);
}

// Per-tile sums of a tile loop without a block barrier per tile.  Each
// warp reduces its 32 rows at once (the xor butterfly of block_sum) and
// parks the warp sum in shared memory; every TS_TILES tiles, and at the end,
// one barrier, then warp w reduces parked entry w (the 32 warp sums of one
// tile, in warp order: again block_sum's tree) into dst[k][tile].  The
// partials are bit for bit block_sum's, while the warps of a block run ahead
// of each other from tile to tile.  The block's tiles are t0, t0 + stride,
// ...; every thread of the block calls add() for every tile, and flush()
// after the loop.
constexpr int TS_TILES = 16;
constexpr int TS_SMEM = TS_TILES * 2 * 32;  // doubles (also >= 33 for block_sum)

template <int K>
struct TileSums {
    double *sm;
    double *dst[K];
    int stride, t0 = 0, g = 0;
    __device__ __forceinline__ TileSums(double *s, int step, double *d0, double *d1 = nullptr)
        : sm(s), stride(step) {
        dst[0] = d0;
        if (K > 1) dst[K - 1] = d1;
    }
    __device__ __forceinline__ void add(int tile, double v0, double v1 = 0.0) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (g == 0) t0 = tile;
        v0 = warp_xor_sum(v0);
        if (lane == 0) sm[(g * K) * 32 + warp] = v0;
        if (K > 1) {
            v1 = warp_xor_sum(v1);
            if (lane == 0) sm[(g * K + K - 1) * 32 + warp] = v1;
        }
        if (++g == TS_TILES) flush();
    }
    __device__ __forceinline__ void flush() {
        if (g == 0) return;
        __syncthreads();
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (warp < g * K) {
            const double v = warp_xor_sum(sm[warp * 32 + lane]);
            double *d = dst[0];
            if (K > 1 && (warp & 1)) d = dst[K - 1];  // a select: no indexed local array
            if (lane == 0) d[t0 + (warp / K) * stride] = v;
        }
        __syncthreads();
        g = 0;
    }
};

// Exact product of two FP32 values, as FP64.
__device__ __forceinline__ double xprod(float a, float b) { return __dmul_rn((double)a, (double)b); }

// U of the block's tiles per step (t0 + u gridDim.x, u < U), the FP32
// passes' form of the tile pairs.  U = 2 measured best on 128^3 Poisson
// (4: 22.3 ms mixed against 19.6 ms).
constexpr int INNER_U = 2;
template <int U>
struct TileGroup {
    int tile[U], row[U];
    bool has[U], ok[U];
    __device__ __forceinline__ TileGroup(int ntiles, int n, int t0) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            tile[u] = t0 + u * (int)gridDim.x;
            has[u] = tile[u] < ntiles;
            row[u] = tile[u] * CG_TILE + (int)threadIdx.x;
            ok[u] = has[u] && row[u] < n;
        }
    }
};
template <int U>
struct Vals32 {
    float v[U];
};

// ------------------------------------------------------------- operators
// CSR entries per row whose loads a thread issues together (CsrOp::apply2_t,
// the FP64 passes): 4 and 8 both took standard CG on 128^3 Poisson from
// 26.4 to 25.5 ms (bit-identical); the same form in the FP32 passes was no
// faster (20.1-20.9 against 19.9-20.2 ms), so those keep one entry per step.
constexpr int CSR_Q = 4;
struct CsrOp {
    const int *rowptr, *col;
    const double *val;
    const float *val32;
    __device__ __forceinline__ double apply(const double *x, int i) const {
        double acc = 0.0;
        const int j1 = rowptr[i + 1];
        for (int j = rowptr[i]; j < j1; ++j) acc = __fma_rn(val[j], x[col[j]], acc);
        return acc;
    }
    __device__ __forceinline__ float apply32(const float *x, int i) const {
        float acc = 0.f;
        const int j1 = rowptr[i + 1];
        for (int j = rowptr[i]; j < j1; ++j) acc = __fmaf_rn(val32[j], x[col[j]], acc);
        return acc;
    }
    // apply for rows i (if v1) and i2 (if v2), their entries interleaved so
    // that both rows' loads are in flight together; 0 for an absent row.
    template <class T>
    __device__ __forceinline__ void apply2_t(const T *v, const T *x, int i, bool v1, int i2,
                                             bool v2, T &y1, T &y2) const {
        int j1 = 0, e1 = 0, j2 = 0, e2 = 0;
        if (v1) {
            j1 = rowptr[i];
            e1 = rowptr[i + 1];
        }
        if (v2) {
            j2 = rowptr[i2];
            e2 = rowptr[i2 + 1];
        }
        T a1 = T(0), a2 = T(0);
        // CSR_Q entries of each row per step: all their col / val loads,
        // then all their x gathers, then the FMAs in entry order (the sum is
        // the one-entry-at-a-time one, bit for bit), so up to 4 CSR_Q
        // independent loads are in flight per thread instead of two chains
        while (j1 < e1 || j2 < e2) {
            int c1[CSR_Q], c2[CSR_Q];
            T w1[CSR_Q], w2[CSR_Q], g1[CSR_Q], g2[CSR_Q];
#pragma unroll
            for (int q = 0; q < CSR_Q; ++q) {
                c1[q] = j1 + q < e1 ? col[j1 + q] : -1;
                c2[q] = j2 + q < e2 ? col[j2 + q] : -1;
                w1[q] = j1 + q < e1 ? v[j1 + q] : T(0);
                w2[q] = j2 + q < e2 ? v[j2 + q] : T(0);
            }
#pragma unroll
            for (int q = 0; q < CSR_Q; ++q) {
                g1[q] = c1[q] >= 0 ? x[c1[q]] : T(0);
                g2[q] = c2[q] >= 0 ? x[c2[q]] : T(0);
            }
#pragma unroll
            for (int q = 0; q < CSR_Q; ++q) {
                if (c1[q] >= 0) a1 = fma_rn(w1[q], g1[q], a1);
                if (c2[q] >= 0) a2 = fma_rn(w2[q], g2[q], a2);
            }
            j1 += CSR_Q;
            j2 += CSR_Q;
        }
        y1 = a1;
        y2 = a2;
    }
    __device__ __forceinline__ static double fma_rn(double u, double w, double c) {
        return __fma_rn(u, w, c);
    }
    __device__ __forceinline__ static float fma_rn(float u, float w, float c) {
        return __fmaf_rn(u, w, c);
    }
    __device__ __forceinline__ void apply2(const double *x, int i, bool v1, int i2, bool v2,
                                           double &y1, double &y2) const {
        apply2_t(val, x, i, v1, i2, v2, y1, y2);
    }
    // FP32 apply for the rows of a tile group (0 for an absent row), their
    // entries interleaved.
    template <int U>
    __device__ __forceinline__ Vals32<U> applyN32(const float *x, const TileGroup<U> &g) const {
        int j[U], e[U];
        Vals32<U> y;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            j[u] = g.ok[u] ? rowptr[g.row[u]] : 0;
            e[u] = g.ok[u] ? rowptr[g.row[u] + 1] : 0;
            y.v[u] = 0.f;
        }
        bool more = true;
        while (more) {
            more = false;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (j[u] < e[u]) {
                    y.v[u] = __fmaf_rn(val32[j[u]], x[col[j[u]]], y.v[u]);
                    ++j[u];
                    more = true;
                }
        }
        return y;
    }
    // A x0 with x0 = 0, summed like apply (always +0)
    __device__ __forceinline__ double apply_zero(int i) const {
        double acc = 0.0;
        const int j1 = rowptr[i + 1];
        for (int j = rowptr[i]; j < j1; ++j) acc = __fma_rn(val[j], 0.0, acc);
        return acc;
    }
};

template <int D>
struct StencilOp {
    int nx, ny, nz;
    const double *we, *wn, *wt, *dg;
    const float *we32, *wn32, *wt32, *dg32;
    __device__ __forceinline__ double apply(const double *x, int i) const {
        const int ix = i % nx, q = i / nx, iy = q % ny;
        double t = __dmul_rn(dg[i], x[i]);
        if (ix > 0) t = __fma_rn(-we[i - 1], x[i - 1], t);
        if (ix < nx - 1) t = __fma_rn(-we[i], x[i + 1], t);
        if (iy > 0) t = __fma_rn(-wn[i - nx], x[i - nx], t);
        if (iy < ny - 1) t = __fma_rn(-wn[i], x[i + nx], t);
        if (D == 3) {
            const int iz = q / ny, P = nx * ny;
            if (iz > 0) t = __fma_rn(-wt[i - P], x[i - P], t);
            if (iz < nz - 1) t = __fma_rn(-wt[i], x[i + P], t);
        }
        return t;
    }
    __device__ __forceinline__ float apply32(const float *x, int i) const {
        const int ix = i % nx, q = i / nx, iy = q % ny;
        float t = __fmul_rn(dg32[i], x[i]);
        if (ix > 0) t = __fmaf_rn(-we32[i - 1], x[i - 1], t);
        if (ix < nx - 1) t = __fmaf_rn(-we32[i], x[i + 1], t);
        if (iy > 0) t = __fmaf_rn(-wn32[i - nx], x[i - nx], t);
        if (iy < ny - 1) t = __fmaf_rn(-wn32[i], x[i + nx], t);
        if (D == 3) {
            const int iz = q / ny, P = nx * ny;
            if (iz > 0) t = __fmaf_rn(-wt32[i - P], x[i - P], t);
            if (iz < nz - 1) t = __fmaf_rn(-wt32[i], x[i + P], t);
        }
        return t;
    }
    __device__ __forceinline__ double apply_zero(int) const { return 0.0; }
    __device__ __forceinline__ void apply2(const double *x, int i, bool v1, int i2, bool v2,
                                           double &y1, double &y2) const {
        y1 = v1 ? apply(x, i) : 0.0;
        y2 = v2 ? apply(x, i2) : 0.0;
    }
    template <int U>
    __device__ __forceinline__ Vals32<U> applyN32(const float *x, const TileGroup<U> &g) const {
        Vals32<U> y;
#pragma unroll
        for (int u = 0; u < U; ++u) y.v[u] = g.ok[u] ? apply32(x, g.row[u]) : 0.f;
        return y;
    }
};

template <class Op>
struct KArgs {
    Op op;
    int n;
    int ntiles;
    const double *b;  // nullptr: ones
    double *x, *r, *p, *s, *t;
    double *z, *w0, *w1;           // pipelined
    float *r32, *p32, *s32, *d32;  // mixed inner
    double *part;                  // NSLOTS * ntiles
    CgResult *res;
    BarrierState *bar;
    int maxiter;
    double tol;
    int inner_maxiter;
    double inner_tol;
    // standard CG only: copy x after every snap_every-th iteration into
    // snap[(k / snap_every - 1) * n ...] while fewer than snap_max are taken
    double *snap;
    int snap_every, snap_max;
};

#define CFM_TILES(a) for (int tile = blockIdx.x; tile < (a).ntiles; tile += gridDim.x)
#define CFM_ROW(a) const int i = tile * CG_TILE + threadIdx.x
// Two of the block's tiles per step (tile, tile2 = tile + gridDim.x): the
// loads of both rows go out before either row's arithmetic, halving the
// chains of dependent memory round trips a warp waits on.
#define CFM_TILE_GROUPS(a, U) for (int tile = blockIdx.x; tile < (a).ntiles; tile += (U) * (int)gridDim.x)
#define CFM_TILE_PAIRS(a) for (int tile = blockIdx.x; tile < (a).ntiles; tile += 2 * (int)gridDim.x)
#define CFM_ROW_PAIR(a)                                                      \
    const int tile2 = tile + (int)gridDim.x;                                 \
    const bool has2 = tile2 < (a).ntiles;                                    \
    const int i = tile * CG_TILE + threadIdx.x, i2 = tile2 * CG_TILE + threadIdx.x; \
    const bool v1 = i < (a).n, v2 = has2 && i2 < (a).n

template <class Op>
__device__ __forceinline__ double *slot(const KArgs<Op> &a, int s) {
    return a.part + (size_t)s * a.ntiles;
}

// -------------------------------------------------------- standard phases
template <class Op>
__device__ void phase_init(const KArgs<Op> &a, double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, SL_G0), slot(a, SL_B));
    CFM_TILES(a) {
        CFM_ROW(a);
        double g = 0.0, bb = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double ri = __fma_rn(-1.0, a.op.apply_zero(i), bi);  // r0 = b - A x0, x0 = 0
            a.x[i] = 0.0;
            a.r[i] = ri;
            a.p[i] = ri;
            g = __dmul_rn(ri, ri);
            bb = __dmul_rn(bi, bi);
        }
        ts.add(tile, g, bb);
    }
    ts.flush();
}

template <class Op>
__device__ void phase_spmv_dot(const KArgs<Op> &a, double *sm) {
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_D0));
    CFM_TILE_PAIRS(a) {
        CFM_ROW_PAIR(a);
        double p1 = 0.0, p2 = 0.0, s1, s2;
        if (v1) p1 = a.p[i];
        if (v2) p2 = a.p[i2];
        a.op.apply2(a.p, i, v1, i2, v2, s1, s2);
        if (v1) a.s[i] = s1;
        if (v2) a.s[i2] = s2;
        ts.add(tile, v1 ? __dmul_rn(p1, s1) : 0.0);
        if (has2) ts.add(tile2, v2 ? __dmul_rn(p2, s2) : 0.0);
    }
    ts.flush();
}

template <class Op>
__device__ void phase_update(const KArgs<Op> &a, double alpha, double *sm) {
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_G0));
    CFM_TILE_PAIRS(a) {
        CFM_ROW_PAIR(a);
        double x1 = 0.0, p1 = 0.0, r1 = 0.0, s1 = 0.0, x2 = 0.0, p2 = 0.0, r2 = 0.0, s2 = 0.0;
        if (v1) {
            x1 = a.x[i];
            p1 = a.p[i];
            r1 = a.r[i];
            s1 = a.s[i];
        }
        if (v2) {
            x2 = a.x[i2];
            p2 = a.p[i2];
            r2 = a.r[i2];
            s2 = a.s[i2];
        }
        double g1 = 0.0, g2 = 0.0;
        if (v1) {
            a.x[i] = __fma_rn(alpha, p1, x1);
            const double ri = __fma_rn(-alpha, s1, r1);
            a.r[i] = ri;
            g1 = __dmul_rn(ri, ri);
        }
        if (v2) {
            a.x[i2] = __fma_rn(alpha, p2, x2);
            const double ri = __fma_rn(-alpha, s2, r2);
            a.r[i2] = ri;
            g2 = __dmul_rn(ri, ri);
        }
        ts.add(tile, g1);
        if (has2) ts.add(tile2, g2);
    }
    ts.flush();
}

// t = b - A x (FP64) and its squared norm into SL_TT
template <class Op>
__device__ void phase_true_residual(const KArgs<Op> &a, double *sm) {
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_TT));
    CFM_TILES(a) {
        CFM_ROW(a);
        double q = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double ti = __dsub_rn(bi, a.op.apply(a.x, i));
            a.t[i] = ti;
            q = __dmul_rn(ti, ti);
        }
        ts.add(tile, q);
    }
    ts.flush();
}

template <class Op>
__device__ void phase_snap(const KArgs<Op> &a, int slot_i) {
    double *dst = a.snap + (size_t)slot_i * a.n;
    CFM_TILES(a) {
        CFM_ROW(a);
        if (i < a.n) dst[i] = a.x[i];
    }
}

template <class Op>
__device__ void phase_restart(const KArgs<Op> &a) {
    CFM_TILES(a) {
        CFM_ROW(a);
        if (i < a.n) {
            a.r[i] = a.t[i];
            a.p[i] = a.t[i];
        }
    }
}

template <class Op>
__device__ void phase_p(const KArgs<Op> &a, double beta) {
    CFM_TILE_PAIRS(a) {
        CFM_ROW_PAIR(a);
        double p1 = 0.0, r1 = 0.0, p2 = 0.0, r2 = 0.0;
        if (v1) {
            p1 = a.p[i];
            r1 = a.r[i];
        }
        if (v2) {
            p2 = a.p[i2];
            r2 = a.r[i2];
        }
        if (v1) a.p[i] = __fma_rn(beta, p1, r1);
        if (v2) a.p[i2] = __fma_rn(beta, p2, r2);
    }
}

__device__ __forceinline__ void write_result(CgResult *res, long long k, int status, int restarts,
                                             double gamma, double bnorm) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        res->iters = k;
        res->status = status;
        res->restarts = restarts;
        res->gamma = gamma;
        res->bnorm = bnorm;
    }
}

// Standard CG; tol > 0 stops when the recursive residual reaches tol ||b||
// and the FP64 true residual confirms it (a restart from the true residual
// otherwise); tol <= 0 runs exactly maxiter iterations (reference -niter).
template <class Op>
__global__ void __launch_bounds__(CG_TILE, 1) cg_std_kernel(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    int site = 0;
    phase_init(a, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    double gamma0 = sum_partials(slot(a, SL_G0), a.ntiles, sm);
    const double bnorm = sqrt(sum_partials(slot(a, SL_B), a.ntiles, sm));
    const bool use_tol = a.tol > 0.0;
    const double target = a.tol * bnorm;
    int status = use_tol ? CFM_NOT_CONVERGED : CFM_OK;
    int restarts = 0;
    long long k = 0;
    if (use_tol && sqrt(gamma0) <= target) status = CFM_OK;
    while (k < a.maxiter && !(use_tol && status == CFM_OK)) {
        phase_spmv_dot(a, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        const double delta = sum_partials(slot(a, SL_D0), a.ntiles, sm);
        const double alpha = gamma0 / delta;
        if (use_tol && !(delta > 0.0 && isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        phase_update(a, alpha, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        const double gamma1 = sum_partials(slot(a, SL_G0), a.ntiles, sm);
        ++k;
        if (a.snap && k % a.snap_every == 0 && k / a.snap_every <= a.snap_max)
            phase_snap(a, (int)(k / a.snap_every) - 1);  // x is stable until the next update
        if (use_tol && sqrt(gamma1) <= target) {
            phase_true_residual(a, sm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            const double tt = sum_partials(slot(a, SL_TT), a.ntiles, sm);
            if (sqrt(tt) <= target) {
                status = CFM_OK;
                gamma0 = gamma1;
                break;
            }
            phase_restart(a);
            ++restarts;
            gamma0 = tt;
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            continue;
        }
        const double beta = gamma1 / gamma0;
        if (use_tol && !isfinite(beta)) {
            status = CFM_BREAKDOWN;
            break;
        }
        phase_p(a, beta);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        gamma0 = gamma1;
    }
    write_result(a.res, k, status, restarts, gamma0, bnorm);
}

// ------------------------------------------------------- pipelined phases
// r0 = b - A x0 with x0 = 0 (into t), and ||b||^2.
template <class Op>
__device__ void phase_pipe_init(const KArgs<Op> &a, double *sm) {
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_B));
    CFM_TILES(a) {
        CFM_ROW(a);
        double bb = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            a.x[i] = 0.0;
            a.t[i] = __fma_rn(-1.0, a.op.apply_zero(i), bi);
            bb = __dmul_rn(bi, bi);
        }
        ts.add(tile, bb);
    }
    ts.flush();
}

// r = v, w = A v, z = s = p = 0; partials <r, r> -> G[par], <w, r> -> D[par].
// v is the initial residual, or the true residual t at a restart.
template <class Op>
__device__ void phase_pipe_start(const KArgs<Op> &a, const double *v, double *w, int par,
                                 double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, par ? SL_G1 : SL_G0), slot(a, par ? SL_D1 : SL_D0));
    CFM_TILES(a) {
        CFM_ROW(a);
        double g = 0.0, d = 0.0;
        if (i < a.n) {
            const double ri = v[i];
            const double wi = a.op.apply(v, i);
            a.r[i] = ri;
            w[i] = wi;
            a.z[i] = 0.0;
            a.s[i] = 0.0;
            a.p[i] = 0.0;
            g = __dmul_rn(ri, ri);
            d = __dmul_rn(wi, ri);
        }
        ts.add(tile, g, d);
    }
    ts.flush();
}

// One pipelined iteration, row-local once q = A w is known:
//   z = q + beta z; s = w + beta s; p = r + beta p
//   x += alpha p; r -= alpha s; w' = w - alpha z
// and the next iteration's partials <r', r'>, <w', r'> into slot parity `nxt`.
template <class Op>
__device__ void phase_pipe_step(const KArgs<Op> &a, const double *w, double *wn, double alpha,
                                double beta, int nxt, double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, nxt ? SL_G1 : SL_G0), slot(a, nxt ? SL_D1 : SL_D0));
    CFM_TILES(a) {
        CFM_ROW(a);
        double g = 0.0, d = 0.0;
        if (i < a.n) {
            const double q = a.op.apply(w, i);
            const double wi = w[i];
            const double zi = __fma_rn(beta, a.z[i], q);
            const double si = __fma_rn(beta, a.s[i], wi);
            const double pi = __fma_rn(beta, a.p[i], a.r[i]);
            a.x[i] = __fma_rn(alpha, pi, a.x[i]);
            const double ri = __fma_rn(-alpha, si, a.r[i]);
            const double wni = __fma_rn(-alpha, zi, wi);
            a.z[i] = zi;
            a.s[i] = si;
            a.p[i] = pi;
            a.r[i] = ri;
            wn[i] = wni;
            g = __dmul_rn(ri, ri);
            d = __dmul_rn(wni, ri);
        }
        ts.add(tile, g, d);
    }
    ts.flush();
}

// Residual replacement, first half: t = b - A x, s = A p.
template <class Op>
__device__ void phase_replace_a(const KArgs<Op> &a) {
    CFM_TILES(a) {
        CFM_ROW(a);
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            a.t[i] = __dsub_rn(bi, a.op.apply(a.x, i));
            a.s[i] = a.op.apply(a.p, i);
        }
    }
}

// Residual replacement, second half: r = t, w = A t, z = A s and the
// partials <r, r> -> G[par], <w, r> -> D[par].
template <class Op>
__device__ void phase_replace_b(const KArgs<Op> &a, double *w, int par, double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, par ? SL_G1 : SL_G0), slot(a, par ? SL_D1 : SL_D0));
    CFM_TILES(a) {
        CFM_ROW(a);
        double g = 0.0, d = 0.0;
        if (i < a.n) {
            const double ri = a.t[i];
            const double wi = a.op.apply(a.t, i);
            a.r[i] = ri;
            w[i] = wi;
            a.z[i] = a.op.apply(a.s, i);
            g = __dmul_rn(ri, ri);
            d = __dmul_rn(wi, ri);
        }
        ts.add(tile, g, d);
    }
    ts.flush();
}

// Iterations between residual replacements in pipelined CG.
constexpr long long PIPE_REPLACE = 50;

// Pipelined CG.  Scalars follow the reference's recurrence
// (CG/src/single-stream/pipelined.cu:262-272): with rr = <r, r>, wr = <w, r>,
//   beta = rr / rr_prev, alpha = rr / (wr - (beta / alpha_prev) rr)
// from the third step of a run on, and beta = 0, alpha = rr / wr on the
// first two (the reference tests `k > 1`).  Convergence as cg_std_kernel.
// The pipelined recurrences let the recursive residual drift from b - A x on
// ill-conditioned systems, so with tol > 0 every PIPE_REPLACE iterations the
// vectors r, w, s, z are recomputed from x and p (residual replacement: two
// extra barriers, four operator applications); the scalar recurrence goes on.
template <class Op>
__global__ void __launch_bounds__(CG_TILE, 1) cg_pipe_kernel(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    int site = 0;
    phase_pipe_init(a, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    const double bnorm = sqrt(sum_partials(slot(a, SL_B), a.ntiles, sm));
    phase_pipe_start(a, a.t, a.w0, 0, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    const bool use_tol = a.tol > 0.0;
    const double target = a.tol * bnorm;
    int status = use_tol ? CFM_NOT_CONVERGED : CFM_OK;
    int restarts = 0, cur = 0;
    long long k = 0, kk = 0, replaced = -1;
    double rr = 0.0, rr_prev = 0.0, alpha = 0.0;
    while (true) {
        double *w = cur ? a.w1 : a.w0;
        rr = sum_partials(slot(a, cur ? SL_G1 : SL_G0), a.ntiles, sm);
        const double wr = sum_partials(slot(a, cur ? SL_D1 : SL_D0), a.ntiles, sm);
        if (use_tol && sqrt(rr) <= target) {
            phase_true_residual(a, sm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            const double tt = sum_partials(slot(a, SL_TT), a.ntiles, sm);
            if (sqrt(tt) <= target) {
                status = CFM_OK;
                break;
            }
            phase_pipe_start(a, a.t, w, cur, sm);  // restart from the true residual
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            ++restarts;
            kk = 0;
            replaced = k;  // a restart needs no replacement at this count
            continue;
        }
        if (k >= a.maxiter) break;
        if (use_tol && k > 0 && k % PIPE_REPLACE == 0 && replaced != k) {
            phase_replace_a(a);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            phase_replace_b(a, w, cur, sm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            replaced = k;
            ++restarts;
            continue;
        }
        double beta;
        if (kk > 1) {
            beta = rr / rr_prev;
            alpha = rr / __dsub_rn(wr, __dmul_rn(beta / alpha, rr));
        } else {
            beta = 0.0;
            alpha = rr / wr;
        }
        if (use_tol && !(isfinite(alpha) && alpha > 0.0 && isfinite(beta))) {
            status = CFM_BREAKDOWN;
            break;
        }
        phase_pipe_step(a, w, cur ? a.w0 : a.w1, alpha, beta, cur ^ 1, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        rr_prev = rr;
        cur ^= 1;
        ++k;
        ++kk;
    }
    write_result(a.res, k, status, restarts, rr, bnorm);
}

// ----------------------------------------------------------- mixed phases
// x = 0, t = b - A x0, partials ||t||^2 (SL_TT) and ||b||^2 (SL_B).
template <class Op>
__device__ void phase_mixed_init(const KArgs<Op> &a, double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, SL_TT), slot(a, SL_B));
    CFM_TILES(a) {
        CFM_ROW(a);
        double q = 0.0, bb = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double ti = __fma_rn(-1.0, a.op.apply_zero(i), bi);
            a.x[i] = 0.0;
            a.t[i] = ti;
            q = __dmul_rn(ti, ti);
            bb = __dmul_rn(bi, bi);
        }
        ts.add(tile, q, bb);
    }
    ts.flush();
}

// Start of the FP32 iteration: r32 = fl32(t * scale), p32 = r32, d32 = 0;
// <r32, r32> -> G0.
template <class Op>
__device__ void phase_inner_start(const KArgs<Op> &a, double scale, double *sm) {
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_G0));
    CFM_TILES(a) {
        CFM_ROW(a);
        double g = 0.0;
        if (i < a.n) {
            const float ri = __double2float_rn(__dmul_rn(a.t[i], scale));
            a.r32[i] = ri;
            a.p32[i] = ri;
            a.d32[i] = 0.f;
            g = xprod(ri, ri);
        }
        ts.add(tile, g);
    }
    ts.flush();
}

template <class Op>
__device__ void phase_inner_spmv(const KArgs<Op> &a, double *sm) {
    constexpr int U = INNER_U;
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_D0));
    CFM_TILE_GROUPS(a, U) {
        const TileGroup<U> g(a.ntiles, a.n, tile);
        float p[U];
#pragma unroll
        for (int u = 0; u < U; ++u) p[u] = g.ok[u] ? a.p32[g.row[u]] : 0.f;
        const Vals32<U> y = a.op.template applyN32<U>(a.p32, g);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (g.ok[u]) a.s32[g.row[u]] = y.v[u];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (g.has[u]) ts.add(g.tile[u], g.ok[u] ? xprod(p[u], y.v[u]) : 0.0);
    }
    ts.flush();
}

template <class Op>
__device__ void phase_inner_update(const KArgs<Op> &a, float af, double *sm) {
    constexpr int U = INNER_U;
    TileSums<1> ts(sm, gridDim.x, slot(a, SL_G0));
    CFM_TILE_GROUPS(a, U) {
        const TileGroup<U> g(a.ntiles, a.n, tile);
        float d[U], p[U], r[U], sv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            d[u] = p[u] = r[u] = sv[u] = 0.f;
            if (g.ok[u]) {
                d[u] = a.d32[g.row[u]];
                p[u] = a.p32[g.row[u]];
                r[u] = a.r32[g.row[u]];
                sv[u] = a.s32[g.row[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            double q = 0.0;
            if (g.ok[u]) {
                a.d32[g.row[u]] = __fmaf_rn(af, p[u], d[u]);
                const float ri = __fmaf_rn(-af, sv[u], r[u]);
                a.r32[g.row[u]] = ri;
                q = xprod(ri, ri);
            }
            if (g.has[u]) ts.add(g.tile[u], q);
        }
    }
    ts.flush();
}

template <class Op>
__device__ void phase_inner_p(const KArgs<Op> &a, float bf) {
    constexpr int U = INNER_U;
    CFM_TILE_GROUPS(a, U) {
        const TileGroup<U> g(a.ntiles, a.n, tile);
        float p[U], r[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            p[u] = r[u] = 0.f;
            if (g.ok[u]) {
                p[u] = a.p32[g.row[u]];
                r[u] = a.r32[g.row[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (g.ok[u]) a.p32[g.row[u]] = __fmaf_rn(bf, p[u], r[u]);
    }
}

// Reliable update, first half: x += |b| d32 in FP64, d32 = 0.
template <class Op>
__device__ void phase_correct(const KArgs<Op> &a, double norm) {
    CFM_TILES(a) {
        CFM_ROW(a);
        if (i < a.n) {
            a.x[i] = __fma_rn(norm, (double)a.d32[i], a.x[i]);
            a.d32[i] = 0.f;
        }
    }
}

// Reliable update, second half: t = b - A x (FP64) with |t|^2 -> TT, and
// r32 = fl32(t / |b|) with <r32, r32> -> G0.
template <class Op>
__device__ void phase_replace32(const KArgs<Op> &a, double scale, double *sm) {
    TileSums<2> ts(sm, gridDim.x, slot(a, SL_TT), slot(a, SL_G0));
    CFM_TILES(a) {
        CFM_ROW(a);
        double q = 0.0, g = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double ti = __dsub_rn(bi, a.op.apply(a.x, i));
            const float ri = __double2float_rn(__dmul_rn(ti, scale));
            a.t[i] = ti;
            a.r32[i] = ri;
            q = __dmul_rn(ti, ti);
            g = xprod(ri, ri);
        }
        ts.add(tile, q, g);
    }
    ts.flush();
}

// Mixed-precision CG with reliable updates.  The iteration runs in FP32
// (FP32 SpMV and axpys; the dots are FP64 sums of the exact FP32 products;
// alpha, beta in FP64, applied rounded to FP32) on r32 = fl32(r / |b|) and
// gathers its steps in an FP32 correction d32.  When <r32, r32> falls to
// tol^2, below inner_tol^2 times its largest value since the last update,
// or after inner_maxiter steps (0: no cap), a reliable update adds |b| d32
// to x in FP64 and replaces r32 by fl32((b - A x) / |b|) from the FP64 true
// residual; the search direction p32 is kept, so the recurrence goes on
// (beta from the replaced residual) instead of restarting (Sleijpen and van
// der Vorst's reliable updated residuals).  Stops when the FP64 true
// residual |b - A x| <= tol |b|; maxiter caps the FP32 steps.
template <class Op>
__global__ void __launch_bounds__(CG_TILE, 1) cg_mixed_kernel(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    int site = 0;
    phase_mixed_init(a, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    const double bnorm = sqrt(sum_partials(slot(a, SL_B), a.ntiles, sm));
    const double target = a.tol * bnorm;
    double tt = sum_partials(slot(a, SL_TT), a.ntiles, sm);
    int status = CFM_NOT_CONVERGED, updates = 0;
    long long k = 0;
    if (sqrt(tt) <= target || bnorm == 0.0) {
        write_result(a.res, 0, sqrt(tt) <= target ? CFM_OK : CFM_NOT_CONVERGED, 0, tt, bnorm);
        return;
    }
    const double scale = 1.0 / bnorm, tol2 = a.tol * a.tol;
    const double delta2 = a.inner_tol * a.inner_tol;
    phase_inner_start(a, scale, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    double g0 = sum_partials(slot(a, SL_G0), a.ntiles, sm), gmax = g0;
    int since = 0;
    while (k < a.maxiter) {
        phase_inner_spmv(a, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        const double delta = sum_partials(slot(a, SL_D0), a.ntiles, sm);
        const double alpha = g0 / delta;
        if (!(delta > 0.0 && isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        phase_inner_update(a, __double2float_rn(alpha), sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        double g1 = sum_partials(slot(a, SL_G0), a.ntiles, sm);
        ++k;
        ++since;
        if (g1 <= tol2 || g1 < delta2 * gmax || k >= a.maxiter ||
            (a.inner_maxiter > 0 && since >= a.inner_maxiter)) {
            phase_correct(a, bnorm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            phase_replace32(a, scale, sm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            tt = sum_partials(slot(a, SL_TT), a.ntiles, sm);
            g1 = sum_partials(slot(a, SL_G0), a.ntiles, sm);
            ++updates;
            since = 0;
            gmax = g1;
            if (sqrt(tt) <= target) {
                status = CFM_OK;
                break;
            }
            if (k >= a.maxiter) break;
        } else if (g1 > gmax) {
            gmax = g1;
        }
        const double beta = g1 / g0;
        phase_inner_p(a, __double2float_rn(beta));
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        g0 = g1;
    }
    if (since > 0) phase_correct(a, bnorm);  // a breakdown left steps in d32
    write_result(a.res, k, status, updates, tt, bnorm);
}

// ------------------------------------------------ host-controlled pieces
// One kernel per operation (the comparator of CG/src/common.cu:458-531).
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_init(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    phase_init(a, sm);
}
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_spmv_dot(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    phase_spmv_dot(a, sm);
}
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_update(KArgs<Op> a, double alpha) {
    __shared__ double sm[TS_SMEM];
    phase_update(a, alpha, sm);
}
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_true_residual(KArgs<Op> a) {
    __shared__ double sm[TS_SMEM];
    phase_true_residual(a, sm);
}
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_restart(KArgs<Op> a) {
    phase_restart(a);
}
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_p(KArgs<Op> a, double beta) {
    phase_p(a, beta);
}
// Single block: reduce partial slot `which` into out[which].
template <class Op>
__global__ void __launch_bounds__(CG_TILE) k_reduce(KArgs<Op> a, int which, double *out) {
    __shared__ double sm[TS_SMEM];
    const double v = sum_partials(slot(a, which), a.ntiles, sm);
    if (threadIdx.x == 0) out[which] = v;
}

// y = A x, one row per thread.
template <class Op>
__global__ void k_apply(Op op, int n, const double *x, double *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = op.apply(x, i);
}

#undef CFM_TILES
#undef CFM_ROW

}  // namespace cfm
