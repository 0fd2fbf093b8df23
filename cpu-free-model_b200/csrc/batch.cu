// Batched uneven solves in ONE persistent launch (no reference counterpart;
// the reference solves one system per run).
//
// Many independent variable-coefficient systems (2D 5-point and 3D 7-point,
// any sizes) are packed into shared buffers.  The resident blocks of one
// cooperative launch are split into size classes, and each class into teams
// of T_c blocks (T_c from the autotuner).  A team takes the next system of
// its class from an atomic queue (systems sorted largest first), solves it
// with PCG behind a team-local bounded barrier, writes its iteration count
// and status, and takes the next; small systems therefore run many at a
// time on one block each, large ones on wide teams, all concurrently.
//
// Per system: PCG in FP64 with the symmetric damped-Jacobi polynomial
// preconditioner z = J_m(r) (m sweeps of z += omega D^-1 (r - A z) from
// z = 0, omega = 0.8; m = 0 means z = D^-1 r), stopping at the recursive
// residual ||r|| <= tol ||b|| (the host reports the FP64 true residual).
// Dots: per-tile partials (1024 rows), summed in a fixed order by every
// block of the team after the barrier.  The launch is captured in a CUDA
// graph (with the reset of the queues and barriers) and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "barrier.cuh"
#include "cfm_internal.h"
#include "krylov.cuh"

namespace cfm {

namespace {

constexpr int BT_MAXCLS = 4;
constexpr double BT_OMEGA = 0.8;

struct BtSys {
    int dims, nx, ny, nz, n, ntiles;
    long long off;   // first element of this system in the packed n-vectors
    long long poff;  // first partial of this system (4 slots of ntiles)
};

struct BtOut {
    long long iters;
    int status;
    int sweeps;     // FP64 reliable updates (mixed precision); 0 in FP64
    double rr, bb;  // final recursive |r|^2, |b|^2
};

struct BtArgs {
    const BtSys *sys;
    const double *we, *wn, *wt, *dg;  // packed coefficients
    const double *b;
    double *x, *r, *p, *s, *z, *z2;   // packed vectors
    double *part;                     // packed partials
    BtOut *out;
    BarrierState *bars;               // one per team
    int *team_sys;                    // current system of each team
    int *qnext;                       // per class queue position
    const int *order;                 // systems grouped by class, largest first
    int cls_start[BT_MAXCLS], cls_count[BT_MAXCLS];
    int cls_team[BT_MAXCLS];          // team size of the class
    int cls_block0[BT_MAXCLS];        // first block of the class
    int cls_team0[BT_MAXCLS];         // first team index of the class
    int ncls;
    int smooth;
    int maxiter;
    double tol;
    // FP32 iteration with FP64 reliable updates (batch_kernel<true>)
    const float *we32, *wn32, *wt32, *dg32;  // FP32 copies of the coefficients
    float *r32, *p32, *s32, *z32, *y32, *d32; // FP32 inner vectors
    int inner_maxiter;                        // most FP32 steps between updates (0: no cap)
    double inner_tol;
};

__device__ __forceinline__ double bt_apply(const BtArgs &a, const BtSys &S, const double *x,
                                           long long i) {
    const long long g = S.off + i;
    const int nx = S.nx, ny = S.ny;
    const int ix = (int)(i % nx), q = (int)(i / nx), iy = q % ny;
    double t = a.dg[g] * x[g];
    if (ix > 0) t = fma(-a.we[g - 1], x[g - 1], t);
    if (ix < nx - 1) t = fma(-a.we[g], x[g + 1], t);
    if (iy > 0) t = fma(-a.wn[g - nx], x[g - nx], t);
    if (iy < ny - 1) t = fma(-a.wn[g], x[g + nx], t);
    if (S.dims == 3) {
        const int iz = q / ny;
        const long long P = (long long)nx * ny;
        if (iz > 0) t = fma(-a.wt[g - P], x[g - P], t);
        if (iz < S.nz - 1) t = fma(-a.wt[g], x[g + P], t);
    }
    return t;
}

// A x in FP32 from the FP32 coefficient copies (same neighbour order).
__device__ __forceinline__ float bt_apply32(const BtArgs &a, const BtSys &S, const float *x,
                                            long long i) {
    const long long g = S.off + i;
    const int nx = S.nx, ny = S.ny;
    const int ix = (int)(i % nx), q = (int)(i / nx), iy = q % ny;
    float t = a.dg32[g] * x[g];
    if (ix > 0) t = fmaf(-a.we32[g - 1], x[g - 1], t);
    if (ix < nx - 1) t = fmaf(-a.we32[g], x[g + 1], t);
    if (iy > 0) t = fmaf(-a.wn32[g - nx], x[g - nx], t);
    if (iy < ny - 1) t = fmaf(-a.wn32[g], x[g + nx], t);
    if (S.dims == 3) {
        const int iz = q / ny;
        const long long P = (long long)nx * ny;
        if (iz > 0) t = fmaf(-a.wt32[g - P], x[g - P], t);
        if (iz < S.nz - 1) t = fmaf(-a.wt32[g], x[g + P], t);
    }
    return t;
}

// Sum of one partial slot over the system's tiles (fixed order).
__device__ __forceinline__ double bt_sum(const BtArgs &a, const BtSys &S, int slot, double *sm) {
    const double *pp = a.part + S.poff + (long long)slot * S.ntiles;
    double acc = 0.0;
    for (int i = threadIdx.x; i < S.ntiles; i += CG_TILE) acc += pp[i];
    return block_sum(acc, sm);
}

// r_i z_i for the <r, z> partials: the FP64 product, or the exact product
// of two FP32 values as FP64.
__device__ __forceinline__ double bt_prod(double u, double v) { return u * v; }
__device__ __forceinline__ double bt_prod(float u, float v) { return (double)u * (double)v; }

struct BtApply64 {
    __device__ __forceinline__ double operator()(const BtArgs &a, const BtSys &S, const double *x,
                                                 long long i) const {
        return bt_apply(a, S, x, i);
    }
};
struct BtApply32 {
    __device__ __forceinline__ float operator()(const BtArgs &a, const BtSys &S, const float *x,
                                                long long i) const {
        return bt_apply32(a, S, x, i);
    }
};

// Two of a block's tiles per step (tile, tile + T): each pass computes both
// rows' values before storing either, so their loads are in flight together.
struct BtPair {
    int t2;
    bool has2, ok1, ok2;
    long long i1, i2;
    __device__ __forceinline__ BtPair(const BtSys &S, int tile, int T) {
        t2 = tile + T;
        has2 = t2 < S.ntiles;
        i1 = (long long)tile * CG_TILE + threadIdx.x;
        i2 = (long long)t2 * CG_TILE + threadIdx.x;
        ok1 = i1 < S.n;
        ok2 = has2 && i2 < S.n;
    }
};

// Preconditioner z = J_m(r) over the team's tiles (damped Jacobi from
// z = 0: the first sweep is w r / d, or r / d for smooth = 0), with the
// <r, z> partials of the result into slot 0 and, when pcopy is set, p = z,
// both in the last sweep.  Sweeps read z at neighbours, so a team barrier
// separates them; the sweeps alternate between z and z2, starting in the
// one that leaves the result in z.  Returns false on a barrier timeout.
template <class V, class Apply>
__device__ bool bt_precond(const BtArgs &a, const BtSys &S, int rank, int T, BarrierState *bar,
                           int &site, double *sm, const V *r, V *z, V *z2, const V *dg,
                           V *pcopy) {
    const V w = (V)BT_OMEGA;
    const int extra = a.smooth > 1 ? a.smooth - 1 : 0;
    V *src = nullptr, *dst = (extra & 1) ? z2 : z;
    for (int m = 0; m <= extra; ++m) {
        if (m > 0 && !grid_barrier(bar, T, site++)) return false;
        const bool last = m == extra;
        TileSums<1> ts(sm, T, a.part + S.poff);
        auto sweep_at = [&](long long i) -> V {
            const long long g = S.off + i;
            if (m == 0) return a.smooth <= 0 ? r[g] / dg[g] : w * r[g] / dg[g];
            return src[g] + w * (r[g] - Apply()(a, S, src, i)) / dg[g];
        };
        for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
            const BtPair q(S, tile, T);
            const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
            V z1 = V(0), z2 = V(0);
            if (q.ok1) z1 = sweep_at(q.i1);
            if (q.ok2) z2 = sweep_at(q.i2);
            if (q.ok1) dst[g1] = z1;
            if (q.ok2) dst[g2] = z2;
            if (last) {
                double p1 = 0.0, p2 = 0.0;
                if (q.ok1) {
                    if (pcopy) pcopy[g1] = z1;
                    p1 = bt_prod(r[g1], z1);
                }
                if (q.ok2) {
                    if (pcopy) pcopy[g2] = z2;
                    p2 = bt_prod(r[g2], z2);
                }
                ts.add(tile, p1);
                if (q.has2) ts.add(q.t2, p2);
            }
        }
        if (last) ts.flush();
        src = dst;
        dst = dst == z ? z2 : z;
    }
    return true;
}

// Mixed-precision PCG with reliable updates for one system.  The iteration
// runs in FP32 (FP32 operator, preconditioner and vectors r, z, p, s; dots
// as FP64 sums of exact FP32 products; alpha, beta in FP64, applied rounded
// to FP32) and gathers its steps in an FP32 correction d.  When the
// recursive residual falls below the tolerance, below delta times its
// largest norm since the last update (a.inner_tol = delta), or after
// a.inner_maxiter steps (0: no cap), the update folds d into x in FP64 and
// replaces r by the FP64 true residual t = b - A x (rounded to FP32); the
// search direction p is kept, so the Krylov recurrence goes on instead of
// restarting (residual replacement as in Sleijpen and van der Vorst's
// reliable updates).  It stops when |t| <= tol |b| in FP64.  The FP64 r
// array holds t.  Slots: 0 <r, z>, 1 <p, s>, 2 <r, r>, 3 <b, b> then <t, t>.
__device__ bool bt_solve_mixed(const BtArgs &a, int sid, int rank, int T, BarrierState *bar,
                               double *sm) {
    const BtSys S = a.sys[sid];
    int site = 0;
    double *part = a.part + S.poff;
    double *t64 = a.r;
    // x = 0, d = 0, r = fl32(b); |b|^2, |r|^2
    {
        TileSums<2> ts(sm, T, part + 3 * S.ntiles, part + 2 * S.ntiles);
        for (int tile = rank; tile < S.ntiles; tile += T) {
            const long long i = (long long)tile * CG_TILE + threadIdx.x;
            double bb = 0.0, q = 0.0;
            if (i < S.n) {
                const long long g = S.off + i;
                const double bi = a.b[g];
                const float ri = (float)bi;
                a.x[g] = 0.0;
                a.d32[g] = 0.f;
                a.r32[g] = ri;
                bb = bi * bi;
                q = bt_prod(ri, ri);
            }
            ts.add(tile, bb, q);
        }
        ts.flush();
    }
    // z = M r, p = z, <r, z>
    if (!bt_precond<float, BtApply32>(a, S, rank, T, bar, site, sm, a.r32, a.z32, a.y32, a.dg32,
                                      a.p32))
        return false;
    if (!grid_barrier(bar, T, site++)) return false;
    const double bb = bt_sum(a, S, 3, sm);
    const double target2 = a.tol * a.tol * bb;
    const double delta2 = a.inner_tol * a.inner_tol;
    double rr = bt_sum(a, S, 2, sm), rz = bt_sum(a, S, 0, sm);
    double tt = bb, rmax2 = rr;
    long long k = 0;
    int updates = 0, since = 0, status = CFM_NOT_CONVERGED;
    if (tt <= target2) status = CFM_OK;
    while (status != CFM_OK && k < a.maxiter) {
        // s = A p; <p, s>
        {
            TileSums<1> ts(sm, T, part + S.ntiles);
            for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
                const BtPair q(S, tile, T);
                const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
                float s1 = 0.f, s2 = 0.f, p1 = 0.f, p2 = 0.f;
                if (q.ok1) {
                    s1 = bt_apply32(a, S, a.p32, q.i1);
                    p1 = a.p32[g1];
                }
                if (q.ok2) {
                    s2 = bt_apply32(a, S, a.p32, q.i2);
                    p2 = a.p32[g2];
                }
                if (q.ok1) a.s32[g1] = s1;
                if (q.ok2) a.s32[g2] = s2;
                ts.add(tile, q.ok1 ? bt_prod(p1, s1) : 0.0);
                if (q.has2) ts.add(q.t2, q.ok2 ? bt_prod(p2, s2) : 0.0);
            }
            ts.flush();
        }
        if (!grid_barrier(bar, T, site++)) return false;
        const double ps = bt_sum(a, S, 1, sm);
        const double alpha = rz / ps;
        if (!(ps > 0.0 && isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        const float af = (float)alpha;
        // d += alpha p; r -= alpha s; |r|^2
        {
            TileSums<1> ts(sm, T, part + 2 * S.ntiles);
            for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
                const BtPair q(S, tile, T);
                const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
                float d1 = 0.f, p1 = 0.f, s1 = 0.f, r1 = 0.f, d2 = 0.f, p2 = 0.f, s2 = 0.f, r2 = 0.f;
                if (q.ok1) {
                    d1 = a.d32[g1];
                    p1 = a.p32[g1];
                    s1 = a.s32[g1];
                    r1 = a.r32[g1];
                }
                if (q.ok2) {
                    d2 = a.d32[g2];
                    p2 = a.p32[g2];
                    s2 = a.s32[g2];
                    r2 = a.r32[g2];
                }
                double q1 = 0.0, q2 = 0.0;
                if (q.ok1) {
                    a.d32[g1] = fmaf(af, p1, d1);
                    const float ri = fmaf(-af, s1, r1);
                    a.r32[g1] = ri;
                    q1 = bt_prod(ri, ri);
                }
                if (q.ok2) {
                    a.d32[g2] = fmaf(af, p2, d2);
                    const float ri = fmaf(-af, s2, r2);
                    a.r32[g2] = ri;
                    q2 = bt_prod(ri, ri);
                }
                ts.add(tile, q1);
                if (q.has2) ts.add(q.t2, q2);
            }
            ts.flush();
        }
        ++k;
        ++since;
        if (!grid_barrier(bar, T, site++)) return false;
        rr = bt_sum(a, S, 2, sm);
        if (rr <= target2 || rr < delta2 * rmax2 || k >= a.maxiter ||
            (a.inner_maxiter > 0 && since >= a.inner_maxiter)) {
            // reliable update: x += d (FP64), d = 0
            for (int tile = rank; tile < S.ntiles; tile += T) {
                const long long i = (long long)tile * CG_TILE + threadIdx.x;
                if (i < S.n) {
                    const long long g = S.off + i;
                    a.x[g] += (double)a.d32[g];
                    a.d32[g] = 0.f;
                }
            }
            if (!grid_barrier(bar, T, site++)) return false;
            // t = b - A x (FP64), r = fl32(t); |t|^2, |r|^2
            {
                TileSums<2> ts(sm, T, part + 3 * S.ntiles, part + 2 * S.ntiles);
                for (int tile = rank; tile < S.ntiles; tile += T) {
                    const long long i = (long long)tile * CG_TILE + threadIdx.x;
                    double q = 0.0, q32 = 0.0;
                    if (i < S.n) {
                        const long long g = S.off + i;
                        const double ti = a.b[g] - bt_apply(a, S, a.x, i);
                        const float ri = (float)ti;
                        t64[g] = ti;
                        a.r32[g] = ri;
                        q = ti * ti;
                        q32 = bt_prod(ri, ri);
                    }
                    ts.add(tile, q, q32);
                }
                ts.flush();
            }
            if (!grid_barrier(bar, T, site++)) return false;
            tt = bt_sum(a, S, 3, sm);
            rr = bt_sum(a, S, 2, sm);
            ++updates;
            since = 0;
            rmax2 = rr;
            if (tt <= target2) {
                status = CFM_OK;
                break;
            }
            if (k >= a.maxiter) break;
        } else if (rr > rmax2) {
            rmax2 = rr;
        }
        // z = M r, <r, z>
        if (!bt_precond<float, BtApply32>(a, S, rank, T, bar, site, sm, a.r32, a.z32, a.y32,
                                          a.dg32, nullptr))
            return false;
        if (!grid_barrier(bar, T, site++)) return false;
        const double rz1 = bt_sum(a, S, 0, sm);
        const float bf = (float)(rz1 / rz);
        rz = rz1;
        // p = z + beta p
        for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
            const BtPair q(S, tile, T);
            const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
            float p1 = 0.f, z1 = 0.f, p2 = 0.f, z2 = 0.f;
            if (q.ok1) {
                p1 = a.p32[g1];
                z1 = a.z32[g1];
            }
            if (q.ok2) {
                p2 = a.p32[g2];
                z2 = a.z32[g2];
            }
            if (q.ok1) a.p32[g1] = fmaf(bf, p1, z1);
            if (q.ok2) a.p32[g2] = fmaf(bf, p2, z2);
        }
        if (!grid_barrier(bar, T, site++)) return false;
    }
    if (since > 0) {  // a breakdown left steps in d
        for (int tile = rank; tile < S.ntiles; tile += T) {
            const long long i = (long long)tile * CG_TILE + threadIdx.x;
            if (i < S.n) a.x[S.off + i] += (double)a.d32[S.off + i];
        }
    }
    if (rank == 0 && threadIdx.x == 0) {
        a.out[sid].iters = k;
        a.out[sid].status = status;
        a.out[sid].sweeps = updates;
        a.out[sid].rr = tt;
        a.out[sid].bb = bb;
    }
    return true;
}

// Slots: 0 <r, z>, 1 <p, s>, 2 <r, r>, 3 <b, b>.
__device__ bool bt_solve(const BtArgs &a, int sid, int rank, int T, BarrierState *bar,
                         double *sm) {
    const BtSys S = a.sys[sid];
    int site = 0;
    double *part = a.part + S.poff;
    // x = 0, r = b; |b|^2
    {
        TileSums<1> ts(sm, T, part + 3 * S.ntiles);
        for (int tile = rank; tile < S.ntiles; tile += T) {
            const long long i = (long long)tile * CG_TILE + threadIdx.x;
            double bb = 0.0;
            if (i < S.n) {
                const long long g = S.off + i;
                const double bi = a.b[g];
                a.x[g] = 0.0;
                a.r[g] = bi;
                bb = bi * bi;
            }
            ts.add(tile, bb);
        }
        ts.flush();
    }
    // z = M r, p = z, <r, z>
    if (!bt_precond<double, BtApply64>(a, S, rank, T, bar, site, sm, a.r, a.z, a.z2, a.dg, a.p))
        return false;
    if (!grid_barrier(bar, T, site++)) return false;
    const double bb = bt_sum(a, S, 3, sm);
    double rz = bt_sum(a, S, 0, sm);
    const double target2 = a.tol * a.tol * bb;
    long long k = 0;
    double rr = bb;
    int status = CFM_NOT_CONVERGED;
    if (rr <= target2) status = CFM_OK;
    while (status != CFM_OK && k < a.maxiter) {
        // s = A p; <p, s>
        {
            TileSums<1> ts(sm, T, part + S.ntiles);
            for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
                const BtPair q(S, tile, T);
                const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
                double s1 = 0.0, s2 = 0.0, p1 = 0.0, p2 = 0.0;
                if (q.ok1) {
                    s1 = bt_apply(a, S, a.p, q.i1);
                    p1 = a.p[g1];
                }
                if (q.ok2) {
                    s2 = bt_apply(a, S, a.p, q.i2);
                    p2 = a.p[g2];
                }
                if (q.ok1) a.s[g1] = s1;
                if (q.ok2) a.s[g2] = s2;
                ts.add(tile, q.ok1 ? p1 * s1 : 0.0);
                if (q.has2) ts.add(q.t2, q.ok2 ? p2 * s2 : 0.0);
            }
            ts.flush();
        }
        if (!grid_barrier(bar, T, site++)) return false;
        const double ps = bt_sum(a, S, 1, sm);
        const double alpha = rz / ps;
        if (!(ps > 0.0 && isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        // x += alpha p; r -= alpha s; |r|^2
        {
            TileSums<1> ts(sm, T, part + 2 * S.ntiles);
            for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
                const BtPair q(S, tile, T);
                const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
                double x1 = 0.0, p1 = 0.0, s1 = 0.0, r1 = 0.0, x2 = 0.0, p2 = 0.0, s2 = 0.0, r2 = 0.0;
                if (q.ok1) {
                    x1 = a.x[g1];
                    p1 = a.p[g1];
                    s1 = a.s[g1];
                    r1 = a.r[g1];
                }
                if (q.ok2) {
                    x2 = a.x[g2];
                    p2 = a.p[g2];
                    s2 = a.s[g2];
                    r2 = a.r[g2];
                }
                double q1 = 0.0, q2 = 0.0;
                if (q.ok1) {
                    a.x[g1] = fma(alpha, p1, x1);
                    const double ri = fma(-alpha, s1, r1);
                    a.r[g1] = ri;
                    q1 = ri * ri;
                }
                if (q.ok2) {
                    a.x[g2] = fma(alpha, p2, x2);
                    const double ri = fma(-alpha, s2, r2);
                    a.r[g2] = ri;
                    q2 = ri * ri;
                }
                ts.add(tile, q1);
                if (q.has2) ts.add(q.t2, q2);
            }
            ts.flush();
        }
        ++k;
        if (!grid_barrier(bar, T, site++)) return false;
        rr = bt_sum(a, S, 2, sm);
        if (rr <= target2) {
            status = CFM_OK;
            break;
        }
        // z = M r, <r, z>
        if (!bt_precond<double, BtApply64>(a, S, rank, T, bar, site, sm, a.r, a.z, a.z2, a.dg,
                                           nullptr))
            return false;
        if (!grid_barrier(bar, T, site++)) return false;
        const double rz1 = bt_sum(a, S, 0, sm);
        const double beta = rz1 / rz;
        rz = rz1;
        // p = z + beta p
        for (int tile = rank; tile < S.ntiles; tile += 2 * T) {
            const BtPair q(S, tile, T);
            const long long g1 = S.off + q.i1, g2 = S.off + q.i2;
            double p1 = 0.0, z1 = 0.0, p2 = 0.0, z2 = 0.0;
            if (q.ok1) {
                p1 = a.p[g1];
                z1 = a.z[g1];
            }
            if (q.ok2) {
                p2 = a.p[g2];
                z2 = a.z[g2];
            }
            if (q.ok1) a.p[g1] = fma(beta, p1, z1);
            if (q.ok2) a.p[g2] = fma(beta, p2, z2);
        }
        if (!grid_barrier(bar, T, site++)) return false;
    }
    if (rank == 0 && threadIdx.x == 0) {
        a.out[sid].iters = k;
        a.out[sid].status = status;
        a.out[sid].sweeps = 0;
        a.out[sid].rr = rr;
        a.out[sid].bb = bb;
    }
    return true;
}

template <bool MIXED>
__global__ void __launch_bounds__(CG_TILE, 1) batch_kernel(BtArgs a) {
    __shared__ double sm[TS_SMEM];
    __shared__ int s_sys;
    int c = 0;
    while (c + 1 < a.ncls && (int)blockIdx.x >= a.cls_block0[c + 1]) ++c;
    const int T = a.cls_team[c];
    const int rel = (int)blockIdx.x - a.cls_block0[c];
    const int team = a.cls_team0[c] + rel / T, rank = rel % T;
    BarrierState *bar = a.bars + team;
    while (true) {
        if (rank == 0 && threadIdx.x == 0) {
            const int q = atomicAdd(a.qnext + c, 1);
            a.team_sys[team] = q < a.cls_count[c] ? a.order[a.cls_start[c] + q] : -1;
        }
        if (!grid_barrier(bar, T, -1)) return;
        if (threadIdx.x == 0) s_sys = *((volatile int *)(a.team_sys + team));
        __syncthreads();
        const int sid = s_sys;
        if (sid < 0) return;
        if (!(MIXED ? bt_solve_mixed(a, sid, rank, T, bar, sm) : bt_solve(a, sid, rank, T, bar, sm)))
            return;
        // everyone has read team_sys before the leader overwrites it
        if (!grid_barrier(bar, T, -2)) return;
    }
}

__global__ void batch_reset(BarrierState *bars, int nteams, int *qnext, int ncls,
                            unsigned long long timeout_ns) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nteams; t += gridDim.x * blockDim.x) {
        bars[t].count = 0;
        bars[t].gen = 0;
        bars[t].error = 0;
        bars[t].where = 0;
        bars[t].timeout_ns = timeout_ns;
    }
    if (blockIdx.x == 0 && threadIdx.x < ncls) qnext[threadIdx.x] = 0;
}

__global__ void batch_to_f32(const double *in, float *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// True residual of every system: rr_true[s] += |b - A x|^2 (atomics).
__global__ void batch_true_res(BtArgs a, int nsys, double *rr_true) {
    for (int sid = blockIdx.y; sid < nsys; sid += gridDim.y) {
        const BtSys S = a.sys[sid];
        double q = 0.0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < S.n;
             i += (long long)gridDim.x * blockDim.x) {
            const double t = a.b[S.off + i] - bt_apply(a, S, a.x, i);
            q += t * t;
        }
        for (int o = 16; o; o >>= 1) q += __shfl_xor_sync(CG_FULL, q, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(rr_true + sid, q);
    }
}

}  // namespace
}  // namespace cfm

using namespace cfm;

struct cfm_batch {
    int nsys = 0;
    std::vector<BtSys> sys;
    long long ntot = 0, ptot = 0;
    BtSys *d_sys = nullptr;
    double *coef = nullptr;  // we | wn | wt | dg  (4 ntot)
    double *vec = nullptr;   // b x r p s z z2      (7 ntot)
    double *part = nullptr;
    BtOut *out = nullptr;
    int *team_sys = nullptr, *qnext = nullptr, *order = nullptr;
    BarrierState *bars = nullptr;
    double *rr_true = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    // launch configuration (autotuned)
    int ncls = 0, blocks = 0, nteams = 0;
    int cls_team[BT_MAXCLS] = {}, cls_block0[BT_MAXCLS] = {}, cls_team0[BT_MAXCLS] = {};
    int cls_start[BT_MAXCLS] = {}, cls_count[BT_MAXCLS] = {};
    long long thr[BT_MAXCLS] = {};
    int smooth = 4, maxiter = 20000;
    double tol = 1e-8;
    // FP32 iteration with FP64 reliable updates
    bool mixed = false;
    int inner_maxiter = 0;
    double inner_tol = 0.1;
    float *coef32 = nullptr;  // we | wn | wt | dg in FP32 (4 ntot)
    float *vec32 = nullptr;   // r p s z y d in FP32   (6 ntot)
};

namespace {

// Drop the captured graph (the launch it holds no longer matches).
void drop_graph(cfm_batch *h) {
    if (h->exec) {
        cudaGraphExecDestroy(h->exec);
        h->exec = nullptr;
    }
    if (h->graph) {
        cudaGraphDestroy(h->graph);
        h->graph = nullptr;
    }
}

// Classes by size: class c holds systems with n >= thr[c] (thr descending,
// thr[ncls-1] = 0); blocks are shared out in proportion to each class's
// work estimate sum(n * side), rounded to whole teams.
int plan(cfm_batch *h, int ncls, const long long *thr, const int *team, int blocks) {
    CFM_ARG_CHECK(ncls >= 1 && ncls <= BT_MAXCLS, "classes");
    std::vector<int> idx(h->nsys);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return h->sys[x].n > h->sys[y].n; });
    std::vector<int> order;
    std::vector<double> work(ncls, 0.0);
    int start = 0;
    for (int c = 0; c < ncls; ++c) {
        h->cls_start[c] = start;
        int cnt = 0;
        for (int i : idx) {
            const long long n = h->sys[i].n;
            const bool in = n >= thr[c] && (c == 0 || n < thr[c - 1]);
            if (!in) continue;
            order.push_back(i);
            ++cnt;
            const BtSys &S = h->sys[i];
            const double side = S.dims == 3 ? std::cbrt((double)n) : std::sqrt((double)n);
            work[c] += (double)n * side;
        }
        h->cls_count[c] = cnt;
        start += cnt;
    }
    CFM_ARG_CHECK((int)order.size() == h->nsys, "class thresholds must cover every system");
    const double wsum = std::accumulate(work.begin(), work.end(), 0.0);
    int b0 = 0, t0 = 0;
    for (int c = 0; c < ncls; ++c) {
        int nb;
        if (c == ncls - 1) {
            nb = blocks - b0;
        } else {
            nb = (int)std::lround(blocks * (wsum > 0 ? work[c] / wsum : 1.0 / ncls));
        }
        nb = std::max(h->cls_count[c] > 0 ? team[c] : 0, nb / team[c] * team[c]);
        if (b0 + nb > blocks) nb = (blocks - b0) / team[c] * team[c];
        if (h->cls_count[c] > 0 && nb < team[c]) {
            set_error("not enough resident blocks for the class plan");
            return CFM_UNSUPPORTED;
        }
        h->cls_team[c] = team[c];
        h->cls_block0[c] = b0;
        h->cls_team0[c] = t0;
        b0 += nb;
        t0 += nb / team[c];
        h->thr[c] = thr[c];
    }
    h->ncls = ncls;
    h->blocks = b0;
    h->nteams = t0;
    drop_graph(h);
    if (h->order) cudaFree(h->order);
    if (h->bars) cudaFree(h->bars);
    if (h->team_sys) cudaFree(h->team_sys);
    h->order = nullptr;
    h->bars = nullptr;
    h->team_sys = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&h->order, sizeof(int) * std::max(1, h->nsys)));
    CFM_CUDA_TRY(cudaMalloc(&h->bars, sizeof(BarrierState) * std::max(1, h->nteams)));
    CFM_CUDA_TRY(cudaMalloc(&h->team_sys, sizeof(int) * std::max(1, h->nteams)));
    CFM_CUDA_TRY(cudaMemcpy(h->order, order.data(), sizeof(int) * h->nsys, cudaMemcpyHostToDevice));
    return CFM_OK;
}

BtArgs bt_args(cfm_batch *h) {
    BtArgs a{};
    const long long N = h->ntot;
    a.sys = h->d_sys;
    a.we = h->coef;
    a.wn = h->coef + N;
    a.wt = h->coef + 2 * N;
    a.dg = h->coef + 3 * N;
    a.b = h->vec;
    a.x = h->vec + N;
    a.r = h->vec + 2 * N;
    a.p = h->vec + 3 * N;
    a.s = h->vec + 4 * N;
    a.z = h->vec + 5 * N;
    a.z2 = h->vec + 6 * N;
    a.part = h->part;
    a.out = h->out;
    a.bars = h->bars;
    a.team_sys = h->team_sys;
    a.qnext = h->qnext;
    a.order = h->order;
    for (int c = 0; c < BT_MAXCLS; ++c) {
        a.cls_start[c] = h->cls_start[c];
        a.cls_count[c] = h->cls_count[c];
        a.cls_team[c] = h->cls_team[c];
        a.cls_block0[c] = h->cls_block0[c];
        a.cls_team0[c] = h->cls_team0[c];
    }
    a.ncls = h->ncls;
    a.smooth = h->smooth;
    a.maxiter = h->maxiter;
    a.tol = h->tol;
    if (h->coef32 && h->vec32) {
        a.we32 = h->coef32;
        a.wn32 = h->coef32 + N;
        a.wt32 = h->coef32 + 2 * N;
        a.dg32 = h->coef32 + 3 * N;
        a.r32 = h->vec32;
        a.p32 = h->vec32 + N;
        a.s32 = h->vec32 + 2 * N;
        a.z32 = h->vec32 + 3 * N;
        a.y32 = h->vec32 + 4 * N;
        a.d32 = h->vec32 + 5 * N;
    }
    a.inner_maxiter = h->inner_maxiter;
    a.inner_tol = h->inner_tol;
    return a;
}


// Reset + the persistent launch, on h->stream (capturable).
int enqueue(cfm_batch *h) {
    BtArgs a = bt_args(h);
    batch_reset<<<std::max(1, (h->nteams + 255) / 256), 256, 0, h->stream>>>(
        h->bars, h->nteams, h->qnext, h->ncls, barrier_timeout_ns());
    CFM_CUDA_TRY(cudaGetLastError());
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(h->blocks);
    cfg.blockDim = dim3(CG_TILE);
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (h->mixed)
        CFM_CUDA_TRY(cudaLaunchKernelEx(&cfg, batch_kernel<true>, a));
    else
        CFM_CUDA_TRY(cudaLaunchKernelEx(&cfg, batch_kernel<false>, a));
    return CFM_OK;
}

int build_graph_batch(cfm_batch *h) {
    CFM_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int st = enqueue(h);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (st) return st;
    CFM_CUDA_TRY(e);
    h->graph = g;
    CFM_CUDA_TRY(cudaGraphInstantiate(&h->exec, g, 0));
    return CFM_OK;
}

int run_once(cfm_batch *h, float *ms) {
    if (!h->exec) {
        int st = build_graph_batch(h);
        if (st) return st;
    }
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    CFM_CUDA_TRY(cudaGraphLaunch(h->exec, h->stream));
    CFM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    CFM_CUDA_TRY(cudaEventSynchronize(h->ev1));
    CFM_CUDA_TRY(cudaEventElapsedTime(ms, h->ev0, h->ev1));
    std::vector<BarrierState> bs(h->nteams);
    CFM_CUDA_TRY(cudaMemcpy(bs.data(), h->bars, sizeof(BarrierState) * h->nteams,
                            cudaMemcpyDeviceToHost));
    for (const auto &b : bs)
        if (b.error) {
            set_error("batched solve: a team barrier timed out");
            return CFM_BARRIER_TIMEOUT;
        }
    return CFM_OK;
}

int resident_blocks(int *out) {
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    int per_sm64 = 0, per_sm32 = 0;
    CFM_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm64, batch_kernel<false>, CG_TILE, 0));
    CFM_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, batch_kernel<true>, CG_TILE, 0));
    *out = std::min(per_sm64, per_sm32) * di.num_sms;
    return CFM_OK;
}

}  // namespace

extern "C" {

int cfm_batch_create(int nsys, const int *dims, const int *nx, const int *ny, const int *nz,
                     const double *const *k_host, const double *const *b_host, cfm_batch **out) {
    clear_error();
    CFM_ARG_CHECK(out && nsys >= 1 && dims && nx && ny && nz && k_host && b_host, "null argument");
    *out = nullptr;
    cfm_batch *h = new cfm_batch();
    h->nsys = nsys;
    h->sys.resize(nsys);
    long long off = 0, poff = 0;
    for (int i = 0; i < nsys; ++i) {
        BtSys &S = h->sys[i];
        S.dims = dims[i];
        S.nx = nx[i];
        S.ny = ny[i];
        S.nz = dims[i] == 3 ? nz[i] : 1;
        if (!(S.dims == 2 || S.dims == 3) || S.nx < 1 || S.ny < 1 || S.nz < 1 || !k_host[i] ||
            !b_host[i]) {
            delete h;
            set_error("bad argument: system %d", i);
            return CFM_BAD_ARG;
        }
        const long long n = (long long)S.nx * S.ny * S.nz;
        S.n = (int)n;
        S.ntiles = (int)((n + CG_TILE - 1) / CG_TILE);
        S.off = off;
        S.poff = poff;
        off += n;
        poff += 4LL * S.ntiles;
    }
    h->ntot = off;
    h->ptot = poff;
    auto fail = [&](cudaError_t e) {
        cfm_batch_destroy(h);
        set_error("batch setup failed: %s", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_sys, sizeof(BtSys) * nsys)) != cudaSuccess ||
        (e = cudaMalloc(&h->coef, sizeof(double) * 4 * off)) != cudaSuccess ||
        (e = cudaMalloc(&h->vec, sizeof(double) * 7 * off)) != cudaSuccess ||
        (e = cudaMalloc(&h->part, sizeof(double) * poff)) != cudaSuccess ||
        (e = cudaMalloc(&h->out, sizeof(BtOut) * nsys)) != cudaSuccess ||
        (e = cudaMalloc(&h->qnext, sizeof(int) * BT_MAXCLS)) != cudaSuccess ||
        (e = cudaMalloc(&h->rr_true, sizeof(double) * nsys)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev0)) != cudaSuccess || (e = cudaEventCreate(&h->ev1)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemcpy(h->d_sys, h->sys.data(), sizeof(BtSys) * nsys, cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return fail(e);
    std::vector<double> c;
    for (int i = 0; i < nsys; ++i) {
        const BtSys &S = h->sys[i];
        c.assign(4 * (size_t)S.n, 0.0);
        const size_t n = S.n;
        int st = cfm_varcoef_coeffs(S.dims, S.nx, S.ny, S.nz, k_host[i], c.data(), c.data() + n,
                                    c.data() + 2 * n, c.data() + 3 * n);
        if (st) {
            cfm_batch_destroy(h);
            return st;
        }
        for (int q = 0; q < 4; ++q)
            if ((e = cudaMemcpy(h->coef + q * off + S.off, c.data() + q * n, sizeof(double) * n,
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return fail(e);
        if ((e = cudaMemcpy(h->vec + S.off, b_host[i], sizeof(double) * n, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return fail(e);
    }
    // default plan: three classes, team sizes 16 / 4 / 1
    int blocks = 0;
    int st = resident_blocks(&blocks);
    if (st) {
        cfm_batch_destroy(h);
        return st;
    }
    const long long thr[3] = {1LL << 18, 1LL << 15, 0};
    const int team[3] = {16, 4, 1};
    if ((st = plan(h, 3, thr, team, blocks))) {
        cfm_batch_destroy(h);
        return st;
    }
    *out = h;
    return CFM_OK;
}

void cfm_batch_destroy(cfm_batch *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    cudaFree(h->d_sys);
    cudaFree(h->coef);
    cudaFree(h->vec);
    cudaFree(h->part);
    cudaFree(h->out);
    cudaFree(h->qnext);
    cudaFree(h->order);
    cudaFree(h->bars);
    cudaFree(h->team_sys);
    cudaFree(h->rr_true);
    cudaFree(h->coef32);
    cudaFree(h->vec32);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int cfm_batch_set_plan(cfm_batch *h, int ncls, const long long *thresholds, const int *team_sizes) {
    clear_error();
    CFM_ARG_CHECK(h && thresholds && team_sizes, "null argument");
    for (int c = 0; c < ncls; ++c)
        CFM_ARG_CHECK(team_sizes[c] >= 1 && team_sizes[c] <= 64, "team size in [1, 64]");
    CFM_ARG_CHECK(thresholds[ncls - 1] == 0, "the last class threshold must be 0");
    int blocks = 0;
    int st = resident_blocks(&blocks);
    if (st) return st;
    return plan(h, ncls, thresholds, team_sizes, blocks);
}

int cfm_batch_set_solver(cfm_batch *h, int smooth, int maxiter, double tol) {
    CFM_ARG_CHECK(h && smooth >= 0 && smooth <= 16 && maxiter > 0 && tol > 0, "solver parameters");
    h->smooth = smooth;
    h->maxiter = maxiter;
    h->tol = tol;
    drop_graph(h);
    return CFM_OK;
}

int cfm_batch_set_precision(cfm_batch *h, int precision, int inner_maxiter, double inner_tol) {
    clear_error();
    CFM_ARG_CHECK(h && (precision == CFM_FP64 || precision == CFM_FP32), "precision");
    CFM_ARG_CHECK(inner_maxiter >= 0 && inner_tol >= 0 && inner_tol < 1,
                  "inner_maxiter >= 0, 0 <= inner_tol < 1");
    if (precision == CFM_FP32 && !h->coef32) {
        const long long N = h->ntot;
        cudaError_t e;
        if ((e = cudaMalloc(&h->coef32, sizeof(float) * 4 * N)) != cudaSuccess ||
            (e = cudaMalloc(&h->vec32, sizeof(float) * 6 * N)) != cudaSuccess) {
            cudaFree(h->coef32);
            cudaFree(h->vec32);
            h->coef32 = nullptr;
            h->vec32 = nullptr;
            set_error("batch FP32 arrays: %s", cudaGetErrorString(e));
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
        }
        batch_to_f32<<<1024, 256, 0, h->stream>>>(h->coef, h->coef32, 4 * N);
        CFM_CUDA_TRY(cudaGetLastError());
        CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    h->mixed = precision == CFM_FP32;
    h->inner_maxiter = inner_maxiter;
    h->inner_tol = inner_tol > 0 ? inner_tol : 0.1;
    drop_graph(h);
    return CFM_OK;
}

// Solve every system (one graph launch = one persistent kernel).  iters /
// status / relres (true FP64 relative residual) per system, optional.
int cfm_batch_solve(cfm_batch *h, long long *iters, int *status, double *relres, cfm_stats *st) {
    const cfm::NvtxRange nvtx_range("cfm_batch_solve");
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    float ms = 0;
    int e = run_once(h, &ms);
    if (e) return e;
    std::vector<BtOut> o(h->nsys);
    CFM_CUDA_TRY(cudaMemcpy(o.data(), h->out, sizeof(BtOut) * h->nsys, cudaMemcpyDeviceToHost));
    std::vector<double> rt(h->nsys, 0.0);
    if (relres) {
        CFM_CUDA_TRY(cudaMemsetAsync(h->rr_true, 0, sizeof(double) * h->nsys, h->stream));
        BtArgs a = bt_args(h);
        batch_true_res<<<dim3(64, std::min(h->nsys, 1024)), 256, 0, h->stream>>>(a, h->nsys, h->rr_true);
        CFM_CUDA_TRY(cudaGetLastError());
        CFM_CUDA_TRY(cudaMemcpyAsync(rt.data(), h->rr_true, sizeof(double) * h->nsys,
                                     cudaMemcpyDeviceToHost, h->stream));
        CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    int worst = CFM_OK;
    long long total = 0, sweeps = 0;
    for (int i = 0; i < h->nsys; ++i) {
        if (iters) iters[i] = o[i].iters;
        if (status) status[i] = o[i].status;
        if (relres) relres[i] = o[i].bb > 0 ? std::sqrt(rt[i] / o[i].bb) : std::sqrt(rt[i]);
        if (o[i].status != CFM_OK) worst = o[i].status;
        total += o[i].iters;
        sweeps += o[i].sweeps;
    }
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->seconds = ms * 1e-3;
        st->iterations = total;
        st->launches = 2;
        st->status = worst;
        st->refinements = sweeps;
    }
    return worst;
}

// Copy the solution of system i into x_host (n doubles).
int cfm_batch_solution(cfm_batch *h, int i, double *x_host) {
    CFM_ARG_CHECK(h && x_host && i >= 0 && i < h->nsys, "arguments");
    const BtSys &S = h->sys[i];
    CFM_CUDA_TRY(cudaMemcpy(x_host, h->vec + h->ntot + S.off, sizeof(double) * S.n,
                            cudaMemcpyDeviceToHost));
    return CFM_OK;
}

// Autotuner: times each candidate (classes, thresholds, team sizes) on the
// real batch and keeps the fastest; `best_ms` gets its time.
int cfm_batch_autotune(cfm_batch *h, double *best_ms) {
    const cfm::NvtxRange nvtx_range("cfm_batch_autotune");
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    struct Cand {
        int ncls;
        long long thr[BT_MAXCLS];
        int team[BT_MAXCLS];
    };
    const Cand cands[] = {
        {3, {1LL << 18, 1LL << 15, 0}, {16, 4, 1}},
        {3, {1LL << 18, 1LL << 15, 0}, {8, 2, 1}},
        {3, {1LL << 19, 1LL << 16, 0}, {32, 4, 1}},
        {3, {1LL << 17, 1LL << 14, 0}, {8, 2, 1}},
        {2, {1LL << 16, 0}, {8, 1}},
        {4, {1LL << 19, 1LL << 17, 1LL << 14, 0}, {32, 8, 2, 1}},
    };
    double best = 1e300;
    int bi = -1;
    for (int c = 0; c < (int)(sizeof(cands) / sizeof(cands[0])); ++c) {
        if (cfm_batch_set_plan(h, cands[c].ncls, cands[c].thr, cands[c].team) != CFM_OK) continue;
        float ms = 0;
        int e = run_once(h, &ms);
        if (e) return e;
        if (ms < best) {
            best = ms;
            bi = c;
        }
    }
    CFM_ARG_CHECK(bi >= 0, "no candidate plan fits this device");
    int st = cfm_batch_set_plan(h, cands[bi].ncls, cands[bi].thr, cands[bi].team);
    if (st) return st;
    if (best_ms) *best_ms = best;
    return CFM_OK;
}

}  // extern "C"
