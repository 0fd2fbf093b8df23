// Conjugate gradient on one GPU: the CPU-free persistent kernel, the
// host-controlled comparator, and the cfm_csr / cfm_cg handles.
//
// Algorithm (standard CG, CG/src/common.cu:399-538 and
// CG/src/single-stream/standard.cu:158-299):
//   r0 = b - A x0, p0 = r0, gamma0 = <r0, r0>
//   s = A p; delta = <p, s>; alpha = gamma0 / delta
//   x += alpha p; r -= alpha s; gamma1 = <r, r>; beta = gamma1 / gamma0
//   p = r + beta p
// The reference sums the dots with atomicAdd(double) in arrival order
// (CG/src/common.cu:357-389); here every dot is a fixed tree -- tiles of 1024
// consecutive entries, xor-butterfly within each warp, then across the 32
// warp sums; the tile partials are summed the same way -- so the result does
// not depend on the launch shape and the host oracle reproduces it exactly.
// With tol > 0 the loop stops when the recursive residual reaches
// tol * ||b|| and the FP64 true residual b - A x confirms it (a restart from
// the true residual otherwise); tol <= 0 runs exactly maxiter iterations like
// the reference's -niter.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "barrier.cuh"
#include "cfm_internal.h"

namespace cfm {

constexpr int CG_TILE = 1024;  // rows per tile == threads per block
constexpr unsigned CG_FULL = 0xffffffffu;

struct CgResult {
    long long iters;
    int status;
    int restarts;
    double gamma;
    double bnorm;
};

struct CgArgs {
    int n;
    int ntiles;
    const int *rowptr;
    const int *col;
    const double *val;
    const double *b;  // nullptr: ones
    double *x, *r, *p, *s, *t;
    double *part;  // 4 * ntiles partials: gamma | delta | true residual | b
    CgResult *res;
    BarrierState *bar;
    int maxiter;
    double tol;
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

__device__ __forceinline__ double row_spmv(const int *rowptr, const int *col, const double *val,
                                           const double *x, int i) {
    double acc = 0.0;
    const int j1 = rowptr[i + 1];
    for (int j = rowptr[i]; j < j1; ++j) acc = __fma_rn(val[j], x[col[j]], acc);
    return acc;
}

__device__ __forceinline__ double row_spmv_zero(const int *rowptr, const double *val, int i) {
    double acc = 0.0;
    const int j1 = rowptr[i + 1];
    for (int j = rowptr[i]; j < j1; ++j) acc = __fma_rn(val[j], 0.0, acc);
    return acc;
}

// ---------------------------------------------------------------- phases
// Each phase processes whole tiles (one row per thread) and writes one
// partial per tile; tiles are dealt to blocks round-robin.

__device__ void phase_init(const CgArgs &a, double *sm) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        double g = 0.0, bb = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double s0 = row_spmv_zero(a.rowptr, a.val, i);  // A x0 with x0 = 0
            const double ri = __fma_rn(-1.0, s0, bi);
            a.x[i] = 0.0;
            a.r[i] = ri;
            a.p[i] = ri;
            g = __dmul_rn(ri, ri);
            bb = __dmul_rn(bi, bi);
        }
        g = block_sum(g, sm);
        bb = block_sum(bb, sm);
        if (threadIdx.x == 0) {
            a.part[tile] = g;
            a.part[3 * a.ntiles + tile] = bb;
        }
    }
}

__device__ void phase_spmv_dot(const CgArgs &a, double *sm) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        double d = 0.0;
        if (i < a.n) {
            const double si = row_spmv(a.rowptr, a.col, a.val, a.p, i);
            a.s[i] = si;
            d = __dmul_rn(a.p[i], si);
        }
        d = block_sum(d, sm);
        if (threadIdx.x == 0) a.part[a.ntiles + tile] = d;
    }
}

__device__ void phase_update(const CgArgs &a, double alpha, double *sm) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        double g = 0.0;
        if (i < a.n) {
            a.x[i] = __fma_rn(alpha, a.p[i], a.x[i]);
            const double ri = __fma_rn(-alpha, a.s[i], a.r[i]);
            a.r[i] = ri;
            g = __dmul_rn(ri, ri);
        }
        g = block_sum(g, sm);
        if (threadIdx.x == 0) a.part[tile] = g;
    }
}

__device__ void phase_true_residual(const CgArgs &a, double *sm) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        double q = 0.0;
        if (i < a.n) {
            const double bi = a.b ? a.b[i] : 1.0;
            const double ti = __dsub_rn(bi, row_spmv(a.rowptr, a.col, a.val, a.x, i));
            a.t[i] = ti;
            q = __dmul_rn(ti, ti);
        }
        q = block_sum(q, sm);
        if (threadIdx.x == 0) a.part[2 * a.ntiles + tile] = q;
    }
}

__device__ void phase_restart(const CgArgs &a) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        if (i < a.n) {
            a.r[i] = a.t[i];
            a.p[i] = a.t[i];
        }
    }
}

__device__ void phase_p(const CgArgs &a, double beta) {
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const int i = tile * CG_TILE + threadIdx.x;
        if (i < a.n) a.p[i] = __fma_rn(beta, a.p[i], a.r[i]);
    }
}

// The whole solve in one cooperative launch; 3 grid barriers per iteration.
__global__ void __launch_bounds__(CG_TILE, 1) cg_persistent_kernel(CgArgs a) {
    __shared__ double sm[33];
    int site = 0;
    phase_init(a, sm);
    if (!grid_barrier(a.bar, gridDim.x, site++)) return;
    double gamma0 = sum_partials(a.part, a.ntiles, sm);
    const double bnorm = sqrt(sum_partials(a.part + 3 * a.ntiles, a.ntiles, sm));
    const bool use_tol = a.tol > 0.0;
    const double target = a.tol * bnorm;
    int status = use_tol ? CFM_NOT_CONVERGED : CFM_OK;
    int restarts = 0;
    long long k = 0;
    if (use_tol && sqrt(gamma0) <= target) status = CFM_OK;
    while (k < a.maxiter && !(use_tol && status == CFM_OK)) {
        phase_spmv_dot(a, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        const double delta = sum_partials(a.part + a.ntiles, a.ntiles, sm);
        const double alpha = gamma0 / delta;
        if (use_tol && !(delta > 0.0 && isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        phase_update(a, alpha, sm);
        if (!grid_barrier(a.bar, gridDim.x, site++)) return;
        const double gamma1 = sum_partials(a.part, a.ntiles, sm);
        ++k;
        if (use_tol && sqrt(gamma1) <= target) {
            phase_true_residual(a, sm);
            if (!grid_barrier(a.bar, gridDim.x, site++)) return;
            const double tt = sum_partials(a.part + 2 * a.ntiles, a.ntiles, sm);
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.res->iters = k;
        a.res->status = status;
        a.res->restarts = restarts;
        a.res->gamma = gamma0;
        a.res->bnorm = bnorm;
    }
}

// ------------------------------------------------ host-controlled comparator
// One kernel per operation and a host read of every dot, as
// SingleGPUDiscreteStandard::run_single_gpu does (CG/src/common.cu:458-531).
__global__ void __launch_bounds__(CG_TILE) k_init(CgArgs a) {
    __shared__ double sm[33];
    phase_init(a, sm);
}
__global__ void __launch_bounds__(CG_TILE) k_spmv_dot(CgArgs a) {
    __shared__ double sm[33];
    phase_spmv_dot(a, sm);
}
__global__ void __launch_bounds__(CG_TILE) k_update(CgArgs a, double alpha) {
    __shared__ double sm[33];
    phase_update(a, alpha, sm);
}
__global__ void __launch_bounds__(CG_TILE) k_true_residual(CgArgs a) {
    __shared__ double sm[33];
    phase_true_residual(a, sm);
}
__global__ void __launch_bounds__(CG_TILE) k_restart(CgArgs a) { phase_restart(a); }
__global__ void __launch_bounds__(CG_TILE) k_p(CgArgs a, double beta) { phase_p(a, beta); }
// Single block: reduce partial slot `which` into out[which].
__global__ void __launch_bounds__(CG_TILE) k_reduce(CgArgs a, int which, double *out) {
    __shared__ double sm[33];
    const double v = sum_partials(a.part + (size_t)which * a.ntiles, a.ntiles, sm);
    if (threadIdx.x == 0) out[which] = v;
}

// y = A x, one row per thread (row order, fma accumulation).
__global__ void k_spmv(int n, const int *rowptr, const int *col, const double *val,
                       const double *x, double *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = row_spmv(rowptr, col, val, x, i);
}

}  // namespace cfm

using namespace cfm;

struct cfm_csr {
    int n = 0;
    long long nnz = 0;
    int *rowptr = nullptr;
    int *col = nullptr;
    double *val = nullptr;
};

struct cfm_cg {
    cfm_cg_params p{};
    const cfm_csr *A = nullptr;
    int ntiles = 0;
    double *vec = nullptr;  // x r p s t b (6 n)
    double *part = nullptr;
    double *scal = nullptr;  // 4 reduced scalars (discrete variant)
    CgResult *res = nullptr;
    BarrierState *bar = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int blocks = 0;
};

namespace {

CgArgs make_args(cfm_cg *h, const double *b_dev, double *x_dev) {
    CgArgs a{};
    const int n = h->A->n;
    a.n = n;
    a.ntiles = h->ntiles;
    a.rowptr = h->A->rowptr;
    a.col = h->A->col;
    a.val = h->A->val;
    a.b = b_dev;
    a.x = x_dev ? x_dev : h->vec;
    a.r = h->vec + (size_t)n;
    a.p = h->vec + 2 * (size_t)n;
    a.s = h->vec + 3 * (size_t)n;
    a.t = h->vec + 4 * (size_t)n;
    a.part = h->part;
    a.res = h->res;
    a.bar = h->bar;
    a.maxiter = h->p.maxiter;
    a.tol = h->p.tol;
    return a;
}

int run_discrete(cfm_cg *h, const CgArgs &a, CgResult *out, int *launches) {
    const int g = a.ntiles;
    cudaStream_t st = h->stream;
    double hs[4];
    auto fetch = [&](int which) -> int {
        k_reduce<<<1, CG_TILE, 0, st>>>(a, which, h->scal);
        CFM_CUDA_TRY(cudaGetLastError());
        CFM_CUDA_TRY(cudaMemcpyAsync(&hs[which], h->scal + which, sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        CFM_CUDA_TRY(cudaStreamSynchronize(st));
        *launches += 1;
        return CFM_OK;
    };
    int e;
    k_init<<<g, CG_TILE, 0, st>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    *launches += 1;
    if ((e = fetch(0)) || (e = fetch(3))) return e;
    double gamma0 = hs[0];
    const double bnorm = std::sqrt(hs[3]);
    const bool use_tol = a.tol > 0.0;
    const double target = a.tol * bnorm;
    int status = use_tol ? CFM_NOT_CONVERGED : CFM_OK;
    int restarts = 0;
    long long k = 0;
    if (use_tol && std::sqrt(gamma0) <= target) status = CFM_OK;
    while (k < a.maxiter && !(use_tol && status == CFM_OK)) {
        k_spmv_dot<<<g, CG_TILE, 0, st>>>(a);
        *launches += 1;
        if ((e = fetch(1))) return e;
        const double delta = hs[1];
        const double alpha = gamma0 / delta;
        if (use_tol && !(delta > 0.0 && std::isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        k_update<<<g, CG_TILE, 0, st>>>(a, alpha);
        *launches += 1;
        if ((e = fetch(0))) return e;
        const double gamma1 = hs[0];
        ++k;
        if (use_tol && std::sqrt(gamma1) <= target) {
            k_true_residual<<<g, CG_TILE, 0, st>>>(a);
            *launches += 1;
            if ((e = fetch(2))) return e;
            if (std::sqrt(hs[2]) <= target) {
                status = CFM_OK;
                gamma0 = gamma1;
                break;
            }
            k_restart<<<g, CG_TILE, 0, st>>>(a);
            *launches += 1;
            ++restarts;
            gamma0 = hs[2];
            continue;
        }
        const double beta = gamma1 / gamma0;
        if (use_tol && !std::isfinite(beta)) {
            status = CFM_BREAKDOWN;
            break;
        }
        k_p<<<g, CG_TILE, 0, st>>>(a, beta);
        *launches += 1;
        gamma0 = gamma1;
    }
    CFM_CUDA_TRY(cudaGetLastError());
    out->iters = k;
    out->status = status;
    out->restarts = restarts;
    out->gamma = gamma0;
    out->bnorm = bnorm;
    return CFM_OK;
}

// Final FP64 true relative residual (after the timed region).
int true_relres(cfm_cg *h, const CgArgs &a, double bnorm, double *out) {
    k_true_residual<<<a.ntiles, CG_TILE, 0, h->stream>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    k_reduce<<<1, CG_TILE, 0, h->stream>>>(a, 2, h->scal);
    CFM_CUDA_TRY(cudaGetLastError());
    double tt = 0;
    CFM_CUDA_TRY(cudaMemcpyAsync(&tt, h->scal + 2, sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    *out = bnorm > 0 ? std::sqrt(tt) / bnorm : std::sqrt(tt);
    return CFM_OK;
}

int solve_impl(cfm_cg *h, const double *b_dev, double *x_dev, cfm_stats *st, double h2d,
               double d2h, const double *b_host, double *x_host) {
    const int n = h->A->n;
    CgArgs a = make_args(h, b_dev, x_dev);
    BarrierState bs{};
    bs.timeout_ns = barrier_timeout_ns();
    CFM_CUDA_TRY(cudaMemcpyAsync(h->bar, &bs, sizeof(bs), cudaMemcpyHostToDevice, h->stream));
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    int launches = 0;
    CgResult r{};
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    if (b_host) {
        CFM_CUDA_TRY(cudaMemcpyAsync((void *)b_dev, b_host, sizeof(double) * n,
                                     cudaMemcpyHostToDevice, h->stream));
    }
    if (h->p.impl == CFM_CG_DISCRETE) {
        int e = run_discrete(h, a, &r, &launches);
        if (e) return e;
    } else {
        void *args[] = {&a};
        CFM_CUDA_TRY(launch_cooperative((const void *)cg_persistent_kernel, dim3(h->blocks),
                                        dim3(CG_TILE), args, 0, h->stream));
        launches += 1;
    }
    if (x_host) {
        CFM_CUDA_TRY(cudaMemcpyAsync(x_host, a.x, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                     h->stream));
    }
    CFM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    CFM_CUDA_TRY(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CFM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    int status;
    if (h->p.impl != CFM_CG_DISCRETE) {
        CFM_CUDA_TRY(cudaMemcpy(&bs, h->bar, sizeof(bs), cudaMemcpyDeviceToHost));
        if (bs.error) {
            set_error("grid barrier %d timed out", bs.where);
            if (st) {
                std::memset(st, 0, sizeof(*st));
                st->status = CFM_BARRIER_TIMEOUT;
            }
            return CFM_BARRIER_TIMEOUT;
        }
        CFM_CUDA_TRY(cudaMemcpy(&r, h->res, sizeof(r), cudaMemcpyDeviceToHost));
    }
    status = r.status;
    double relres = 0;
    int e = true_relres(h, a, r.bnorm, &relres);
    if (e) return e;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->seconds = ms * 1e-3;
        st->iterations = r.iters;
        st->residual = relres;
        const double nnz = (double)h->A->nnz;
        // FP64 standard CG, fused dots: matrix (12 B/nnz + 4(n+1)) + 11 vector
        // passes of 8 B per row per iteration.
        st->bytes = (double)r.iters * (12.0 * nnz + 4.0 * (n + 1) + 88.0 * n);
        st->gbs = st->seconds > 0 ? st->bytes / st->seconds * 1e-9 : 0;
        st->h2d_bytes = h2d;
        st->d2h_bytes = d2h;
        st->launches = launches;
        st->status = status;
        st->refinements = r.restarts;
    }
    if (status == CFM_NOT_CONVERGED)
        set_error("not converged after %lld iterations (true relres %.3e)", r.iters, relres);
    if (status == CFM_BREAKDOWN) set_error("CG breakdown at iteration %lld", r.iters);
    return status;
}

}  // namespace

extern "C" {

int cfm_csr_create(int n, long long nnz, const int *rowptr, const int *col, const double *val,
                   cfm_csr **out) {
    clear_error();
    CFM_ARG_CHECK(out, "out is null");
    *out = nullptr;
    CFM_ARG_CHECK(n > 0 && nnz >= 0 && rowptr && (nnz == 0 || (col && val)), "csr arrays");
    CFM_ARG_CHECK(nnz < 2147483647LL, "nnz must fit in int32");
    const int base = rowptr[0];
    CFM_ARG_CHECK(base == 0 || base == 1, "rowptr[0] must be 0 or 1");
    CFM_ARG_CHECK((long long)rowptr[n] - base == nnz, "rowptr[n] - base must equal nnz");
    std::vector<int> rp(rowptr, rowptr + n + 1), cc;
    for (int i = 0; i < n; ++i)
        CFM_ARG_CHECK(rowptr[i + 1] >= rowptr[i], "rowptr must be non-decreasing");
    if (base) {
        for (auto &v : rp) v -= 1;
    }
    cc.assign(col, col + nnz);
    for (auto &c : cc) {
        c -= base;
        CFM_ARG_CHECK(c >= 0 && c < n, "column index out of range");
    }
    cfm_csr *A = new cfm_csr();
    A->n = n;
    A->nnz = nnz;
    cudaError_t e;
    if ((e = cudaMalloc(&A->rowptr, sizeof(int) * (n + 1))) != cudaSuccess ||
        (e = cudaMalloc(&A->col, sizeof(int) * std::max(1LL, nnz))) != cudaSuccess ||
        (e = cudaMalloc(&A->val, sizeof(double) * std::max(1LL, nnz))) != cudaSuccess ||
        (e = cudaMemcpy(A->rowptr, rp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (nnz && (e = cudaMemcpy(A->col, cc.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice)) !=
                    cudaSuccess) ||
        (nnz && (e = cudaMemcpy(A->val, val, sizeof(double) * nnz, cudaMemcpyHostToDevice)) !=
                    cudaSuccess)) {
        set_error("csr upload failed: %s", cudaGetErrorString(e));
        cfm_csr_destroy(A);
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    *out = A;
    return CFM_OK;
}

void cfm_csr_destroy(cfm_csr *A) {
    if (!A) return;
    cudaFree(A->rowptr);
    cudaFree(A->col);
    cudaFree(A->val);
    delete A;
}

int cfm_csr_spmv_host(const cfm_csr *A, const double *x, double *y) {
    CFM_ARG_CHECK(A && x && y, "null argument");
    clear_error();
    const size_t bytes = sizeof(double) * A->n;
    double *d = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&d, 2 * bytes));
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_spmv<<<(A->n + 255) / 256, 256>>>(A->n, A->rowptr, A->col, A->val, d, d + A->n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + A->n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    CFM_CUDA_TRY(e);
    return CFM_OK;
}

int cfm_cg_create(const cfm_csr *A, const cfm_cg_params *p, cfm_cg **out) {
    clear_error();
    CFM_ARG_CHECK(A && p && out, "null argument");
    *out = nullptr;
    CFM_ARG_CHECK(p->impl == CFM_CG_DISCRETE || p->impl == CFM_CG_PERSISTENT,
                  "impl (pipelined and mixed are not built yet)");
    CFM_ARG_CHECK(p->maxiter >= 0, "maxiter");
    cfm_cg *h = new cfm_cg();
    h->p = *p;
    h->A = A;
    const int n = A->n;
    h->ntiles = (n + CG_TILE - 1) / CG_TILE;
    auto fail = [&](int s) {
        cfm_cg_destroy(h);
        return s;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&h->vec, sizeof(double) * 6 * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc(&h->part, sizeof(double) * 4 * (size_t)h->ntiles)) != cudaSuccess ||
        (e = cudaMalloc(&h->scal, sizeof(double) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&h->res, sizeof(CgResult))) != cudaSuccess ||
        (e = cudaMalloc(&h->bar, sizeof(BarrierState))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev1)) != cudaSuccess) {
        set_error("cg handle setup failed: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR);
    }
    h->own_stream = true;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return fail(st);
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_persistent_kernel, CG_TILE, 0);
    if (e != cudaSuccess || per_sm < 1) {
        set_error("cg kernel cannot be resident");
        return fail(CFM_UNSUPPORTED);
    }
    h->blocks = std::min(per_sm * di.num_sms, h->ntiles);
    *out = h;
    return CFM_OK;
}

void cfm_cg_destroy(cfm_cg *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->vec);
    cudaFree(h->part);
    cudaFree(h->scal);
    cudaFree(h->res);
    cudaFree(h->bar);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int cfm_cg_set_stream(cfm_cg *h, void *cuda_stream) {
    CFM_ARG_CHECK(h, "handle is null");
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (!cuda_stream) {
        if (!h->own_stream) {
            CFM_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
            h->own_stream = true;
        }
        return CFM_OK;
    }
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)cuda_stream;
    return CFM_OK;
}

int cfm_cg_solve(cfm_cg *h, const double *b_host, double *x_host, cfm_stats *st) {
    CFM_ARG_CHECK(h && x_host, "null argument");
    clear_error();
    const int n = h->A->n;
    double *b_dev = b_host ? h->vec + 5 * (size_t)n : nullptr;
    return solve_impl(h, b_dev, nullptr, st, b_host ? 8.0 * n : 0.0, 8.0 * n, b_host, x_host);
}

int cfm_cg_solve_device(cfm_cg *h, const double *b_dev, double *x_dev, cfm_stats *st) {
    CFM_ARG_CHECK(h && x_dev, "null argument");
    clear_error();
    return solve_impl(h, b_dev, x_dev, st, 0, 0, nullptr, nullptr);
}

}  // extern "C"

// ------------------------------------------- CG without device allocation
// cfm_cg_solve_noalloc runs cg_persistent_kernel with its scratch carved out
// of one fixed device array instead of cudaMalloc'd buffers, for callers
// that cannot allocate device memory (an outside allocator owns the pool,
// the memory is reserved up front, or an allocation would synchronise).
// Layout, in doubles (256-byte aligned pieces):
//   [0, 32)            header: BarrierState at byte 0, CgResult at byte 64,
//                      4 reduced scalars at byte 128
//   [32, 32 + 4T)      dot partials, T = CFM_CG_NOALLOC_MAX_N / 1024 tiles
//   then 4 N           the vectors r, p, s, t (N = CFM_CG_NOALLOC_MAX_N)
namespace cfm {

constexpr size_t NA_MAX_N = CFM_CG_NOALLOC_MAX_N;
constexpr size_t NA_MAX_TILES = NA_MAX_N / CG_TILE;
constexpr size_t NA_HDR = 32;
constexpr size_t NA_PART = NA_HDR;
constexpr size_t NA_VEC = NA_PART + 4 * NA_MAX_TILES;
constexpr size_t NA_TOTAL = NA_VEC + 4 * NA_MAX_N;
static_assert(NA_MAX_N % CG_TILE == 0, "whole tiles");
static_assert(sizeof(BarrierState) <= 64 && sizeof(CgResult) <= 64, "header layout");

// Held by every GPU that loads the library, until the process exits.
static __device__ __align__(256) double g_cg_noalloc_scratch[NA_TOTAL];

// Zeroes the barrier (the only scratch read before it is written) and sets
// its wait budget.
__global__ void k_noalloc_reset(BarrierState *b, unsigned long long timeout_ns) {
    b->count = 0;
    b->gen = 0;
    b->error = 0;
    b->where = 0;
    b->timeout_ns = timeout_ns;
}

namespace {

// Device address of g_cg_noalloc_scratch on the current device.  In host
// code the symbol names a host-side stand-in, so the address is looked up
// once per device with that device current and cached.
int noalloc_scratch(double **out) {
    static std::mutex mu;
    static double *addr[64] = {};
    int dev = 0;
    CFM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("device index %d out of range", dev);
        return CFM_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cg_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(g_cg_noalloc_scratch) failed: %s",
                      cudaGetErrorString(e));
            return CFM_CUDA_ERROR;
        }
        addr[dev] = static_cast<double *>(p);
    }
    *out = addr[dev];
    return CFM_OK;
}

}  // namespace
}  // namespace cfm

extern "C" int cfm_cg_solve_noalloc(int n, long long nnz, const int *rowptr_dev,
                                    const int *col_dev, const double *val_dev,
                                    const double *b_dev, double *x_dev, int maxiter, double tol,
                                    void *cuda_stream, cfm_stats *st) {
    clear_error();
    CFM_ARG_CHECK(n > 0, "n must be positive");
    if ((size_t)n > NA_MAX_N) {
        set_error("bad argument: n = %d exceeds CFM_CG_NOALLOC_MAX_N = %d (the fixed scratch "
                  "array of cfm_cg_solve_noalloc)", n, (int)NA_MAX_N);
        return CFM_BAD_ARG;
    }
    CFM_ARG_CHECK(nnz >= 0 && nnz < 2147483647LL, "nnz");
    CFM_ARG_CHECK(rowptr_dev && x_dev && (nnz == 0 || (col_dev && val_dev)), "null argument");
    CFM_ARG_CHECK(maxiter >= 0, "maxiter");
    double *scr = nullptr;
    int e = noalloc_scratch(&scr);
    if (e) return e;
    DeviceInfo di;
    if ((e = current_device_info(&di))) return e;
    int per_sm = 0;
    CFM_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_persistent_kernel, CG_TILE, 0));
    if (per_sm < 1) {
        set_error("cg kernel cannot be resident");
        return CFM_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    CgArgs a{};
    a.n = n;
    a.ntiles = (n + CG_TILE - 1) / CG_TILE;
    a.rowptr = rowptr_dev;
    a.col = col_dev;
    a.val = val_dev;
    a.b = b_dev;
    a.x = x_dev;
    a.r = scr + NA_VEC;
    a.p = a.r + n;
    a.s = a.p + n;
    a.t = a.s + n;
    a.part = scr + NA_PART;
    a.bar = reinterpret_cast<BarrierState *>(scr);
    a.res = reinterpret_cast<CgResult *>(reinterpret_cast<char *>(scr) + 64);
    double *scal = scr + 16;
    a.maxiter = maxiter;
    a.tol = tol;
    const int blocks = std::min(per_sm * di.num_sms, a.ntiles);
    const auto t0 = std::chrono::steady_clock::now();
    k_noalloc_reset<<<1, 1, 0, s>>>(a.bar, barrier_timeout_ns());
    CFM_CUDA_TRY(cudaGetLastError());
    void *args[] = {&a};
    CFM_CUDA_TRY(launch_cooperative((const void *)cg_persistent_kernel, dim3(blocks),
                                    dim3(CG_TILE), args, 0, s));
    // final FP64 true residual b - A x into partial slot 2, reduced to scal[2]
    k_true_residual<<<a.ntiles, CG_TILE, 0, s>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    k_reduce<<<1, CG_TILE, 0, s>>>(a, 2, scal);
    CFM_CUDA_TRY(cudaGetLastError());
    double hdr[NA_HDR];
    CFM_CUDA_TRY(cudaMemcpyAsync(hdr, scr, sizeof(hdr), cudaMemcpyDeviceToHost, s));
    CFM_CUDA_TRY(cudaStreamSynchronize(s));
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    BarrierState bs;
    CgResult r;
    std::memcpy(&bs, hdr, sizeof(bs));
    std::memcpy(&r, reinterpret_cast<const char *>(hdr) + 64, sizeof(r));
    if (bs.error) {
        set_error("grid barrier %d timed out", bs.where);
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->status = CFM_BARRIER_TIMEOUT;
        }
        return CFM_BARRIER_TIMEOUT;
    }
    const double tt = hdr[16 + 2];
    const double relres = r.bnorm > 0 ? std::sqrt(tt) / r.bnorm : std::sqrt(tt);
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->seconds = secs;
        st->iterations = r.iters;
        st->residual = relres;
        st->bytes = (double)r.iters * (12.0 * (double)nnz + 4.0 * (n + 1) + 88.0 * n);
        st->gbs = secs > 0 ? st->bytes / secs * 1e-9 : 0;
        st->launches = 4;
        st->status = r.status;
        st->refinements = r.restarts;
    }
    if (r.status == CFM_NOT_CONVERGED)
        set_error("not converged after %lld iterations (true relres %.3e)", r.iters, relres);
    if (r.status == CFM_BREAKDOWN) set_error("CG breakdown at iteration %lld", r.iters);
    return r.status;
}
