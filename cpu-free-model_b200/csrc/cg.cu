// Conjugate gradient on one GPU: the cfm_csr / cfm_stencil operators, the
// cfm_cg handle and its solvers (kernels in krylov.cuh).
//
// Algorithm (standard CG, CG/src/common.cu:399-538 and
// CG/src/single-stream/standard.cu:158-299):
//   r0 = b - A x0, p0 = r0, gamma0 = <r0, r0>
//   s = A p; delta = <p, s>; alpha = gamma0 / delta
//   x += alpha p; r -= alpha s; gamma1 = <r, r>; beta = gamma1 / gamma0
//   p = r + beta p
// The reference sums the dots with atomicAdd(double) in arrival order
// (CG/src/common.cu:357-389); here every dot is a fixed tree, so the result
// does not depend on the launch shape and the host oracle reproduces it.
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

#include "cfm_internal.h"
#include "krylov.cuh"

namespace cfm {
// FP32 copy of n doubles (device).
__global__ void k_to_f32(const double *in, float *out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(in[i]);
}
}  // namespace cfm

using namespace cfm;

struct cfm_csr {
    int n = 0;
    long long nnz = 0;
    int *rowptr = nullptr;
    int *col = nullptr;
    double *val = nullptr;
    float *val32 = nullptr;
};

struct cfm_stencil {
    int dims = 2, nx = 0, ny = 0, nz = 1, n = 0;
    double *c64 = nullptr;  // we | wn | wt | dg  (4 n)
    float *c32 = nullptr;   // FP32 copies        (4 n)
};

struct cfm_cg {
    cfm_cg_params p{};
    int kind = 0;  // 0 CSR, 2 / 3 stencil of that dimension
    const cfm_csr *A = nullptr;
    const cfm_stencil *S = nullptr;
    int n = 0;
    int ntiles = 0;
    double *vec = nullptr;  // x r p s t b z w0 w1 (9 n)
    float *vec32 = nullptr; // r32 p32 s32 d32 (4 n)
    double *part = nullptr;
    double *scal = nullptr;  // NSLOTS reduced scalars (discrete variant, final residual)
    CgResult *res = nullptr;
    BarrierState *bar = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int blocks = 0;
};

namespace {

CsrOp csr_op(const cfm_csr *A) { return CsrOp{A->rowptr, A->col, A->val, A->val32}; }

template <int D>
StencilOp<D> stencil_op(const cfm_stencil *S) {
    const size_t n = S->n;
    StencilOp<D> o;
    o.nx = S->nx;
    o.ny = S->ny;
    o.nz = S->nz;
    o.we = S->c64;
    o.wn = S->c64 + n;
    o.wt = S->c64 + 2 * n;
    o.dg = S->c64 + 3 * n;
    o.we32 = S->c32;
    o.wn32 = S->c32 + n;
    o.wt32 = S->c32 + 2 * n;
    o.dg32 = S->c32 + 3 * n;
    return o;
}

template <class Op>
KArgs<Op> make_args(cfm_cg *h, const Op &op, const double *b_dev, double *x_dev) {
    KArgs<Op> a{};
    const size_t n = h->n;
    a.op = op;
    a.n = h->n;
    a.ntiles = h->ntiles;
    a.b = b_dev;
    a.x = x_dev ? x_dev : h->vec;
    a.r = h->vec + n;
    a.p = h->vec + 2 * n;
    a.s = h->vec + 3 * n;
    a.t = h->vec + 4 * n;
    a.z = h->vec + 6 * n;
    a.w0 = h->vec + 7 * n;
    a.w1 = h->vec + 8 * n;
    a.r32 = h->vec32;
    a.p32 = h->vec32 + n;
    a.s32 = h->vec32 + 2 * n;
    a.d32 = h->vec32 + 3 * n;
    a.part = h->part;
    a.res = h->res;
    a.bar = h->bar;
    a.maxiter = h->p.maxiter;
    a.tol = h->p.tol;
    a.inner_maxiter = h->p.inner_maxiter;  // 0: no cap per sweep
    a.inner_tol = h->p.inner_tol > 0 ? h->p.inner_tol : 0.1;
    return a;
}

template <class Op>
int run_discrete(cfm_cg *h, const KArgs<Op> &a, CgResult *out, int *launches) {
    const int g = a.ntiles;
    cudaStream_t st = h->stream;
    double hs[NSLOTS];
    auto fetch = [&](int which) -> int {
        k_reduce<Op><<<1, CG_TILE, 0, st>>>(a, which, h->scal);
        CFM_CUDA_TRY(cudaGetLastError());
        CFM_CUDA_TRY(cudaMemcpyAsync(&hs[which], h->scal + which, sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        CFM_CUDA_TRY(cudaStreamSynchronize(st));
        *launches += 1;
        return CFM_OK;
    };
    int e;
    k_init<Op><<<g, CG_TILE, 0, st>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    *launches += 1;
    if ((e = fetch(SL_G0)) || (e = fetch(SL_B))) return e;
    double gamma0 = hs[SL_G0];
    const double bnorm = std::sqrt(hs[SL_B]);
    const bool use_tol = a.tol > 0.0;
    const double target = a.tol * bnorm;
    int status = use_tol ? CFM_NOT_CONVERGED : CFM_OK;
    int restarts = 0;
    long long k = 0;
    if (use_tol && std::sqrt(gamma0) <= target) status = CFM_OK;
    while (k < a.maxiter && !(use_tol && status == CFM_OK)) {
        k_spmv_dot<Op><<<g, CG_TILE, 0, st>>>(a);
        *launches += 1;
        if ((e = fetch(SL_D0))) return e;
        const double delta = hs[SL_D0];
        const double alpha = gamma0 / delta;
        if (use_tol && !(delta > 0.0 && std::isfinite(alpha))) {
            status = CFM_BREAKDOWN;
            break;
        }
        k_update<Op><<<g, CG_TILE, 0, st>>>(a, alpha);
        *launches += 1;
        if ((e = fetch(SL_G0))) return e;
        const double gamma1 = hs[SL_G0];
        ++k;
        if (use_tol && std::sqrt(gamma1) <= target) {
            k_true_residual<Op><<<g, CG_TILE, 0, st>>>(a);
            *launches += 1;
            if ((e = fetch(SL_TT))) return e;
            if (std::sqrt(hs[SL_TT]) <= target) {
                status = CFM_OK;
                gamma0 = gamma1;
                break;
            }
            k_restart<Op><<<g, CG_TILE, 0, st>>>(a);
            *launches += 1;
            ++restarts;
            gamma0 = hs[SL_TT];
            continue;
        }
        const double beta = gamma1 / gamma0;
        if (use_tol && !std::isfinite(beta)) {
            status = CFM_BREAKDOWN;
            break;
        }
        k_p<Op><<<g, CG_TILE, 0, st>>>(a, beta);
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
template <class Op>
int true_relres(cfm_cg *h, const KArgs<Op> &a, double bnorm, double *out) {
    k_true_residual<Op><<<a.ntiles, CG_TILE, 0, h->stream>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    k_reduce<Op><<<1, CG_TILE, 0, h->stream>>>(a, SL_TT, h->scal);
    CFM_CUDA_TRY(cudaGetLastError());
    double tt = 0;
    CFM_CUDA_TRY(cudaMemcpyAsync(&tt, h->scal + SL_TT, sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    *out = bnorm > 0 ? std::sqrt(tt) / bnorm : std::sqrt(tt);
    return CFM_OK;
}

template <class Op>
const void *solver_fn(int impl) {
    switch (impl) {
        case CFM_CG_PERSISTENT_PIPELINED: return (const void *)cg_pipe_kernel<Op>;
        case CFM_CG_MIXED: return (const void *)cg_mixed_kernel<Op>;
        default: return (const void *)cg_std_kernel<Op>;
    }
}

// Algorithmic HBM bytes of one iteration: operator data plus the vector
// passes of the method (8 B per FP64 entry read or written, 4 per FP32).
double bytes_per_iter(const cfm_cg *h) {
    const double n = h->n;
    double op64, op32;
    if (h->kind == 0) {
        const double nnz = (double)h->A->nnz;
        op64 = 12.0 * nnz + 4.0 * (n + 1);
        op32 = 8.0 * nnz + 4.0 * (n + 1);
    } else {
        op64 = 8.0 * h->kind * n;  // dims face arrays + diagonal
        op32 = 4.0 * h->kind * n;
    }
    switch (h->p.impl) {
        case CFM_CG_PERSISTENT_PIPELINED: return op64 + 96.0 * n;
        case CFM_CG_MIXED: return op32 + 44.0 * n;
        default: return op64 + 88.0 * n;
    }
}

template <class Op>
int solve_t(cfm_cg *h, const Op &op, const double *b_dev, double *x_dev, cfm_stats *st,
            double h2d, double d2h, const double *b_host, double *x_host) {
    const int n = h->n;
    KArgs<Op> a = make_args(h, op, b_dev, x_dev);
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
        CFM_CUDA_TRY(launch_cooperative(solver_fn<Op>(h->p.impl), dim3(h->blocks), dim3(CG_TILE),
                                        args, 0, h->stream));
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
    const int status = r.status;
    double relres = 0;
    int e = true_relres(h, a, r.bnorm, &relres);
    if (e) return e;
    if (st) {
        std::memset(st, 0, sizeof(*st));
        st->seconds = ms * 1e-3;
        st->iterations = r.iters;
        st->residual = relres;
        st->bytes = (double)r.iters * bytes_per_iter(h);
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

int solve_impl(cfm_cg *h, const double *b_dev, double *x_dev, cfm_stats *st, double h2d,
               double d2h, const double *b_host, double *x_host) {
    switch (h->kind) {
        case 2: return solve_t(h, stencil_op<2>(h->S), b_dev, x_dev, st, h2d, d2h, b_host, x_host);
        case 3: return solve_t(h, stencil_op<3>(h->S), b_dev, x_dev, st, h2d, d2h, b_host, x_host);
        default: return solve_t(h, csr_op(h->A), b_dev, x_dev, st, h2d, d2h, b_host, x_host);
    }
}

template <class Op>
int occupancy(int impl, int *per_sm) {
    CFM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, solver_fn<Op>(impl),
                                                               CG_TILE, 0));
    return CFM_OK;
}

int create_common(cfm_cg *h, const cfm_cg_params *p) {
    h->p = *p;
    const size_t n = h->n;
    h->ntiles = (int)((n + CG_TILE - 1) / CG_TILE);
    cudaError_t e;
    if ((e = cudaMalloc(&h->vec, sizeof(double) * 9 * n)) != cudaSuccess ||
        (e = cudaMalloc(&h->vec32, sizeof(float) * 4 * n)) != cudaSuccess ||
        (e = cudaMalloc(&h->part, sizeof(double) * NSLOTS * (size_t)h->ntiles)) != cudaSuccess ||
        (e = cudaMalloc(&h->scal, sizeof(double) * NSLOTS)) != cudaSuccess ||
        (e = cudaMalloc(&h->res, sizeof(CgResult))) != cudaSuccess ||
        (e = cudaMalloc(&h->bar, sizeof(BarrierState))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev1)) != cudaSuccess) {
        set_error("cg handle setup failed: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    h->own_stream = true;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    int per_sm = 0;
    switch (h->kind) {
        case 2: st = occupancy<StencilOp<2>>(p->impl, &per_sm); break;
        case 3: st = occupancy<StencilOp<3>>(p->impl, &per_sm); break;
        default: st = occupancy<CsrOp>(p->impl, &per_sm); break;
    }
    if (st) return st;
    if (per_sm < 1) {
        set_error("cg kernel cannot be resident");
        return CFM_UNSUPPORTED;
    }
    h->blocks = std::min(per_sm * di.num_sms, h->ntiles);
    return CFM_OK;
}

int check_cg_params(const cfm_cg_params *p) {
    CFM_ARG_CHECK(p->impl >= CFM_CG_DISCRETE && p->impl <= CFM_CG_MIXED, "impl");
    CFM_ARG_CHECK(p->maxiter >= 0, "maxiter");
    CFM_ARG_CHECK(p->impl != CFM_CG_MIXED || p->tol > 0, "mixed precision needs tol > 0");
    CFM_ARG_CHECK(p->inner_maxiter >= 0 && p->inner_tol >= 0 && p->inner_tol < 1,
                  "inner_maxiter, inner_tol");
    return CFM_OK;
}

}  // namespace

namespace cfm {

// Standard persistent CG on a stencil operator with iterate snapshots (the
// training data of the learned preconditioner): solves A x = b (device
// vectors, x0 = 0) to tol, storing x after every `every`-th iteration into
// snap (up to `max_snaps` n-vectors).  Returns the status; *iters and
// *taken (snapshots written) optional.
int cg_stencil_snapshots(const cfm_stencil *S, const double *b_dev, double *x_dev, double tol,
                         int maxiter, double *snap, int every, int max_snaps, long long *iters,
                         int *taken, cudaStream_t stream) {
    CFM_ARG_CHECK(S && b_dev && x_dev && every > 0 && max_snaps >= 0, "snapshot solve arguments");
    cfm_cg_params p{};
    p.impl = CFM_CG_PERSISTENT;
    p.maxiter = maxiter;
    p.tol = tol;
    cfm_cg *h = nullptr;
    int st = cfm_cg_create_stencil(S, &p, &h);
    if (st) return st;
    if (stream) cfm_cg_set_stream(h, stream);
    auto run = [&](auto op) -> int {
        KArgs<decltype(op)> a = make_args(h, op, b_dev, x_dev);
        a.snap = snap;
        a.snap_every = every;
        a.snap_max = max_snaps;
        BarrierState bs{};
        bs.timeout_ns = barrier_timeout_ns();
        CFM_CUDA_TRY(cudaMemcpyAsync(h->bar, &bs, sizeof(bs), cudaMemcpyHostToDevice, h->stream));
        void *args[] = {&a};
        CFM_CUDA_TRY(launch_cooperative((const void *)cg_std_kernel<decltype(op)>, dim3(h->blocks),
                                        dim3(CG_TILE), args, 0, h->stream));
        CgResult r{};
        CFM_CUDA_TRY(cudaMemcpyAsync(&bs, h->bar, sizeof(bs), cudaMemcpyDeviceToHost, h->stream));
        CFM_CUDA_TRY(cudaMemcpyAsync(&r, h->res, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
        CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
        if (bs.error) {
            set_error("grid barrier %d timed out", bs.where);
            return CFM_BARRIER_TIMEOUT;
        }
        if (iters) *iters = r.iters;
        if (taken) *taken = (int)std::min<long long>(r.iters / every, max_snaps);
        return r.status;
    };
    st = S->dims == 2 ? run(stencil_op<2>(S)) : run(stencil_op<3>(S));
    cfm_cg_destroy(h);
    return st;
}

// Device coefficient arrays of a stencil (we | wn | wt | dg, 4 n doubles,
// and their FP32 copies).
const double *stencil_coeffs(const cfm_stencil *S) { return S->c64; }
const float *stencil_coeffs32(const cfm_stencil *S) { return S->c32; }
void stencil_shape(const cfm_stencil *S, int *dims, int *nx, int *ny, int *nz) {
    *dims = S->dims;
    *nx = S->nx;
    *ny = S->ny;
    *nz = S->nz;
}

}  // namespace cfm

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
    const size_t nz1 = (size_t)std::max(1LL, nnz);
    cudaError_t e;
    if ((e = cudaMalloc(&A->rowptr, sizeof(int) * (n + 1))) != cudaSuccess ||
        (e = cudaMalloc(&A->col, sizeof(int) * nz1)) != cudaSuccess ||
        (e = cudaMalloc(&A->val, sizeof(double) * nz1)) != cudaSuccess ||
        (e = cudaMalloc(&A->val32, sizeof(float) * nz1)) != cudaSuccess ||
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
    if (nnz) {
        k_to_f32<<<1024, 256>>>(A->val, A->val32, (size_t)nnz);
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
            set_error("csr fp32 copy failed: %s", cudaGetErrorString(e));
            cfm_csr_destroy(A);
            return CFM_CUDA_ERROR;
        }
    }
    *out = A;
    return CFM_OK;
}

void cfm_csr_destroy(cfm_csr *A) {
    if (!A) return;
    cudaFree(A->rowptr);
    cudaFree(A->col);
    cudaFree(A->val);
    cudaFree(A->val32);
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
        k_apply<CsrOp><<<(A->n + 255) / 256, 256>>>(csr_op(A), A->n, d, d + A->n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + A->n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    CFM_CUDA_TRY(e);
    return CFM_OK;
}

int cfm_stencil_create(int dims, int nx, int ny, int nz, const double *k_host,
                       cfm_stencil **out) {
    clear_error();
    CFM_ARG_CHECK(out && k_host, "null argument");
    *out = nullptr;
    CFM_ARG_CHECK(dims == 2 || dims == 3, "dims must be 2 or 3");
    if (dims == 2) nz = 1;
    CFM_ARG_CHECK(nx >= 1 && ny >= 1 && nz >= 1, "sizes");
    const double cells = (double)nx * ny * nz;
    CFM_ARG_CHECK(cells < 2.0e9, "grid too large for int32 rows");
    const size_t n = (size_t)nx * ny * nz;
    for (size_t i = 0; i < n; ++i)
        CFM_ARG_CHECK(k_host[i] > 0 && std::isfinite(k_host[i]), "k must be positive and finite");
    std::vector<double> c(4 * n, 0.0);
    int st = cfm_varcoef_coeffs(dims, nx, ny, nz, k_host, c.data(), c.data() + n,
                                c.data() + 2 * n, c.data() + 3 * n);
    if (st) return st;
    cfm_stencil *S = new cfm_stencil();
    S->dims = dims;
    S->nx = nx;
    S->ny = ny;
    S->nz = nz;
    S->n = (int)n;
    cudaError_t e;
    if ((e = cudaMalloc(&S->c64, sizeof(double) * 4 * n)) != cudaSuccess ||
        (e = cudaMalloc(&S->c32, sizeof(float) * 4 * n)) != cudaSuccess ||
        (e = cudaMemcpy(S->c64, c.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        set_error("stencil upload failed: %s", cudaGetErrorString(e));
        cfm_stencil_destroy(S);
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    k_to_f32<<<1024, 256>>>(S->c64, S->c32, 4 * n);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
        set_error("stencil fp32 copy failed: %s", cudaGetErrorString(e));
        cfm_stencil_destroy(S);
        return CFM_CUDA_ERROR;
    }
    *out = S;
    return CFM_OK;
}

void cfm_stencil_destroy(cfm_stencil *S) {
    if (!S) return;
    cudaFree(S->c64);
    cudaFree(S->c32);
    delete S;
}

int cfm_stencil_apply_host(const cfm_stencil *S, const double *x, double *y) {
    CFM_ARG_CHECK(S && x && y, "null argument");
    clear_error();
    const size_t bytes = sizeof(double) * S->n;
    double *d = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&d, 2 * bytes));
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int g = (S->n + 255) / 256;
        if (S->dims == 2)
            k_apply<StencilOp<2>><<<g, 256>>>(stencil_op<2>(S), S->n, d, d + S->n);
        else
            k_apply<StencilOp<3>><<<g, 256>>>(stencil_op<3>(S), S->n, d, d + S->n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + S->n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    CFM_CUDA_TRY(e);
    return CFM_OK;
}

int cfm_cg_create(const cfm_csr *A, const cfm_cg_params *p, cfm_cg **out) {
    clear_error();
    CFM_ARG_CHECK(A && p && out, "null argument");
    *out = nullptr;
    int st = check_cg_params(p);
    if (st) return st;
    cfm_cg *h = new cfm_cg();
    h->kind = 0;
    h->A = A;
    h->n = A->n;
    if ((st = create_common(h, p))) {
        cfm_cg_destroy(h);
        return st;
    }
    *out = h;
    return CFM_OK;
}

int cfm_cg_create_stencil(const cfm_stencil *S, const cfm_cg_params *p, cfm_cg **out) {
    clear_error();
    CFM_ARG_CHECK(S && p && out, "null argument");
    *out = nullptr;
    int st = check_cg_params(p);
    if (st) return st;
    cfm_cg *h = new cfm_cg();
    h->kind = S->dims;
    h->S = S;
    h->n = S->n;
    if ((st = create_common(h, p))) {
        cfm_cg_destroy(h);
        return st;
    }
    *out = h;
    return CFM_OK;
}

void cfm_cg_destroy(cfm_cg *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->vec);
    cudaFree(h->vec32);
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
    const cfm::NvtxRange nvtx_range("cfm_cg_solve");
    CFM_ARG_CHECK(h && x_host, "null argument");
    clear_error();
    const int n = h->n;
    double *b_dev = b_host ? h->vec + 5 * (size_t)n : nullptr;
    return solve_impl(h, b_dev, nullptr, st, b_host ? 8.0 * n : 0.0, 8.0 * n, b_host, x_host);
}

int cfm_cg_solve_device(cfm_cg *h, const double *b_dev, double *x_dev, cfm_stats *st) {
    const cfm::NvtxRange nvtx_range("cfm_cg_solve_device");
    CFM_ARG_CHECK(h && x_dev, "null argument");
    clear_error();
    return solve_impl(h, b_dev, x_dev, st, 0, 0, nullptr, nullptr);
}

}  // extern "C"

// ------------------------------------------- CG without device allocation
// cfm_cg_solve_noalloc runs cg_std_kernel<CsrOp> with its scratch carved out
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
// once per device with that device current and cached.  With lazy module
// loading (the CUDA default) that first lookup is also what loads this
// file's kernels and the array onto the device, so it can allocate device
// memory: an allocation failure there is CFM_OUT_OF_MEMORY.  The cache
// assumes the device's primary context lives as long as the process; after
// a cudaDeviceReset the array may sit at another address.
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
            return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
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
    const NvtxRange nvtx_range("cfm_cg_solve_noalloc");
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
    // The kernel zeroes x first and reads b again for the true residual.
    CFM_ARG_CHECK(b_dev == nullptr || (const void *)b_dev != (const void *)x_dev,
                  "b and x must not be the same array");
    double *scr = nullptr;
    int e = noalloc_scratch(&scr);
    if (e) return e;
    DeviceInfo di;
    if ((e = current_device_info(&di))) return e;
    int per_sm = 0;
    CFM_CUDA_TRY(
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_std_kernel<CsrOp>, CG_TILE, 0));
    if (per_sm < 1) {
        set_error("cg kernel cannot be resident");
        return CFM_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    KArgs<CsrOp> a{};
    a.n = n;
    a.ntiles = (n + CG_TILE - 1) / CG_TILE;
    a.op.rowptr = rowptr_dev;
    a.op.col = col_dev;
    a.op.val = val_dev;
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
    CFM_CUDA_TRY(launch_cooperative((const void *)cg_std_kernel<CsrOp>, dim3(blocks),
                                    dim3(CG_TILE), args, 0, s));
    // final FP64 true residual b - A x into partial slot 2, reduced to scal[2]
    k_true_residual<CsrOp><<<a.ntiles, CG_TILE, 0, s>>>(a);
    CFM_CUDA_TRY(cudaGetLastError());
    k_reduce<CsrOp><<<1, CG_TILE, 0, s>>>(a, SL_TT, scal);
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
    const double tt = hdr[16 + SL_TT];
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
