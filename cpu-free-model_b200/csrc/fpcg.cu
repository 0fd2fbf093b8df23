// Learned preconditioning on one GPU (no reference counterpart):
//  - training pairs from plain CG: for fresh seeds, the 2D variable-
//    coefficient problem is solved by the persistent FP64 CG kernel to
//    1e-10 (x*), then again with iterate snapshots x_j; each pair is the
//    residual r_j = b - A x_j (input, with log k) and the error
//    e_j = x* - x_j (target), both scaled to unit RMS;
//  - training of the U-Net (learned.cu) with Adam on the per-sample
//    energy-norm loss 1 - <z, r>^2 / (<z, A z> <e, r>), z = net(r): one minus
//    the fraction of the A-norm error ||e||_A^2 a CG step along z removes.
//    It is blind to the output's scale (which flexible CG ignores) and,
//    unlike an L2 loss, punishes output noise that A amplifies;
//  - flexible PCG (Notay 2000; Polak-Ribiere beta, clipped at 0) with the
//    hybrid preconditioner z = J(z0 + c y): z0 = J(0) damped Jacobi sweeps,
//    y = net(r1) on the smoothed residual r1 = r - A z0, c the optimal step
//    <y, r1> / <y, A y>; FP64 vectors and dots, the network in BF16 on the
//    tensor cores.  One iteration is a fixed
//    kernel sequence; it is captured once into a CUDA graph whose
//    conditional WHILE node repeats it on the device until the residual
//    reaches the tolerance, so the host launches the whole solve once.
//    If the loop stalls or hits its cap, plain FP64 persistent CG finishes
//    from the current iterate (the fallback) and checks the result by the
//    FP64 true residual.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <type_traits>
#include <vector>

#include "cfm_internal.h"
#include "krylov.cuh"
#include "learned_internal.h"

namespace cfm {
int cg_stencil_snapshots(const cfm_stencil *S, const double *b_dev, double *x_dev, double tol,
                         int maxiter, double *snap, int every, int max_snaps, long long *iters,
                         int *taken, cudaStream_t stream);
const double *stencil_coeffs(const cfm_stencil *S);
const float *stencil_coeffs32(const cfm_stencil *S);
void stencil_shape(const cfm_stencil *S, int *dims, int *nx, int *ny, int *nz);
}  // namespace cfm

namespace cfm {

namespace {

// n-vectors in cfm_fpcg::vec: x r rold p s z b t d za zb r1.
constexpr int FP_NVEC = 8;  // x r z b t d za r1

// Damping of the Jacobi smoothing sweeps around the network.
constexpr double JACOBI_OMEGA = 0.8;

StencilOp<2> op2(const cfm_stencil *S) {
    int dims, nx, ny, nz;
    stencil_shape(S, &dims, &nx, &ny, &nz);
    const double *c = stencil_coeffs(S);
    const size_t n = (size_t)nx * ny;
    StencilOp<2> o{};
    o.nx = nx;
    o.ny = ny;
    o.nz = 1;
    o.we = c;
    o.wn = c + n;
    o.wt = c + 2 * n;
    o.dg = c + 3 * n;
    return o;
}

// Cross-block sums of K doubles that come out the same on every run.  The
// participating block `idx` of `n` stores its K values (v, read on thread 0)
// at slots[idx * K + j]; the last participant to arrive (counted on *count)
// adds the slots in participant order -- lane l of its first warp takes
// participants l, l + 32, ..., then a fixed xor butterfly -- writes out[j]
// (adds to it when `add`) and re-arms *count for the next launch.  Every
// thread of a participating block calls it.
template <int K>
__device__ void ordered_grid_sum(const double *v, double *slots, int idx, int n, unsigned int *count,
                                 double *out, bool add) {
    __shared__ int s_last;
    if (threadIdx.x == 0) {
        for (int j = 0; j < K; ++j) slots[(size_t)idx * K + j] = v[j];
        __threadfence();
        s_last = atomicAdd(count, 1u) == (unsigned int)(n - 1);
    }
    __syncthreads();
    if (s_last && threadIdx.x < 32) {
        __threadfence();
        double t[K];
        for (int j = 0; j < K; ++j) t[j] = 0.0;
        for (int i = threadIdx.x; i < n; i += 32)
            for (int j = 0; j < K; ++j) t[j] += __ldcg(slots + (size_t)i * K + j);
        for (int o = 16; o; o >>= 1)
            for (int j = 0; j < K; ++j) t[j] += __shfl_xor_sync(CG_FULL, t[j], o);
        if (threadIdx.x == 0) {
            for (int j = 0; j < K; ++j) out[j] = add ? out[j] + t[j] : t[j];
            *count = 0;
        }
    }
}

// ------------------------------------------------------- training data
// r = b - A xj, e = xs - xj; |r|^2, <e, r> into acc[0], acc[1] (grid sums in
// block order: slots of 2 x gridDim.x doubles, one counter).
__global__ void k_pair(StencilOp<2> op, int n, const double *b, const double *xs, const double *xj,
                       double *r, double *e, double *acc, double *slots, unsigned int *count) {
    __shared__ double red[2][32];
    double rr = 0, er = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = b[i] - (xj ? op.apply(xj, i) : 0.0);
        const double ei = xs[i] - (xj ? xj[i] : 0.0);
        r[i] = ri;
        e[i] = ei;
        rr += ri * ri;
        er += ei * ri;
    }
    for (int o = 16; o; o >>= 1) {
        rr += __shfl_xor_sync(CG_FULL, rr, o);
        er += __shfl_xor_sync(CG_FULL, er, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = rr;
        red[1][threadIdx.x >> 5] = er;
    }
    __syncthreads();
    double v[2] = {0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)blockDim.x / 32; ++w) {
            v[0] += red[0][w];
            v[1] += red[1][w];
        }
    ordered_grid_sum<2>(v, slots, blockIdx.x, gridDim.x, count, acc, false);
}

// Damped Jacobi sweep for the training pairs: zout = zin + omega (r - A zin) / diag.
__global__ void k_data_jacobi(StencilOp<2> op, int n, const double *r, const double *zin,
                              double *zout) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double res = zin ? r[i] - op.apply(zin, i) : r[i];
        zout[i] = __fma_rn(JACOBI_OMEGA / op.dg[i], res, zin ? zin[i] : 0.0);  // as the solver's sweeps
    }
}

// After pre-smoothing z: r <- r - A z, e <- e - z (the pair the network sees
// inside the preconditioner); |r|^2, <e, r> into acc (as k_pair).
__global__ void k_data_smoothed(StencilOp<2> op, int n, const double *z, double *r, double *e,
                                double *r1, double *acc, double *slots, unsigned int *count) {
    __shared__ double red[2][32];
    double rr = 0, er = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = r[i] - op.apply(z, i);
        const double ei = e[i] - z[i];
        r1[i] = ri;
        e[i] = ei;
        rr += ri * ri;
        er += ei * ri;
    }
    for (int o = 16; o; o >>= 1) {
        rr += __shfl_xor_sync(CG_FULL, rr, o);
        er += __shfl_xor_sync(CG_FULL, er, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = rr;
        red[1][threadIdx.x >> 5] = er;
    }
    __syncthreads();
    double v[2] = {0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)blockDim.x / 32; ++w) {
            v[0] += red[0][w];
            v[1] += red[1][w];
        }
    ordered_grid_sum<2>(v, slots, blockIdx.x, gridDim.x, count, acc, false);
}

// One training sample at residual scale sr = 1 / rms(r) (r on the nx x ny
// grid): the fine residual r1 = r sr (FP32, for the loss), the network
// input on the (nx / f) x (ny / f) grid [R(r) sr, gc] with R the mean over
// f x f blocks and gc the block-mean log k, and <e, r> sr^2.
__global__ void k_pair_store(int nx, int ny, int f, const double *r, const float *gc, const double *acc,
                             float *xin, float *r1, double *er_out) {
    const int n = nx * ny, ncx = nx / f, nc = n / (f * f);
    const double sr = acc[0] > 0 ? sqrt((double)n / acc[0]) : 0.0;
    const double inv = 1.0 / (f * f);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        r1[i] = (float)(r[i] * sr);
    for (int ic = blockIdx.x * blockDim.x + threadIdx.x; ic < nc; ic += gridDim.x * blockDim.x) {
        const int cx = ic % ncx, cy = ic / ncx;
        double sum = 0;
        for (int dy = 0; dy < f; ++dy)
            for (int dx = 0; dx < f; ++dx) sum += r[(size_t)(cy * f + dy) * nx + cx * f + dx] * sr;
        xin[2 * ic] = (float)(sum * inv);
        xin[2 * ic + 1] = gc[ic];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *er_out = acc[1] * sr * sr;
}

// ------------------------------------------------------------- the loss
// The network output y lives on the (nx / f) x (ny / f) grid; the correction
// is its piecewise-constant prolongation z = P y on the nx x ny grid,
// z[i] = y[cell(i)].  Per batch element b (sample ids[b] of system
// ids[b] / per, whose FP32 stencil coefficients we | wn | dg sit at
// coef + sys * 3 n and whose fine residual r is r1 + ids[b] n):
//   Az = A z (FP32 apply), s[0] = <z, r>, s[1] = <z, A z> (FP64, the blocks
//   of batch element b summed in block order: slots 2 x gridDim.x from
//   slots + 2 b gridDim.x, counter count[b]).
__device__ __forceinline__ int coarse_cell(int ix, int iy, int f, int ncx) {
    return (iy / f) * ncx + ix / f;
}

__global__ void k_loss_anorm_dots(const float *y, const float *r1, const float *coef,
                                  const long long *ids, int per, int nx, int ny, int f, float *Az,
                                  double *s, double *slots, unsigned int *count) {
    const int b = blockIdx.y, n = nx * ny, ncx = nx / f, nc = n / (f * f);
    const float *c = coef + (size_t)(ids[b] / per) * 3 * n;
    const float *we = c, *wn = c + n, *dg = c + 2 * n;
    const float *r = r1 + (size_t)ids[b] * n;
    y += (size_t)b * nc;
    Az += (size_t)b * n;
    __shared__ double red[2][32];
    double zr = 0, zaz = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ix = i % nx, iy = i / nx;
        const float zi = y[coarse_cell(ix, iy, f, ncx)];
        float t = dg[i] * zi;
        if (ix > 0) t -= we[i - 1] * y[coarse_cell(ix - 1, iy, f, ncx)];
        if (ix < nx - 1) t -= we[i] * y[coarse_cell(ix + 1, iy, f, ncx)];
        if (iy > 0) t -= wn[i - nx] * y[coarse_cell(ix, iy - 1, f, ncx)];
        if (iy < ny - 1) t -= wn[i] * y[coarse_cell(ix, iy + 1, f, ncx)];
        Az[i] = t;
        zr += (double)zi * r[i];
        zaz += (double)zi * t;
    }
    for (int o = 16; o; o >>= 1) {
        zr += __shfl_xor_sync(CG_FULL, zr, o);
        zaz += __shfl_xor_sync(CG_FULL, zaz, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = zr;
        red[1][threadIdx.x >> 5] = zaz;
    }
    __syncthreads();
    double v[2] = {0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)blockDim.x / 32; ++w) {
            v[0] += red[0][w];
            v[1] += red[1][w];
        }
    ordered_grid_sum<2>(v, slots + (size_t)2 * b * gridDim.x, blockIdx.x, gridDim.x, count + b, s + 2 * b,
                        false);
}

// L_b = 1 - a^2 / (q c), a = <z, r>, q = <z, A z>, c = <e, r>;
// dL_b/dz = (2 a / (q c)) ((a / q) A z - r) and dL_b/dy = P^T dL_b/dz (the
// sum over each f x f block); the batch mean (added to *loss, the batch
// elements in order: slots of gridDim.y doubles, one counter) and its gradient.
__global__ void k_loss_anorm_grad(const float *Az, const float *r1, const double *s,
                                  const double *er, const long long *ids, int nx, int ny, int f, int B,
                                  float *dout, double *loss, double *slots, unsigned int *count) {
    const int b = blockIdx.y, n = nx * ny, ncx = nx / f, nc = n / (f * f);
    const double a = s[2 * b], q = s[2 * b + 1], c = er[ids[b]];
    const bool ok = q > 0 && c > 0;
    const double fb = ok ? 2.0 * a / (q * c) / B : 0.0, aq = ok ? a / q : 0.0;
    const float *r = r1 + (size_t)ids[b] * n;
    const float *az = Az + (size_t)b * n;
    for (int ic = blockIdx.x * blockDim.x + threadIdx.x; ic < nc; ic += gridDim.x * blockDim.x) {
        const int cx = ic % ncx, cy = ic / ncx;
        double g = 0;
        for (int dy = 0; dy < f; ++dy)
            for (int dx = 0; dx < f; ++dx) {
                const size_t j = (size_t)(cy * f + dy) * nx + cx * f + dx;
                g += fb * (aq * az[j] - (double)r[j]);
            }
        dout[(size_t)b * nc + ic] = (float)g;
    }
    if (blockIdx.x == 0) {
        const double v = ok ? (1.0 - a * a / (q * c)) / B : 0.0;
        ordered_grid_sum<1>(&v, slots, b, gridDim.y, count, loss, true);
    }
}

// ------------------------------------------------------------------ FPCG
enum : int {
    FP_PS = 0, FP_RR = 1, FP_PR = 2, FP_BB = 3, FP_R1 = 4, FP_YR = 5, FP_YAY = 6,
    FP_ZS = 7,  // FP_ZS + j: <z_k, s_{k-1-j}>, j < m
};
// Truncated flexible CG (Notay's FCG(m)): each direction is A-orthogonalised
// against the last m; directions p_j and s_j = A p_j live in a ring of m + 1
// slots (slot j mod (m + 1)).
constexpr int FP_MAX_TRUNC = 8;
constexpr int FP_RES_BLOCKS = 256;  // grid of the true-residual pass
constexpr int FP_TT = FP_ZS + FP_MAX_TRUNC;  // |b - A x|^2 of a reliable update (mixed)
constexpr int FP_NSLOT = FP_TT + 1;

struct FpState {
    double ps[FP_MAX_TRUNC + 1];  // <p_j, s_j> by ring slot
    double target;       // tol * |b|
    double best_rr;      // smallest |r|^2 seen
    long long k;         // iterations
    long long best_k;    // iteration of best_rr
    int done;            // 1 converged, 2 stalled / capped
    int pad;
    // mixed precision: largest |r32|^2 since the last reliable update, the
    // parity of the FP64 iterate / FP32 correction buffers, a reliable update
    // waiting for k_fp_pre, and the updates so far
    double gmax;
    int par, pending, updates, pad2;
};

struct FpArgs {
    StencilOp<2> op;
    int n, ntiles;
    const double *b;
    double *x, *r, *z;
    double *za, *r1;       // pre-smoothed z0, r1 = r - A z0
    double *pring, *sring;  // FCG directions p_j and A p_j: ring slots of n
    int m, ring;            // truncation m and ring size m + 1
    float *xin, *out;
    double *part;
    FpState *st;
    double *hist;  // |r| before each preconditioner application (maxiter + 1 entries)
    long long maxiter;
    int stall;
    int f, ncx, nc;  // network grid: (nx / f) x (ny / f) = nc cells, ncx per row
    int fsh;         // log2 f
    int ntiles2, tx2;  // FP_TILE x FP_TILE tiles of the smoothing kernels (tx2 per row)
    const float *we32, *wn32, *dg32, *wd32;  // FP32 operator and omega / dg for the smoothing
    int pstride;       // partial-sum slot stride: max(ntiles, ntiles2)
    int smooth;
    // mixed precision: the Krylov vectors in FP32 (residual r32,
    // preconditioned residual z32, direction rings), the iterate in FP64 as
    // xm + dm (FP64 iterate at the last reliable update + FP32 steps since),
    // both double-buffered by the update parity in FpState
    int mixed;
    double delta2;  // a reliable update when |r32|^2 < delta^2 max |r32|^2 since the last
    float *r32, *z32, *pring32, *sring32;
    double *xm[2];
    float *dm[2];
    // batches (cfm_fpcg_create_batch): member y = blockIdx.y of every launch
    // works on its slice of each per-member array (n cells, the nx x ny
    // frame; direction ring slots sstride = nmem n apart), and only cells
    // inside its extent (mx, my from ext[y]) take the network's correction
    int nmem;
    long long sstride;
    const int2 *ext;
    int mx, my;
};

// Offsets every per-member pointer of `a` to member blockIdx.y (nothing for
// member 0 and for a single system) and sets the member's extent.
__device__ __forceinline__ void fp_member(FpArgs &a) {
    const int y = blockIdx.y;
    if (a.ext) {
        a.mx = a.ext[y].x;
        a.my = a.ext[y].y;
    }
    if (y == 0) return;
    const size_t o = (size_t)y * a.n;
    a.op.we += o;
    a.op.wn += o;
    a.op.dg += o;
    a.op.we32 += o;
    a.op.wn32 += o;
    a.op.dg32 += o;
    a.we32 += o;
    a.wn32 += o;
    a.dg32 += o;
    a.wd32 += o;
    a.b += o;
    a.x += o;
    a.r += o;
    a.z += o;
    a.za += o;
    a.r1 += o;
    a.pring += o;
    a.sring += o;
    a.xin += (size_t)y * 2 * a.nc;
    a.out += (size_t)y * a.nc;
    a.part += (size_t)y * FP_NSLOT * a.pstride;
    a.st += y;
    a.hist += (size_t)y * (a.maxiter + 1);
    if (a.mixed) {
        a.r32 += o;
        a.z32 += o;
        a.pring32 += o;
        a.sring32 += o;
        a.xm[0] += o;
        a.xm[1] += o;
        a.dm[0] += o;
        a.dm[1] += o;
    }
}

// In a batch, the kernels of a converged member return at once.
#define FP_MEMBER(a)                                  \
    fp_member(a);                                     \
    if (a.nmem > 1 && a.st->done) return


__device__ __forceinline__ double *fslot(const FpArgs &a, int s) { return a.part + (size_t)s * a.pstride; }

// Block sums of nv <= FP_MAX_TRUNC values at once (one barrier round instead
// of nv): warp xor trees, then warp 0 adds the 32 warp sums in a fixed order.
// Every thread gets the sums in v.  sm: 32 * FP_MAX_TRUNC + FP_MAX_TRUNC doubles.
__device__ void block_sum_multi(double *v, int nv, double *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = 0; j < nv; ++j) {
        double x = v[j];
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sm[warp * FP_MAX_TRUNC + j] = x;
    }
    __syncthreads();
    if (warp == 0)
        for (int j = 0; j < nv; ++j) {
            double x = lane < nw ? sm[lane * FP_MAX_TRUNC + j] : 0.0;
            for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) sm[32 * FP_MAX_TRUNC + j] = x;
        }
    __syncthreads();
    for (int j = 0; j < nv; ++j) v[j] = sm[32 * FP_MAX_TRUNC + j];
    __syncthreads();
}

#define FP_ROW const int i = blockIdx.x * CG_TILE + threadIdx.x

// x = 0, r = b; partials |b|^2, |r|^2.
__global__ void __launch_bounds__(CG_TILE) k_fp_init(FpArgs a, double tol) {
    fp_member(a);
    __shared__ double sm[33];
    FP_ROW;
    double bb = 0;
    if (i < a.n) {
        const double bi = a.b[i];
        a.x[i] = 0.0;
        a.r[i] = bi;
        bb = __dmul_rn(bi, bi);
    }
    bb = block_sum(bb, sm);
    if (threadIdx.x == 0) {
        fslot(a, FP_BB)[blockIdx.x] = bb;
        fslot(a, FP_RR)[blockIdx.x] = bb;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->k = 0;
        a.st->done = 0;
        a.st->best_rr = 1e300;
        a.st->best_k = 0;
        for (int j = 0; j <= FP_MAX_TRUNC; ++j) a.st->ps[j] = 0;
        a.st->target = -tol;  // resolved by k_fp_pre from |b|
    }
}

// ------------------------------------------------ smoothing, temporally blocked
// The preconditioner's Jacobi sweeps run in FP32 (the Krylov recurrences
// around them stay FP64; a preconditioner may be inexact in flexible CG) on
// FP_TILE x FP_TILE tiles held in shared memory with a halo as wide as the
// sweeps need, so that all sweeps of one application (and what surrounds
// them) take one launch: each sweep shrinks the valid region by one cell,
// and the arithmetic is the operator's (A u)_i = dg u_i - we_{i-1} u_{i-1} -
// we_i u_{i+1} - wn_{i-nx} u_{i-nx} - wn_i u_{i+nx}, in that order.  The
// region holds we = wn = r = u = 0, dg = 1 and wd = 0 outside the grid, and
// the face coefficients of the grid's last column and row are 0, so the
// apply needs no boundary test: a term across the boundary adds -0 * 0 or
// -0 * u, which leaves the sum unchanged (up to the sign of a zero), and a
// sweep leaves the cells outside the grid at 0.  A thread visits the region
// cells threadIdx.x + j blockDim.x, j < FP_MAXC, in every loop (no division
// inside the sweeps: each cell's margin is computed once).
constexpr int FP_TILE = 32;  // one thread per tile cell: FP_TILE^2 = CG_TILE threads
static_assert(FP_TILE * FP_TILE == CG_TILE, "one thread per tile cell");
constexpr int FP_MAX_SMOOTH = 8;
constexpr int FP_MAXC = 3;  // region cells per thread: (FP_TILE + 2 FP_MAX_SMOOTH)^2 <= FP_MAXC CG_TILE
static_assert((FP_TILE + 2 * FP_MAX_SMOOTH) * (FP_TILE + 2 * FP_MAX_SMOOTH) <= FP_MAXC * CG_TILE, "region cells");

// Region arrays [R * R] each, region-local, one after the other in shared
// memory: r, z0, z1, we, wn, dg, wd = omega / dg (addressed from one base
// to keep registers free).
struct FpTile {
    int x0, y0, H, R, RR;  // tile origin, halo, region side (FP_TILE + 2 H), R * R
    float *d;
    __device__ __forceinline__ float *r() const { return d; }
    __device__ __forceinline__ float *z0() const { return d + RR; }
    __device__ __forceinline__ float *z1() const { return d + 2 * RR; }
    __device__ __forceinline__ float *we() const { return d + 3 * RR; }
    __device__ __forceinline__ float *wn() const { return d + 4 * RR; }
    __device__ __forceinline__ float *dg() const { return d + 5 * RR; }
    __device__ __forceinline__ float *wd() const { return d + 6 * RR; }
};

__device__ __forceinline__ bool fp_inside(const FpTile &t, const FpArgs &a, int row, int col, int *gi) {
    const int gx = t.x0 - t.H + col, gy = t.y0 - t.H + row;
    *gi = gy * a.op.nx + gx;
    return gx >= 0 && gx < a.op.nx && gy >= 0 && gy < a.op.ny;
}

// Loads the region (r and the operator, zero outside the grid) and sets
// z0[l] = init(l, row, col, inside, global index, wd[l], r[l]) for every
// region cell; the margins of this thread's cells go to mg[].
template <class Init>
__device__ FpTile fp_tile(const FpArgs &a, int bx, int H, unsigned char *smem, int *mg, Init init) {
    FpTile t;
    t.x0 = (bx % a.tx2) * FP_TILE;
    t.y0 = (bx / a.tx2) * FP_TILE;
    t.H = H;
    t.R = FP_TILE + 2 * H;
    t.d = reinterpret_cast<float *>(smem);
    t.RR = t.R * t.R;
#pragma unroll
    for (int j = 0; j < FP_MAXC; ++j) {
        const int l = threadIdx.x + j * CG_TILE;
        mg[j] = -1;
        if (l >= t.RR) continue;
        const int row = l / t.R, col = l - row * t.R;
        mg[j] = min(min(row, col), min(t.R - 1 - row, t.R - 1 - col));
        int i;
        const bool in = fp_inside(t, a, row, col, &i);
        const float r = in ? (a.mixed ? a.r32[i] : (float)a.r[i]) : 0.f;
        const float wd = in ? a.wd32[i] : 0.f;
        t.r()[l] = r;
        t.we()[l] = in ? a.we32[i] : 0.f;
        t.wn()[l] = in ? a.wn32[i] : 0.f;
        t.dg()[l] = in ? a.dg32[i] : 1.f;
        t.wd()[l] = wd;
        t.z0()[l] = init(l, row, col, in, i, wd, r);
    }
    return t;
}

// (A u) at region cell l (not on the region's outer ring); no boundary test
// (see above).
__device__ __forceinline__ float fp_apply(const FpTile &t, const float *u, int l) {
    const float *we = t.we(), *wn = t.wn();
    float v = __fmul_rn(t.dg()[l], u[l]);
    v = __fmaf_rn(-we[l - 1], u[l - 1], v);
    v = __fmaf_rn(-we[l], u[l + 1], v);
    v = __fmaf_rn(-wn[l - t.R], u[l - t.R], v);
    v = __fmaf_rn(-wn[l], u[l + t.R], v);
    return v;
}

// `sweeps` damped Jacobi sweeps on A z = r, z += (omega / dg) (r - A z),
// starting from *cur (valid at margin m0 of the region); returns the buffer
// holding the result, valid at margin m0 + sweeps.  Sweep s updates the
// cells of margin >= m0 + s + 1 only, so it reads only cells the previous
// sweep (or the start) wrote.
__device__ float *fp_sweeps(const FpTile &t, const int *mg, float *cur, float *nxt, int m0, int sweeps) {
    for (int s = 0; s < sweeps; ++s) {
        const int m = m0 + s + 1;
#pragma unroll
        for (int j = 0; j < FP_MAXC; ++j) {
            if (mg[j] < m) continue;
            const int l = threadIdx.x + j * CG_TILE;
            const float res = t.r()[l] - fp_apply(t, cur, l);
            nxt[l] = __fmaf_rn(t.wd()[l], res, cur[l]);
        }
        __syncthreads();
        float *sw = cur;
        cur = nxt;
        nxt = sw;
    }
    return cur;
}

// Start of the preconditioner (one launch): [k += 1 when `tick`; block 0:
// |r|^2 history, convergence / stall test]; z0 = `smooth` sweeps from zero
// and, when the network follows (`net_next`), r1 = r - A z0, partial
// |r1|^2, and the network input channel 0 = R(r1) (f x f means; the network
// scales it by 1 / rms(r1) itself).
__device__ __forceinline__ void k_fp_pre_blk(const FpArgs &a, int bx, int tick, int net_next) {
    __syncthreads();  // a previous call on this block has read its shared tile
    extern __shared__ __align__(16) unsigned char fp_smem[];
    __shared__ double sm[33];
    if (bx == 0) {
        const double rr = sum_partials(fslot(a, FP_RR), a.ntiles, sm);
        const double bb = sum_partials(fslot(a, FP_BB), a.ntiles, sm);
        const double tt = a.mixed ? sum_partials(fslot(a, FP_TT), a.ntiles, sm) : 0.0;
        if (threadIdx.x == 0) {
            FpState *st = a.st;
            if (tick) st->k += 1;
            double target = st->target;
            if (target < 0) {  // first call: target = tol * |b|
                target = -target * sqrt(bb);
                st->target = target;
            }
            if (st->k <= a.maxiter) a.hist[st->k] = sqrt(rr);
            if (!a.mixed) {
                if (sqrt(rr) <= target) st->done = 1;
            } else if (st->pending) {  // a reliable update ran: the FP64 true residual judges
                st->par ^= 1;
                st->pending = 0;
                st->updates += 1;
                st->gmax = rr;
                if (sqrt(tt) <= target) st->done = 1;
            } else if (rr > st->gmax) {
                st->gmax = rr;
            }
            if (rr < st->best_rr) {
                st->best_rr = rr;
                st->best_k = st->k;
            } else if (st->k - st->best_k > a.stall) {
                st->done = 2;
            }
            if (st->k >= a.maxiter && !st->done) st->done = 2;
        }
    }
    const int H = a.smooth > 0 ? a.smooth : 1;
    int mg[FP_MAXC];
    // sweep 1 from zero is pointwise: z = (omega / dg) r on the whole region
    const int smooth = a.smooth;
    FpTile t = fp_tile(a, bx, H, fp_smem, mg, [&](int, int, int, bool, int, float wd, float r) {
        return smooth > 0 ? wd * r : 0.f;
    });
    __syncthreads();
    const float *z = a.smooth > 1 ? fp_sweeps(t, mg, t.z0(), t.z1(), 0, a.smooth - 1) : t.z0();
    // this thread's tile cell
    const int lx = threadIdx.x & (FP_TILE - 1), ly = threadIdx.x / FP_TILE;
    const int row = H + ly, col = H + lx, l = row * t.R + col;
    int i;
    const bool in = fp_inside(t, a, row, col, &i);
    if (!net_next) {
        if (in) a.za[i] = (double)z[l];
        return;
    }
    double q = 0;
    if (in) {
        const double v = (double)(t.r()[l] - fp_apply(t, z, l));
        a.r1[i] = v;
        a.za[i] = (double)z[l];
        q = v * v;
    }
    q = block_sum(q, sm);  // (its barriers also order the r1 stores before the restriction)
    if (threadIdx.x == 0) fslot(a, FP_R1)[bx] = q;
    // restriction of this tile's cells (f divides FP_TILE and the tile origin)
    const int f = a.f, cs = FP_TILE / f;
    if (threadIdx.x < cs * cs) {
        const int cx = threadIdx.x % cs, cy = threadIdx.x / cs;
        const int gx = t.x0 + cx * f, gy = t.y0 + cy * f;
        if (gx < a.op.nx && gy < a.op.ny) {
            double sum = 0;
            for (int dy = 0; dy < f; ++dy)
                for (int dx = 0; dx < f; ++dx)
                    sum += a.r1[(size_t)(gy + dy) * a.op.nx + gx + dx];
            a.xin[2 * ((gy / f) * a.ncx + gx / f)] = (float)(sum / (f * f));
        }
    }
}
__global__ void __launch_bounds__(CG_TILE, 2) k_fp_pre(FpArgs a, int tick, int net_next) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_pre_blk(a, blockIdx.x, tick, net_next);
}

// End of the preconditioner (one launch): z = `smooth` sweeps starting from
// z0 + c P y, c = <P y, r1> / <P y, A P y> from the ydots partials (of all
// multiples of P y, c P y removes the most A-norm error from A d = r1, so the
// network's correction can only help the smoothed iterate), written to a.z
// with the partials <z_k, s_{k-1-j}> (j < min(k, m)) of the orthogonalisation.
__device__ __forceinline__ void k_fp_post_blk(const FpArgs &a, int bx, int use_y) {
    __syncthreads();  // a previous call on this block has read its shared tile
    extern __shared__ __align__(16) unsigned char fp_smem[];
    __shared__ double sm[33];
    double c = 0.0;  // without the network's y this iteration: smoothing alone
    if (use_y) {
        const double yr = sum_partials(fslot(a, FP_YR), a.ntiles, sm);
        const double yay = sum_partials(fslot(a, FP_YAY), a.ntiles, sm);
        c = yay > 0 ? yr / yay : 0.0;
    }
    const int H = a.smooth;
    int mg[FP_MAXC];
    const int x0 = (bx % a.tx2) * FP_TILE - H, y0 = (bx / a.tx2) * FP_TILE - H;
    FpTile t = fp_tile(a, bx, H, fp_smem, mg, [&](int, int row, int col, bool in, int i, float, float) {
        const int gx = x0 + col, gy = y0 + row;
        return in ? __double2float_rn(c != 0.0 && gx < a.mx && gy < a.my
                                          ? __fma_rn(c, (double)a.out[(gy >> a.fsh) * a.ncx + (gx >> a.fsh)], a.za[i])
                                          : a.za[i])
                  : 0.f;
    });
    __syncthreads();
    const float *z = fp_sweeps(t, mg, t.z0(), t.z1(), 0, a.smooth);
    const int lx = threadIdx.x & (FP_TILE - 1), ly = threadIdx.x / FP_TILE;
    const int row = H + ly, col = H + lx, l = row * t.R + col;
    int i;
    const bool in = fp_inside(t, a, row, col, &i);
    double zi = 0;
    if (in) {
        zi = (double)z[l];
        if (a.mixed) a.z32[i] = z[l];
        else a.z[i] = zi;
    }
    const int k = (int)a.st->k;
    const int nj = min(a.m, k);
    if (nj > 0) {
        __shared__ double smm[33 * FP_MAX_TRUNC];
        __shared__ size_t sj[FP_MAX_TRUNC];  // ring slot offsets of s_{k-1-j}
        if (threadIdx.x < nj) sj[threadIdx.x] = (size_t)((k - 1 - (int)threadIdx.x) % a.ring) * a.sstride;
        __syncthreads();
        double v[FP_MAX_TRUNC];
#pragma unroll
        for (int j = 0; j < FP_MAX_TRUNC; ++j)
            v[j] = (j < nj && in) ? (a.mixed ? xprod(z[l], a.sring32[sj[j] + i])
                                             : __dmul_rn(zi, a.sring[sj[j] + i]))
                                  : 0.0;
        block_sum_multi(v, nj, smm);
        if (threadIdx.x < nj) fslot(a, FP_ZS + threadIdx.x)[bx] = v[threadIdx.x];
    }
}
__global__ void __launch_bounds__(CG_TILE, 2) k_fp_post(FpArgs a, int use_y) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_post_blk(a, blockIdx.x, use_y);
}

size_t fp_smem_bytes(int H) { return 7 * sizeof(float) * (size_t)(FP_TILE + 2 * H) * (FP_TILE + 2 * H); }

// omega / dg in FP32 for the smoothing (once per solver).
__global__ void k_fp_wd(const float *dg32, float *wd32, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        wd32[i] = (float)(JACOBI_OMEGA / (double)dg32[i]);
}

// Identity in place of the network: out = R(r1) (unscaled; c absorbs the scale).
__global__ void k_fp_identity(FpArgs a) {
    pdl_enter();
    const long long nall = (long long)a.nc * a.nmem;  // every member's coarse cells, one after the other
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < nall; i += gridDim.x * blockDim.x)
        a.out[i] = a.xin[2 * i];
}

// Partials <z, r1> and <z, A z> of the prolongated network output z = P y
// (FP32 values, applied in FP64).
__device__ __forceinline__ void k_fp_ydots_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const int i = bx * CG_TILE + threadIdx.x;
    double yr = 0, yay = 0;
    if (i < a.n) {
        const StencilOp<2> &o = a.op;
        const int nx = o.nx, iy = i / nx, ix = i - iy * nx;
        const int sh = a.fsh, cx = ix >> sh, cy = iy >> sh;
        const float *y = a.out;  // z = P y on this grid: z[j] = y[cell(j)]
        const float *yrow = y + cy * a.ncx;
        // P y inside the member's extent (the whole grid for one system), 0 outside
        const int mx = a.mx, my = a.my;
        auto pv = [&](int jx, int jy) {
            return (jx < mx && jy < my) ? (double)y[(jy >> sh) * a.ncx + (jx >> sh)] : 0.0;
        };
        const double zi = (ix < mx && iy < my) ? (double)yrow[cx] : 0.0;
        double t = __dmul_rn(o.dg[i], zi);
        if (ix > 0) t = __fma_rn(-o.we[i - 1], pv(ix - 1, iy), t);
        if (ix < nx - 1) t = __fma_rn(-o.we[i], pv(ix + 1, iy), t);
        if (iy > 0) t = __fma_rn(-o.wn[i - nx], pv(ix, iy - 1), t);
        if (iy < o.ny - 1) t = __fma_rn(-o.wn[i], pv(ix, iy + 1), t);
        yr = __dmul_rn(zi, a.r1[i]);
        yay = __dmul_rn(zi, t);
    }
    yr = block_sum(yr, sm);
    yay = block_sum(yay, sm);
    if (threadIdx.x == 0) {
        fslot(a, FP_YR)[bx] = yr;
        fslot(a, FP_YAY)[bx] = yay;
    }
}
__global__ void __launch_bounds__(CG_TILE) k_fp_ydots(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_ydots_blk(a, blockIdx.x);
}

// p_k = z_k - sum_j (<z_k, s_j> / <p_j, s_j>) p_j over the last min(k, m)
// directions (into ring slot k mod (m + 1)), partial <p_k, r_k>, and the
// loop condition.
__device__ __forceinline__ void k_fp_dir_blk(const FpArgs &a, int bx, cudaGraphConditionalHandle cond, int set_cond) {
    __shared__ double sm[33];
    const int k = (int)a.st->k;
    const int nj = min(a.m, k);
    __shared__ const double *pj[FP_MAX_TRUNC];
    if (threadIdx.x < nj) pj[threadIdx.x] = a.pring + (size_t)((k - 1 - (int)threadIdx.x) % a.ring) * a.sstride;
    double beta[FP_MAX_TRUNC];
    if (nj > 0) {
        __shared__ double smm[33 * FP_MAX_TRUNC];
#pragma unroll
        for (int j = 0; j < FP_MAX_TRUNC; ++j) {
            double acc = 0.0;
            if (j < nj)
                for (int t = threadIdx.x; t < a.ntiles2; t += blockDim.x) acc += fslot(a, FP_ZS + j)[t];
            beta[j] = acc;
        }
        block_sum_multi(beta, nj, smm);
        for (int j = 0; j < nj; ++j) {
            const double ps = a.st->ps[(k - 1 - j) % a.ring];
            beta[j] = ps != 0.0 ? beta[j] / ps : 0.0;
        }
    }
    __syncthreads();  // pj
    const int i = bx * CG_TILE + threadIdx.x;
    double pr = 0;
    if (i < a.n) {
        if (a.mixed) {  // FP32 direction, beta rounded to FP32
            float pi = a.z32[i];
            for (int j = 0; j < nj; ++j)
                pi = __fmaf_rn(-__double2float_rn(beta[j]),
                               a.pring32[(size_t)((k - 1 - j) % a.ring) * a.sstride + i], pi);
            a.pring32[(size_t)(k % a.ring) * a.sstride + i] = pi;
            pr = xprod(pi, a.r32[i]);
        } else {
            double pi = a.z[i];
            for (int j = 0; j < nj; ++j) pi = __fma_rn(-beta[j], pj[j][i], pi);
            a.pring[(size_t)(k % a.ring) * a.sstride + i] = pi;
            pr = __dmul_rn(pi, a.r[i]);
        }
    }
    pr = block_sum(pr, sm);
    if (threadIdx.x == 0) fslot(a, FP_PR)[bx] = pr;
    if (set_cond && bx == 0 && threadIdx.x == 0)
        cudaGraphSetConditional(cond, a.st->done ? 0u : 1u);
}
__global__ void __launch_bounds__(CG_TILE) k_fp_dir(FpArgs a, cudaGraphConditionalHandle cond, int set_cond) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_dir_blk(a, blockIdx.x, cond, set_cond);
}

// s_k = A p_k; partial <p_k, s_k>.
__device__ __forceinline__ void k_fp_spmv_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const int slot = (int)a.st->k % a.ring;
    const double *p = a.pring + (size_t)slot * a.sstride;
    const int i = bx * CG_TILE + threadIdx.x;
    double ps = 0;
    if (i < a.n) {
        const double si = a.op.apply(p, i);
        a.sring[(size_t)slot * a.sstride + i] = si;
        ps = __dmul_rn(p[i], si);
    }
    ps = block_sum(ps, sm);
    if (threadIdx.x == 0) fslot(a, FP_PS)[bx] = ps;
}
__global__ void __launch_bounds__(CG_TILE) k_fp_spmv(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_spmv_blk(a, blockIdx.x);
}

// alpha = <p_k, r_k> / <p_k, s_k>; x += alpha p_k; r -= alpha s_k; |r|^2;
// <p_k, s_k> kept in the ring for the orthogonalisations to come.
__device__ __forceinline__ void k_fp_update_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const double ps = sum_partials(fslot(a, FP_PS), a.ntiles, sm);
    const double pr = sum_partials(fslot(a, FP_PR), a.ntiles, sm);
    const int slot = (int)a.st->k % a.ring;
    const double alpha = ps != 0.0 ? pr / ps : 0.0;
    const int i = bx * CG_TILE + threadIdx.x;
    double rr = 0;
    if (i < a.n) {
        a.x[i] = __fma_rn(alpha, a.pring[(size_t)slot * a.sstride + i], a.x[i]);
        const double rn = __fma_rn(-alpha, a.sring[(size_t)slot * a.sstride + i], a.r[i]);
        a.r[i] = rn;
        rr = __dmul_rn(rn, rn);
    }
    rr = block_sum(rr, sm);
    if (threadIdx.x == 0) fslot(a, FP_RR)[bx] = rr;
    if (bx == 0 && threadIdx.x == 0) a.st->ps[slot] = ps;
}
__global__ void __launch_bounds__(CG_TILE) k_fp_update(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fp_update_blk(a, blockIdx.x);
}

// ------------------------------------------------- mixed-precision kernels
// x = 0 (FP64 iterate and FP32 correction of parity 0), r32 = fl32(b);
// partials |b|^2 (FP64) and |r32|^2.
// The parity buffers of a mixed solve, chosen by a select rather than an
// index into the argument struct (a runtime index would copy the whole
// struct into local memory on every thread).
__device__ __forceinline__ double *fp_xm(const FpArgs &a, int par) { return par ? a.xm[1] : a.xm[0]; }
__device__ __forceinline__ float *fp_dm(const FpArgs &a, int par) { return par ? a.dm[1] : a.dm[0]; }

__global__ void __launch_bounds__(CG_TILE) k_fpm_init(FpArgs a, double tol) {
    fp_member(a);
    __shared__ double sm[33];
    FP_ROW;
    double bb = 0, rr = 0;
    if (i < a.n) {
        const double bi = a.b[i];
        const float ri = __double2float_rn(bi);
        a.xm[0][i] = 0.0;
        a.dm[0][i] = 0.f;
        a.r32[i] = ri;
        bb = __dmul_rn(bi, bi);
        rr = xprod(ri, ri);
    }
    bb = block_sum(bb, sm);
    rr = block_sum(rr, sm);
    if (threadIdx.x == 0) {
        fslot(a, FP_BB)[blockIdx.x] = bb;
        fslot(a, FP_RR)[blockIdx.x] = rr;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.st->k = 0;
        a.st->done = 0;
        a.st->best_rr = 1e300;
        a.st->best_k = 0;
        for (int j = 0; j <= FP_MAX_TRUNC; ++j) a.st->ps[j] = 0;
        a.st->target = -tol;
        a.st->gmax = 0.0;
        a.st->par = 0;
        a.st->pending = 0;
        a.st->updates = 0;
    }
}

// s32 = A p32 with the FP32 operator; partial <p32, s32> (FP64 sum of the
// exact FP32 products).
__device__ __forceinline__ void k_fpm_spmv_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const int slot = (int)a.st->k % a.ring;
    const float *p = a.pring32 + (size_t)slot * a.sstride;
    const int i = bx * CG_TILE + threadIdx.x;
    double ps = 0;
    if (i < a.n) {
        const float si = a.op.apply32(p, i);
        a.sring32[(size_t)slot * a.sstride + i] = si;
        ps = xprod(p[i], si);
    }
    ps = block_sum(ps, sm);
    if (threadIdx.x == 0) fslot(a, FP_PS)[bx] = ps;
}
__global__ void __launch_bounds__(CG_TILE) k_fpm_spmv(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fpm_spmv_blk(a, blockIdx.x);
}

// alpha = <p, r> / <p, s> (FP64, applied rounded to FP32); d += alpha p,
// r32 -= alpha s (FP32); partial |r32|^2.
__device__ __forceinline__ void k_fpm_update_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const double ps = sum_partials(fslot(a, FP_PS), a.ntiles, sm);
    const double pr = sum_partials(fslot(a, FP_PR), a.ntiles, sm);
    const int slot = (int)a.st->k % a.ring;
    const float af = __double2float_rn(ps != 0.0 ? pr / ps : 0.0);
    float *d = fp_dm(a, a.st->par);
    const int i = bx * CG_TILE + threadIdx.x;
    double rr = 0;
    if (i < a.n) {
        d[i] = __fmaf_rn(af, a.pring32[(size_t)slot * a.sstride + i], d[i]);
        const float rn = __fmaf_rn(-af, a.sring32[(size_t)slot * a.sstride + i], a.r32[i]);
        a.r32[i] = rn;
        rr = xprod(rn, rn);
    }
    rr = block_sum(rr, sm);
    if (threadIdx.x == 0) fslot(a, FP_RR)[bx] = rr;
    if (bx == 0 && threadIdx.x == 0) a.st->ps[slot] = ps;
}
__global__ void __launch_bounds__(CG_TILE) k_fpm_update(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fpm_update_blk(a, blockIdx.x);
}

// Reliable update, when |r32|^2 has reached tol^2 |b|^2 or fallen below
// delta^2 times its largest value since the last update (every block sums
// the same partials in the same order, so all decide alike; otherwise they
// return at once): x' = x + d in FP64 into
// the other parity's buffer, d' = 0, t = b - A x' (FP64, A x' from x + d on
// the fly, so no grid barrier), r32 = fl32(t); partials |t|^2 and |r32|^2.
// k_fp_pre flips the parity and judges convergence by |t|.
__device__ __forceinline__ void k_fpm_reliable_blk(const FpArgs &a, int bx) {
    __shared__ double sm[33];
    const double g = sum_partials(fslot(a, FP_RR), a.ntiles, sm);
    const FpState *st = a.st;
    const double target = st->target;
    if (!(g <= target * target || g < a.delta2 * st->gmax)) return;
    const int par = st->par;
    const double *x = fp_xm(a, par);
    const float *d = fp_dm(a, par);
    const int i = bx * CG_TILE + threadIdx.x;
    double tt = 0, rr = 0;
    if (i < a.n) {
        const StencilOp<2> &o = a.op;
        const int nx = o.nx, iy = i / nx, ix = i - iy * nx;
        auto xv = [&](int j) { return __dadd_rn(x[j], (double)d[j]); };
        const double xi = xv(i);
        double t = __dmul_rn(o.dg[i], xi);
        if (ix > 0) t = __fma_rn(-o.we[i - 1], xv(i - 1), t);
        if (ix < nx - 1) t = __fma_rn(-o.we[i], xv(i + 1), t);
        if (iy > 0) t = __fma_rn(-o.wn[i - nx], xv(i - nx), t);
        if (iy < o.ny - 1) t = __fma_rn(-o.wn[i], xv(i + nx), t);
        const double ti = __dsub_rn(a.b[i], t);
        const float ri = __double2float_rn(ti);
        fp_xm(a, par ^ 1)[i] = xi;
        fp_dm(a, par ^ 1)[i] = 0.f;
        a.r32[i] = ri;
        tt = __dmul_rn(ti, ti);
        rr = xprod(ri, ri);
    }
    tt = block_sum(tt, sm);
    rr = block_sum(rr, sm);
    if (threadIdx.x == 0) {
        fslot(a, FP_TT)[bx] = tt;
        fslot(a, FP_RR)[bx] = rr;
    }
    if (bx == 0 && threadIdx.x == 0) a.st->pending = 1;
}
__global__ void __launch_bounds__(CG_TILE) k_fpm_reliable(FpArgs a) {
    pdl_enter();
    FP_MEMBER(a);
    k_fpm_reliable_blk(a, blockIdx.x);
}

// ------------------------------------------------------ single-system device loop
// The phases of one or more FPCG iterations of a single system in one
// cooperative launch, a grid barrier between phases instead of a kernel
// boundary: each phase walks its blocks (row tiles, or smoothing tiles for
// pre / post) as virtual blocks of the persistent grid and runs the same
// block body as its kernel, so the arithmetic, and every result, is the
// per-kernel path's.  The network runs between two such launches.
enum FpPhaseCode : int {
    FPP_SPMV,
    FPP_UPDATE,
    FPP_MSPMV,
    FPP_MUPDATE,
    FPP_MRELIABLE,
    FPP_PRE,       // x: tick, y: net_next
    FPP_IDENTITY,  // the network's stand-in without a network: y = R r1
    FPP_YDOTS,
    FPP_POST,      // x: use_y
    FPP_DIR        // x: set the loop condition
};
struct FpOp {
    int code, x, y;
};
constexpr int FP_MAX_OPS = 48;
struct FpProgram {
    int n;
    FpOp op[FP_MAX_OPS];
};

__global__ void __launch_bounds__(CG_TILE, 2)
    k_fp_loop(const FpArgs a, const FpProgram pg, BarrierState *bar, cudaGraphConditionalHandle cond) {
    for (int s = 0; s < pg.n; ++s) {
        const int code = pg.op[s].code, ox = pg.op[s].x, oy = pg.op[s].y;
        if (code == FPP_IDENTITY) {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.nc;
                 i += (long long)gridDim.x * blockDim.x)
                a.out[i] = a.xin[2 * i];
        } else {
            const int nvb = (code == FPP_PRE || code == FPP_POST) ? a.ntiles2 : a.ntiles;
            for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
                switch (code) {
                    case FPP_SPMV: k_fp_spmv_blk(a, vb); break;
                    case FPP_UPDATE: k_fp_update_blk(a, vb); break;
                    case FPP_MSPMV: k_fpm_spmv_blk(a, vb); break;
                    case FPP_MUPDATE: k_fpm_update_blk(a, vb); break;
                    case FPP_MRELIABLE: k_fpm_reliable_blk(a, vb); break;
                    case FPP_PRE: k_fp_pre_blk(a, vb, ox, oy); break;
                    case FPP_YDOTS: k_fp_ydots_blk(a, vb); break;
                    case FPP_POST: k_fp_post_blk(a, vb, ox); break;
                    case FPP_DIR: k_fp_dir_blk(a, vb, cond, ox); break;
                    default: break;
                }
            }
        }
        if (s + 1 < pg.n && !grid_barrier(bar, gridDim.x, s)) return;
    }
}

// The result of a mixed solve: x = xm + dm of the current parity (FP64), for
// every member (each with its own parity).
__global__ void k_fpm_finish(FpArgs a, const FpState *st) {
    const long long nall = (long long)a.n * a.nmem;
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < nall; i += gridDim.x * blockDim.x) {
        const int par = st[i / a.n].par;
        a.x[i] = __dadd_rn(fp_xm(a, par)[i], (double)fp_dm(a, par)[i]);
    }
}

// Loop condition of a batch: go on while any member is not done.
__global__ void k_fpb_cond(const FpState *st, int nmem, cudaGraphConditionalHandle cond) {
    pdl_enter();
    int open = 0;
    for (int y = threadIdx.x; y < nmem; y += blockDim.x) open |= st[y].done == 0;
    open = __any_sync(0xffffffffu, open);
    if (threadIdx.x == 0) cudaGraphSetConditional(cond, open ? 1u : 0u);
}

// Per-member FP64 true residual t = b - A x, |t|^2 into acc[y] (grid sums in
// block order: slots of gridDim.x doubles and one counter per member).
__global__ void k_fpb_true_res(FpArgs a, double *t, double *acc, double *slots, unsigned int *count) {
    fp_member(a);
    const int y = blockIdx.y;
    t += (size_t)y * a.n;
    __shared__ double red[32];
    double q = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double ti = a.b[i] - a.op.apply(a.x, i);
        t[i] = ti;
        q += ti * ti;
    }
    for (int o = 16; o; o >>= 1) q += __shfl_xor_sync(CG_FULL, q, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q;
    __syncthreads();
    double v = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)blockDim.x / 32; ++w) v += red[w];
    ordered_grid_sum<1>(&v, slots + (size_t)y * gridDim.x, blockIdx.x, gridDim.x, count + y, acc + y, false);
}

// t = b - A x, |t|^2 into acc[0] (the judged true residual; grid sum in
// block order: slots of gridDim.x doubles, one counter).
__global__ void k_fp_true_res(StencilOp<2> op, int n, const double *b, const double *x, double *t,
                              double *acc, double *slots, unsigned int *count) {
    __shared__ double red[32];
    double q = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ti = b[i] - op.apply(x, i);
        t[i] = ti;
        q += ti * ti;
    }
    for (int o = 16; o; o >>= 1) q += __shfl_xor_sync(CG_FULL, q, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q;
    __syncthreads();
    double v = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)blockDim.x / 32; ++w) v += red[w];
    ordered_grid_sum<1>(&v, slots, blockIdx.x, gridDim.x, count, acc, false);
}

// Network input channel 1: the mean of log k over each f x f block.
__global__ void k_log_coarse(const double *k, float *xin, int nx, int ny, int f) {
    const int ncx = nx / f, nc = (nx / f) * (ny / f);
    for (int ic = blockIdx.x * blockDim.x + threadIdx.x; ic < nc; ic += gridDim.x * blockDim.x) {
        const int cx = ic % ncx, cy = ic / ncx;
        double sum = 0;
        for (int dy = 0; dy < f; ++dy)
            for (int dx = 0; dx < f; ++dx) sum += log(k[(size_t)(cy * f + dy) * nx + cx * f + dx]);
        xin[2 * ic + 1] = (float)(sum / (f * f));
    }
}

__global__ void k_axpy_inplace(double *x, const double *d, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += d[i];
}

}  // namespace

}  // namespace cfm

using namespace cfm;

struct cfm_fpcg {
    const cfm_stencil *S = nullptr;
    cfm_unet *net = nullptr;
    int n = 0, ntiles = 0, nx = 0, ny = 0;
    int ntiles2 = 0, tx2 = 0, pstride = 0;  // smoothing tiles (FP_TILE^2) and partial-slot stride
    int coarsen = 1, nc = 0;  // the network runs on (nx / coarsen) x (ny / coarsen) = nc cells
    long long maxiter = 0;
    double tol = 0;
    double *vec = nullptr;   // x r z b t d za r1 (FP_NVEC n)
    int m = 0;               // FCG truncation
    int net_every = 1;       // the network in one of every net_every iterations
    float *wd32 = nullptr;   // omega / dg (FP32)
    double *ring = nullptr;  // p and A p ring slots: 2 (m + 1) n
    int smooth = 0;
    float *xin = nullptr, *out = nullptr;
    double *part = nullptr, *acc = nullptr, *hist = nullptr;
    double *rslots = nullptr;       // block sums of the true residual (FP_RES_BLOCKS)
    unsigned int *rcount = nullptr;  // their arrival counter
    FpState *st = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool conditional = false;
    long long last_k = 0;
    // mixed precision (cfm_fpcg_set_precision): r32 z32 | FP32 rings (2 (m + 1) n)
    // | FP32 corrections (2 n) and FP64 iterates (2 n) by update parity
    int mixed = 0;
    double delta = 0.1;
    float *vec32 = nullptr, *ring32 = nullptr;
    double *xm = nullptr;
    int last_updates = 0;
    // a batch (cfm_fpcg_create_batch): nmem members, each embedded in the
    // nx x ny frame; every per-member array holds nmem slices of n (vector
    // k of FP_NVEC at k n nmem), the coefficients we | wn | wt | dg likewise
    int nmem = 1;
    double *c64b = nullptr;
    float *c32b = nullptr;
    int2 *ext = nullptr;         // member extents (device)
    double *cells = nullptr;     // member cell counts (device; the network's input scale)
    std::vector<int2> ext_h;
    // single-system device loop (k_fp_loop, cfm_fpcg_set_device_loop): off
    // by default (slower than the per-phase kernels chained by programmatic
    // dependent launch); its grid (0: unavailable) and barrier
    int loop = 0;
    int loop_grid = 0;
    BarrierState *bar = nullptr;
};

namespace {

FpArgs fp_args(cfm_fpcg *h) {
    FpArgs a{};
    const size_t n = h->n, N = n * h->nmem;  // N: one vector of every member
    const double *c64 = h->c64b ? h->c64b : stencil_coeffs(h->S);    // we | wn | wt | dg
    const float *c32 = h->c32b ? h->c32b : stencil_coeffs32(h->S);
    a.op.nx = h->nx;
    a.op.ny = h->ny;
    a.op.nz = 1;
    a.op.we = c64;
    a.op.wn = c64 + N;
    a.op.wt = c64 + 2 * N;
    a.op.dg = c64 + 3 * N;
    a.n = h->n;
    a.ntiles = h->ntiles;
    a.x = h->vec;
    a.r = h->vec + N;
    a.z = h->vec + 2 * N;
    a.b = h->vec + 3 * N;
    a.za = h->vec + 6 * N;
    a.r1 = h->vec + 7 * N;
    static_assert(FP_NVEC == 8, "x r z b t d za r1");
    a.m = h->m;
    a.ring = h->m + 1;
    a.pring = h->ring;
    a.sring = h->ring + (size_t)(h->m + 1) * N;
    a.nmem = h->nmem;
    a.sstride = (long long)N;
    a.ext = h->ext;
    a.mx = h->nx;
    a.my = h->ny;
    a.xin = h->xin;
    a.out = h->out;
    a.part = h->part;
    a.st = h->st;
    a.hist = h->hist;
    a.maxiter = h->maxiter;
    a.stall = 200;
    a.f = h->coarsen;
    a.fsh = h->coarsen == 2 ? 1 : 0;
    a.ncx = h->nx / h->coarsen;
    a.nc = h->nc;
    a.ntiles2 = h->ntiles2;
    a.we32 = c32;
    a.wn32 = c32 + N;
    a.dg32 = c32 + 3 * N;
    a.wd32 = h->wd32;
    a.op.we32 = c32;  // the operator's FP32 apply (mixed precision)
    a.op.wn32 = c32 + N;
    a.op.wt32 = c32 + 2 * N;
    a.op.dg32 = c32 + 3 * N;
    a.tx2 = h->tx2;
    a.pstride = h->pstride;
    a.smooth = h->smooth;
    a.mixed = h->mixed;
    a.delta2 = h->delta * h->delta;
    if (h->mixed) {
        a.r32 = h->vec32;
        a.z32 = h->vec32 + N;
        a.dm[0] = h->vec32 + 2 * N;
        a.dm[1] = h->vec32 + 3 * N;
        a.pring32 = h->ring32;
        a.sring32 = h->ring32 + (size_t)(h->m + 1) * N;
        a.xm[0] = h->xm;
        a.xm[1] = h->xm + N;
    }
    return a;
}

// One FPCG iteration's tail (from the preconditioner on), five launches:
// k_fp_pre (k += 1 when `tick`, convergence test, z0 = `smooth` Jacobi
// sweeps from zero, r1 = r - A z0, R(r1)), the network y = net(R(r1) /
// rms(r1), log k) (or the identity), k_fp_ydots (<P y, r1>, <P y, A P y>),
// k_fp_post (z = `smooth` sweeps from z0 + c P y, <z, r>, <z, r_old>) and
// k_fp_dir (beta, p, the loop condition).
// The network on R r1 of every member: the members in chunks of the
// network's largest batch; image z of a chunk scales its input by its own
// member's |r1| partials and cells.
int fp_network(cfm_fpcg *h, const FpArgs &a) {
    const int M = h->nmem;
    const long long mstride = (long long)FP_NSLOT * a.pstride;
    for (int m0 = 0; m0 < M; m0 += h->net->maxB) {
        const int B = std::min(h->net->maxB, M - m0);
        UNetInputScale sc{a.part + (size_t)FP_R1 * a.pstride + (size_t)m0 * mstride, h->ntiles2, (double)h->n};
        sc.part_stride = mstride;
        sc.cells_img = h->cells ? h->cells + m0 : nullptr;
        const int st = unet_forward(h->net->u, B, h->xin + (size_t)m0 * 2 * h->nc, h->out + (size_t)m0 * h->nc,
                                    h->stream, &sc);
        if (st) return st;
    }
    return CFM_OK;
}

int fp_precond_dir(cfm_fpcg *h, const FpArgs &a, cudaGraphConditionalHandle cond, int set_cond, int tick,
                   bool use_net = true) {
    cudaStream_t s = h->stream;
    const int net_next = !(h->net && !use_net);
    const int M = h->nmem;
    CFM_CUDA_TRY(launch_pdl(k_fp_pre, dim3(h->ntiles2, M), dim3(CG_TILE), fp_smem_bytes(std::max(h->smooth, 1)),
                            s, a, tick, net_next));
    if (!net_next) {
        // smoothing alone this iteration: no r1, no network, c = 0
        CFM_CUDA_TRY(launch_pdl(k_fp_post, dim3(h->ntiles2, M), dim3(CG_TILE), fp_smem_bytes(h->smooth), s, a, 0));
        CFM_CUDA_TRY(launch_pdl(k_fp_dir, dim3(h->ntiles, M), dim3(CG_TILE), 0, s, a, cond, set_cond));
        return CFM_OK;
    }
    if (h->net) {
        const int st = fp_network(h, a);
        if (st) return st;
    } else {
        CFM_CUDA_TRY(launch_pdl(k_fp_identity, dim3(256), dim3(256), 0, s, a));
    }
    CFM_CUDA_TRY(launch_pdl(k_fp_ydots, dim3(h->ntiles, M), dim3(CG_TILE), 0, s, a));
    CFM_CUDA_TRY(launch_pdl(k_fp_post, dim3(h->ntiles2, M), dim3(CG_TILE), fp_smem_bytes(h->smooth), s, a, 1));
    CFM_CUDA_TRY(launch_pdl(k_fp_dir, dim3(h->ntiles, M), dim3(CG_TILE), 0, s, a, cond, set_cond));
    return CFM_OK;
}

int fp_iteration(cfm_fpcg *h, const FpArgs &a, cudaGraphConditionalHandle cond, int set_cond, bool use_net) {
    const dim3 g(h->ntiles, h->nmem);
    if (h->mixed) {
        CFM_CUDA_TRY(launch_pdl(k_fpm_spmv, g, dim3(CG_TILE), 0, h->stream, a));
        CFM_CUDA_TRY(launch_pdl(k_fpm_update, g, dim3(CG_TILE), 0, h->stream, a));
        CFM_CUDA_TRY(launch_pdl(k_fpm_reliable, g, dim3(CG_TILE), 0, h->stream, a));
    } else {
        CFM_CUDA_TRY(launch_pdl(k_fp_spmv, g, dim3(CG_TILE), 0, h->stream, a));
        CFM_CUDA_TRY(launch_pdl(k_fp_update, g, dim3(CG_TILE), 0, h->stream, a));
    }
    return fp_precond_dir(h, a, cond, set_cond, 1, use_net);
}

// Drops the captured iteration graph (it holds buffer addresses and the
// kernel sequence); the next solve builds it again.
void drop_graph(cfm_fpcg *h) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->exec = nullptr;
    h->graph = nullptr;
    h->conditional = false;
}

// FP32 rings of the mixed solve for truncation m.
int alloc_ring32(cfm_fpcg *h, int m) {
    float *r = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&r, sizeof(float) * 2 * (m + 1) * (size_t)h->n * h->nmem));
    cudaFree(h->ring32);
    h->ring32 = r;
    return CFM_OK;
}

// One pass of the device loop: h->net_every iterations, the network in the
// first (a converged system may take up to net_every - 1 extra iterations,
// which only lower its residual further).
// One device-loop launch of the program's phases (none: nothing).
int fp_loop_launch(cfm_fpcg *h, const FpArgs &a, FpProgram &pg, cudaGraphConditionalHandle cond) {
    if (pg.n == 0) return CFM_OK;
    void *args[] = {(void *)&a, (void *)&pg, (void *)&h->bar, (void *)&cond};
    CFM_CUDA_TRY(launch_cooperative((const void *)k_fp_loop, dim3(h->loop_grid), dim3(CG_TILE), args,
                                    fp_smem_bytes(std::max(h->smooth, 1)), h->stream));
    pg.n = 0;
    return CFM_OK;
}

// The iterations of fp_body as device-loop launches: the phases of
// fp_iteration in order, a launch boundary only where the network runs
// (or where the program is full).
int fp_body_loop(cfm_fpcg *h, const FpArgs &a, cudaGraphConditionalHandle cond, int set_cond) {
    FpProgram pg{};
    int st;
    auto add = [&](int code, int x, int y) -> int {
        if (pg.n == FP_MAX_OPS) {
            const int e = fp_loop_launch(h, a, pg, cond);
            if (e) return e;
        }
        pg.op[pg.n++] = FpOp{code, x, y};
        return CFM_OK;
    };
    for (int j = 0; j < h->net_every; ++j) {
        const int set = set_cond && j == h->net_every - 1;
        const int net_next = !(h->net && j != 0);
        if ((st = add(h->mixed ? FPP_MSPMV : FPP_SPMV, 0, 0)) || (st = add(h->mixed ? FPP_MUPDATE : FPP_UPDATE, 0, 0)))
            return st;
        if (h->mixed && (st = add(FPP_MRELIABLE, 0, 0))) return st;
        if ((st = add(FPP_PRE, 1, net_next))) return st;
        if (!net_next) {
            if ((st = add(FPP_POST, 0, 0)) || (st = add(FPP_DIR, set, 0))) return st;
            continue;
        }
        if (h->net) {
            if ((st = fp_loop_launch(h, a, pg, cond)) || (st = fp_network(h, a))) return st;
        } else if ((st = add(FPP_IDENTITY, 0, 0))) {
            return st;
        }
        if ((st = add(FPP_YDOTS, 0, 0)) || (st = add(FPP_POST, 1, 0)) || (st = add(FPP_DIR, set, 0))) return st;
    }
    return fp_loop_launch(h, a, pg, cond);
}

int fp_body(cfm_fpcg *h, const FpArgs &a, cudaGraphConditionalHandle cond, int set_cond) {
    if (h->nmem == 1 && h->loop && h->loop_grid > 0) return fp_body_loop(h, a, cond, set_cond);
    const bool batch = h->nmem > 1;
    for (int j = 0; j < h->net_every; ++j) {
        const int st = fp_iteration(h, a, cond, set_cond && !batch && j == h->net_every - 1, j == 0);
        if (st) return st;
    }
    if (set_cond && batch)  // a batch goes on while any member is open
        CFM_CUDA_TRY(launch_pdl(k_fpb_cond, dim3(1), dim3(32), 0, h->stream, (const FpState *)h->st, h->nmem, cond));
    return CFM_OK;
}

// Graph: a conditional WHILE node whose body is one FPCG iteration.
int build_graph(cfm_fpcg *h) {
    const FpArgs a = fp_args(h);
    CFM_CUDA_TRY(cudaGraphCreate(&h->graph, 0));
    cudaGraphConditionalHandle cond;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, h->graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, h->graph, nullptr, 0, &cp);
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            CFM_CUDA_TRY(cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal));
            int st = fp_body(h, a, cond, 1);
            cudaGraph_t captured = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(h->stream, &captured);
            if (st) return st;
            CFM_CUDA_TRY(ce);
            h->conditional = true;
        }
    }
    if (!h->conditional) {
        // no conditional nodes: a graph of 16 iterations the host relaunches
        cudaGetLastError();
        cudaGraphDestroy(h->graph);
        h->graph = nullptr;
        CFM_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int st = 0;
        for (int i = 0; i < 16 && !st; ++i) st = fp_body(h, a, 0, 0);
        const cudaError_t ce = cudaStreamEndCapture(h->stream, &h->graph);
        if (st) return st;
        CFM_CUDA_TRY(ce);
    }
    CFM_CUDA_TRY(cudaGraphInstantiate(&h->exec, h->graph, 0));
    return CFM_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// Handle fields and device buffers of `nmem` systems on an nx x ny grid
// (frame); the coefficients, omega / dg and the network's log k channel are
// set by the caller.
int fp_setup(cfm_fpcg *h, int nx, int ny, int f, cfm_unet *net, int smooth, int maxiter, double tol,
             int nmem) {
    h->coarsen = f;
    h->nc = (nx / f) * (ny / f);
    h->smooth = smooth;
    h->net = net;
    h->nx = nx;
    h->ny = ny;
    h->n = nx * ny;
    h->nmem = nmem;
    h->ntiles = (h->n + CG_TILE - 1) / CG_TILE;
    h->tx2 = (nx + FP_TILE - 1) / FP_TILE;
    h->ntiles2 = h->tx2 * ((ny + FP_TILE - 1) / FP_TILE);
    h->pstride = std::max(h->ntiles, h->ntiles2);
    h->maxiter = maxiter;
    h->tol = tol;
    const size_t N = (size_t)h->n * nmem;
    // a linear SPD preconditioner (Jacobi alone) needs no more than the
    // one-term recurrence; the network's nonlinear one gains from a deeper one
    h->m = net ? FP_MAX_TRUNC : 1;
    h->net_every = net ? 2 : 1;  // network every other iteration (smoothing alone in between)
    cudaError_t e;
    if ((e = cudaMalloc(&h->vec, sizeof(double) * FP_NVEC * N)) != cudaSuccess ||
        (e = cudaMalloc(&h->ring, sizeof(double) * 2 * (h->m + 1) * N)) != cudaSuccess ||
        (e = cudaMalloc(&h->wd32, sizeof(float) * N)) != cudaSuccess ||
        (e = cudaMalloc(&h->xin, sizeof(float) * 2 * (size_t)h->nc * nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->out, sizeof(float) * (size_t)h->nc * nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->part, sizeof(double) * FP_NSLOT * (size_t)h->pstride * nmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_pre, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)fp_smem_bytes(FP_MAX_SMOOTH))) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_post, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)fp_smem_bytes(FP_MAX_SMOOTH))) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_pre, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_post, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
        (e = cudaMalloc(&h->acc, sizeof(double) * std::max(4, nmem))) != cudaSuccess ||
        (e = cudaMalloc(&h->rslots, sizeof(double) * FP_RES_BLOCKS * (size_t)nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->rcount, sizeof(unsigned int) * nmem)) != cudaSuccess ||
        (e = cudaMemset(h->rcount, 0, sizeof(unsigned int) * nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->st, sizeof(FpState) * nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->bar, sizeof(BarrierState))) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_loop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)fp_smem_bytes(FP_MAX_SMOOTH))) != cudaSuccess ||
        (e = cudaFuncSetAttribute(k_fp_loop, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
        (e = cudaMalloc(&h->hist, sizeof(double) * (maxiter + 1) * (size_t)nmem)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev0)) != cudaSuccess || (e = cudaEventCreate(&h->ev1)) != cudaSuccess) {
        cudaGetLastError();
        set_error("FPCG buffers: %s", cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    // the device loop's grid: every block co-resident (its grid barriers)
    DeviceInfo di;
    int per_sm = 0;
    if (current_device_info(&di) == CFM_OK &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fp_loop, CG_TILE,
                                                      fp_smem_bytes(std::max(smooth, 1))) == cudaSuccess &&
        per_sm > 0)
        h->loop_grid = std::min(std::max(h->ntiles, h->ntiles2), per_sm * di.num_sms);
    cudaGetLastError();
    return CFM_OK;
}

}  // namespace

extern "C" {

int cfm_fpcg_create(const cfm_stencil *S, const double *k_host, cfm_unet *net, int smooth,
                    int maxiter, double tol, cfm_fpcg **out) {
    clear_error();
    CFM_ARG_CHECK(S && k_host && out, "null argument");
    *out = nullptr;
    int dims, nx, ny, nz;
    stencil_shape(S, &dims, &nx, &ny, &nz);
    CFM_ARG_CHECK(dims == 2, "the learned preconditioner is 2D");
    CFM_ARG_CHECK(tol > 0 && maxiter > 0, "tol, maxiter");
    CFM_ARG_CHECK(smooth >= 0 && smooth <= FP_MAX_SMOOTH, "smooth must be in [0, 8]");
    const int f = net ? net->coarsen : 1;
    if (net) {
        int H = 0, W = 0;
        unet_shape(net->u, &H, &W);
        CFM_ARG_CHECK((long long)H * f == ny && (long long)W * f == nx,
                      "the network's grid must be the stencil's divided by the factor it was trained with");
        CFM_ARG_CHECK(smooth == net->smooth, "smooth must equal the sweeps the network was trained with");
    }
    cfm_fpcg *h = new cfm_fpcg();
    h->S = S;
    int st = fp_setup(h, nx, ny, f, net, smooth, maxiter, tol, 1);
    if (st) {
        cfm_fpcg_destroy(h);
        return st;
    }
    const size_t n = h->n;
    double *kd = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&kd, sizeof(double) * n)) != cudaSuccess ||
        (e = cudaMemcpy(kd, k_host, sizeof(double) * n, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFree(kd);
        cfm_fpcg_destroy(h);
        CFM_CUDA_TRY(e);
    }
    k_log_coarse<<<256, 256>>>(kd, h->xin, nx, ny, f);
    k_fp_wd<<<256, 256>>>(stencil_coeffs32(S) + 3 * n, h->wd32, h->n);
    e = cudaDeviceSynchronize();
    cudaFree(kd);
    if (e != cudaSuccess) {
        cfm_fpcg_destroy(h);
        CFM_CUDA_TRY(e);
    }
    *out = h;
    return CFM_OK;
}

int cfm_fpcg_create_batch(int nmem, const int *nx, const int *ny, const double *const *k_host, cfm_unet *net,
                          int smooth, int maxiter, double tol, cfm_fpcg **out) {
    clear_error();
    CFM_ARG_CHECK(out && nx && ny && k_host && nmem >= 1, "arguments");
    *out = nullptr;
    CFM_ARG_CHECK(tol > 0 && maxiter > 0, "tol, maxiter");
    CFM_ARG_CHECK(smooth >= 0 && smooth <= FP_MAX_SMOOTH, "smooth must be in [0, 8]");
    const int f = net ? net->coarsen : 1;
    int FX = 0, FY = 0;  // the frame
    if (net) {
        int H = 0, W = 0;
        unet_shape(net->u, &H, &W);
        FX = W * f;
        FY = H * f;
        CFM_ARG_CHECK(smooth == net->smooth, "smooth must equal the sweeps the network was trained with");
    } else {
        for (int m = 0; m < nmem; ++m) {
            FX = std::max(FX, nx[m]);
            FY = std::max(FY, ny[m]);
        }
    }
    for (int m = 0; m < nmem; ++m) {
        CFM_ARG_CHECK(k_host[m] && nx[m] >= 1 && ny[m] >= 1, "member arguments");
        CFM_ARG_CHECK(nx[m] <= FX && ny[m] <= FY, "a member is larger than the network's grid times its factor");
    }
    CFM_ARG_CHECK((double)FX * FY * nmem < 1.5e9, "batch too large");
    cfm_fpcg *h = new cfm_fpcg();
    int st = fp_setup(h, FX, FY, f, net, smooth, maxiter, tol, nmem);
    if (st) {
        cfm_fpcg_destroy(h);
        return st;
    }
    // Frame coefficients: each member at the frame's origin, its faces to
    // the padding zero and the padding's diagonal 1, so the padding is an
    // identity block that stays at zero (b = 0 there and the network's
    // correction is kept inside the member).  FP32 copies rounded to nearest.
    const size_t n = h->n, N = n * nmem;
    std::vector<double> c(4 * N, 0.0);
    std::vector<float> xin(2 * (size_t)h->nc * nmem, 0.f);
    std::vector<double> cells(nmem);
    h->ext_h.resize(nmem);
    for (int m = 0; m < nmem; ++m) {
        const int mx = nx[m], my = ny[m];
        const size_t mn = (size_t)mx * my;
        std::vector<double> we(mn), wn(mn), wt(mn), dg(mn);
        if ((st = cfm_varcoef_coeffs(2, mx, my, 1, k_host[m], we.data(), wn.data(), wt.data(), dg.data()))) {
            cfm_fpcg_destroy(h);
            return st;
        }
        double *fwe = c.data() + m * n, *fwn = c.data() + N + m * n, *fdg = c.data() + 3 * N + m * n;
        for (size_t i = 0; i < n; ++i) fdg[i] = 1.0;
        for (int y = 0; y < my; ++y)
            for (int x = 0; x < mx; ++x) {
                const size_t src = (size_t)y * mx + x, dst = (size_t)y * FX + x;
                fwe[dst] = x < mx - 1 ? we[src] : 0.0;
                fwn[dst] = y < my - 1 ? wn[src] : 0.0;
                fdg[dst] = dg[src];
            }
        // the network's second channel: block-mean log k (k = 1 in the padding)
        const int ncx = FX / f;
        for (int ic = 0; ic < h->nc; ++ic) {
            const int cx = ic % ncx, cy = ic / ncx;
            double sum = 0;
            for (int dy = 0; dy < f; ++dy)
                for (int dx = 0; dx < f; ++dx) {
                    const int gx = cx * f + dx, gy = cy * f + dy;
                    if (gx < mx && gy < my) sum += std::log(k_host[m][(size_t)gy * mx + gx]);
                }
            xin[2 * ((size_t)m * h->nc + ic) + 1] = (float)(sum / (f * f));
        }
        h->ext_h[m] = make_int2(mx, my);
        cells[m] = (double)mn;
    }
    std::vector<float> c32(4 * N);
    for (size_t i = 0; i < 4 * N; ++i) c32[i] = (float)c[i];
    cudaError_t e;
    if ((e = cudaMalloc(&h->c64b, sizeof(double) * 4 * N)) != cudaSuccess ||
        (e = cudaMalloc(&h->c32b, sizeof(float) * 4 * N)) != cudaSuccess ||
        (e = cudaMalloc(&h->ext, sizeof(int2) * nmem)) != cudaSuccess ||
        (e = cudaMalloc(&h->cells, sizeof(double) * nmem)) != cudaSuccess ||
        (e = cudaMemcpy(h->c64b, c.data(), sizeof(double) * 4 * N, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->c32b, c32.data(), sizeof(float) * 4 * N, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->ext, h->ext_h.data(), sizeof(int2) * nmem, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->cells, cells.data(), sizeof(double) * nmem, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(h->xin, xin.data(), sizeof(float) * xin.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaGetLastError();
        set_error("batch upload: %s", cudaGetErrorString(e));
        cfm_fpcg_destroy(h);
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    k_fp_wd<<<1024, 256>>>(h->c32b + 3 * N, h->wd32, (int)N);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
        cfm_fpcg_destroy(h);
        CFM_CUDA_TRY(e);
    }
    *out = h;
    return CFM_OK;
}

void cfm_fpcg_destroy(cfm_fpcg *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    cudaFree(h->vec);
    cudaFree(h->ring);
    cudaFree(h->wd32);
    cudaFree(h->xin);
    cudaFree(h->out);
    cudaFree(h->part);
    cudaFree(h->acc);
    cudaFree(h->rslots);
    cudaFree(h->rcount);
    cudaFree(h->vec32);
    cudaFree(h->ring32);
    cudaFree(h->xm);
    cudaFree(h->c64b);
    cudaFree(h->c32b);
    cudaFree(h->ext);
    cudaFree(h->cells);
    cudaFree(h->st);
    cudaFree(h->bar);
    cudaFree(h->hist);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int cfm_fpcg_set_truncation(cfm_fpcg *h, int m) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(m >= 1 && m <= FP_MAX_TRUNC, "truncation must be in [1, 8]");
    if (m == h->m) return CFM_OK;
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    double *ring = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&ring, sizeof(double) * 2 * (m + 1) * (size_t)h->n * h->nmem));
    cudaFree(h->ring);
    h->ring = ring;
    if (h->mixed) {
        const int st = alloc_ring32(h, m);
        if (st) return st;
    }
    h->m = m;
    // the captured iteration graph holds the old ring: build it again
    drop_graph(h);
    return CFM_OK;
}

int cfm_fpcg_set_device_loop(cfm_fpcg *h, int on) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(on == 0 || on == 1, "on must be 0 or 1");
    if (on == h->loop) return CFM_OK;
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->loop = on;
    drop_graph(h);  // the captured iteration is the other form
    return CFM_OK;
}

int cfm_fpcg_set_precision(cfm_fpcg *h, int precision, double delta) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(precision == CFM_FP64 || precision == CFM_FP32, "precision");
    CFM_ARG_CHECK(delta > 0.0 && delta < 1.0, "delta must be in (0, 1)");
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const int mixed = precision == CFM_FP32;
    if (mixed && !h->vec32) {
        const size_t n = (size_t)h->n * h->nmem;
        float *v = nullptr;
        double *xm = nullptr;
        CFM_CUDA_TRY(cudaMalloc(&v, sizeof(float) * 4 * n));
        if (cudaMalloc(&xm, sizeof(double) * 2 * n) != cudaSuccess) {
            cudaFree(v);
            cudaGetLastError();
            set_error("mixed-precision buffers: out of device memory");
            return CFM_OUT_OF_MEMORY;
        }
        h->vec32 = v;
        h->xm = xm;
        const int st = alloc_ring32(h, h->m);
        if (st) return st;
    }
    if (mixed != h->mixed || delta != h->delta) drop_graph(h);
    h->mixed = mixed;
    h->delta = delta;
    return CFM_OK;
}

int cfm_fpcg_reliable_updates(const cfm_fpcg *h) { return h ? h->last_updates : -1; }

int cfm_fpcg_set_network_period(cfm_fpcg *h, int every) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(every >= 1 && every <= 8, "period must be in [1, 8]");
    if (every == h->net_every) return CFM_OK;
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->net_every = every;
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->exec = nullptr;
    h->graph = nullptr;
    h->conditional = false;
    return CFM_OK;
}

int cfm_fpcg_solve(cfm_fpcg *h, const double *b_host, double *x_host, cfm_stats *stats) {
    const cfm::NvtxRange nvtx_range("cfm_fpcg_solve");
    clear_error();
    CFM_ARG_CHECK(h && b_host && x_host, "null argument");
    CFM_ARG_CHECK(h->nmem == 1, "a batch handle: use cfm_fpcg_solve_batch");
    const size_t n = h->n;
    FpArgs a = fp_args(h);
    cudaStream_t s = h->stream;
    double *b = h->vec + 3 * n, *t = h->vec + 4 * n, *d = h->vec + 5 * n;
    CFM_CUDA_TRY(cudaMemcpyAsync(b, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (h->net) CFM_CUDA_TRY(cudaMemsetAsync(unet_err(h->net->u), 0, sizeof(int), s));
    int st = 0;
    if (!h->exec) {
        // eager warm-up of the network (kernel attributes) before capture
        if (h->net && (st = unet_forward(h->net->u, 1, h->xin, h->out, s))) return st;
        CFM_CUDA_TRY(cudaStreamSynchronize(s));
        if ((st = build_graph(h))) return st;
    }
    {  // the device loop's barrier: counters and error word cleared, wait budget set
        BarrierState bs{};
        bs.timeout_ns = barrier_timeout_ns();
        CFM_CUDA_TRY(cudaMemcpyAsync(h->bar, &bs, sizeof(bs), cudaMemcpyHostToDevice, s));
    }
    int launches = 0;
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, s));
    if (h->mixed)
        k_fpm_init<<<h->ntiles, CG_TILE, 0, s>>>(a, h->tol);
    else
        k_fp_init<<<h->ntiles, CG_TILE, 0, s>>>(a, h->tol);
    CFM_CUDA_TRY(cudaGetLastError());
    if ((st = fp_precond_dir(h, a, 0, 0, 0))) return st;
    launches += 2;
    FpState hs{};
    if (h->conditional) {
        CFM_CUDA_TRY(cudaGraphLaunch(h->exec, s));
        ++launches;
    } else {
        for (;;) {
            CFM_CUDA_TRY(cudaGraphLaunch(h->exec, s));
            ++launches;
            CFM_CUDA_TRY(cudaMemcpyAsync(&hs, h->st, sizeof(hs), cudaMemcpyDeviceToHost, s));
            CFM_CUDA_TRY(cudaStreamSynchronize(s));
            if (hs.done) break;
        }
    }
    if (h->mixed) {  // x = FP64 iterate + the FP32 steps since the last update
        k_fpm_finish<<<256, 256, 0, s>>>(a, h->st);
        CFM_CUDA_TRY(cudaGetLastError());
        ++launches;
    }
    CFM_CUDA_TRY(cudaMemcpyAsync(&hs, h->st, sizeof(hs), cudaMemcpyDeviceToHost, s));
    // FP64 true residual; plain persistent CG finishes if FPCG fell short
    CFM_CUDA_TRY(cudaMemsetAsync(h->acc, 0, sizeof(double) * 2, s));
    k_fp_true_res<<<FP_RES_BLOCKS, 256, 0, s>>>(a.op, h->n, b, a.x, t, h->acc, h->rslots, h->rcount);
    double acc[2] = {0, 0};
    CFM_CUDA_TRY(cudaMemcpyAsync(acc, h->acc, sizeof(double), cudaMemcpyDeviceToHost, s));
    CFM_CUDA_TRY(cudaStreamSynchronize(s));
    if (h->net && (st = unet_check_err(h->net->u))) return st;
    {
        BarrierState bs{};
        CFM_CUDA_TRY(cudaMemcpy(&bs, h->bar, sizeof(bs), cudaMemcpyDeviceToHost));
        if (bs.error) {
            set_error("FPCG device loop: grid barrier %d timed out", bs.where);
            return CFM_BARRIER_TIMEOUT;
        }
    }
    h->last_k = hs.k;
    h->last_updates = h->mixed ? hs.updates : 0;
    const double bnorm = hs.target / h->tol;
    double tnorm = std::sqrt(acc[0]);
    int fallback = 0;
    long long fb_iters = 0;
    int status = CFM_OK;
    if (!(tnorm <= h->tol * bnorm)) {
        fallback = 1;
        const double tol2 = h->tol * bnorm / tnorm;
        status = cg_stencil_snapshots(h->S, t, d, tol2, 50000, nullptr, 1, 0, &fb_iters, nullptr, s);
        if (status != CFM_OK && status != CFM_NOT_CONVERGED) return status;
        k_axpy_inplace<<<256, 256, 0, s>>>(a.x, d, h->n);
        CFM_CUDA_TRY(cudaMemsetAsync(h->acc, 0, sizeof(double), s));
        k_fp_true_res<<<FP_RES_BLOCKS, 256, 0, s>>>(a.op, h->n, b, a.x, t, h->acc, h->rslots, h->rcount);
        CFM_CUDA_TRY(cudaMemcpyAsync(acc, h->acc, sizeof(double), cudaMemcpyDeviceToHost, s));
        launches += 3;
    }
    CFM_CUDA_TRY(cudaMemcpyAsync(x_host, a.x, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CFM_CUDA_TRY(cudaEventRecord(h->ev1, s));
    CFM_CUDA_TRY(cudaEventSynchronize(h->ev1));
    float ms = 0;
    CFM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    tnorm = std::sqrt(acc[0]);
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->seconds = ms * 1e-3;
        stats->iterations = hs.k + fb_iters;
        stats->residual = tnorm / bnorm;
        stats->h2d_bytes = 8.0 * n;
        stats->d2h_bytes = 8.0 * n;
        stats->launches = launches;
        stats->refinements = fallback;
        stats->status = status;
        stats->lups = (double)hs.k;  // FPCG iterations alone (before any fallback)
    }
    return status;
}

// |r| before each preconditioner application of the last solve (k + 1 values).
int cfm_fpcg_solve_batch(cfm_fpcg *h, const double *const *b_host, double *const *x_host, long long *iters,
                         int *status, double *relres, cfm_stats *stats) {
    const cfm::NvtxRange nvtx_range("cfm_fpcg_solve_batch");
    clear_error();
    CFM_ARG_CHECK(h && b_host && x_host, "null argument");
    const int M = h->nmem;
    for (int m = 0; m < M; ++m) CFM_ARG_CHECK(b_host[m] && x_host[m], "null member vector");
    const size_t n = h->n, N = n * M;
    FpArgs a = fp_args(h);
    cudaStream_t s = h->stream;
    double *b = h->vec + 3 * N, *t = h->vec + 4 * N;
    // right-hand sides into the frames (zero in the padding)
    std::vector<double> frame(N, 0.0);
    for (int m = 0; m < M; ++m) {
        const int mx = h->ext_h[m].x, my = h->ext_h[m].y;
        for (int y = 0; y < my; ++y)
            std::memcpy(frame.data() + m * n + (size_t)y * h->nx, b_host[m] + (size_t)y * mx, sizeof(double) * mx);
    }
    CFM_CUDA_TRY(cudaMemcpyAsync(b, frame.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
    if (h->net) CFM_CUDA_TRY(cudaMemsetAsync(unet_err(h->net->u), 0, sizeof(int), s));
    int st = 0;
    if (!h->exec) {
        if (h->net && (st = unet_forward(h->net->u, 1, h->xin, h->out, s))) return st;
        CFM_CUDA_TRY(cudaStreamSynchronize(s));
        if ((st = build_graph(h))) return st;
    }
    int launches = 0;
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, s));
    if (h->mixed)
        k_fpm_init<<<dim3(h->ntiles, M), CG_TILE, 0, s>>>(a, h->tol);
    else
        k_fp_init<<<dim3(h->ntiles, M), CG_TILE, 0, s>>>(a, h->tol);
    CFM_CUDA_TRY(cudaGetLastError());
    if ((st = fp_precond_dir(h, a, 0, 0, 0))) return st;
    launches += 2;
    std::vector<FpState> hs(M);
    if (h->conditional) {
        CFM_CUDA_TRY(cudaGraphLaunch(h->exec, s));
        ++launches;
    } else {
        for (;;) {
            CFM_CUDA_TRY(cudaGraphLaunch(h->exec, s));
            ++launches;
            CFM_CUDA_TRY(cudaMemcpyAsync(hs.data(), h->st, sizeof(FpState) * M, cudaMemcpyDeviceToHost, s));
            CFM_CUDA_TRY(cudaStreamSynchronize(s));
            bool open = false;
            for (const FpState &q : hs) open |= q.done == 0;
            if (!open) break;
        }
    }
    if (h->mixed) {
        k_fpm_finish<<<1024, 256, 0, s>>>(a, h->st);
        CFM_CUDA_TRY(cudaGetLastError());
        ++launches;
    }
    k_fpb_true_res<<<dim3(FP_RES_BLOCKS, M), 256, 0, s>>>(a, t, h->acc, h->rslots, h->rcount);
    CFM_CUDA_TRY(cudaGetLastError());
    ++launches;
    CFM_CUDA_TRY(cudaMemcpyAsync(frame.data(), a.x, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    std::vector<double> acc(M);
    CFM_CUDA_TRY(cudaMemcpyAsync(acc.data(), h->acc, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
    CFM_CUDA_TRY(cudaMemcpyAsync(hs.data(), h->st, sizeof(FpState) * M, cudaMemcpyDeviceToHost, s));
    CFM_CUDA_TRY(cudaEventRecord(h->ev1, s));
    CFM_CUDA_TRY(cudaEventSynchronize(h->ev1));
    if (h->net && (st = unet_check_err(h->net->u))) return st;
    float ms = 0;
    CFM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    int worst = CFM_OK, updates = 0;
    long long kmax = 0;
    for (int m = 0; m < M; ++m) {
        const int mx = h->ext_h[m].x, my = h->ext_h[m].y;
        for (int y = 0; y < my; ++y)
            std::memcpy(x_host[m] + (size_t)y * mx, frame.data() + m * n + (size_t)y * h->nx, sizeof(double) * mx);
        const double bnorm = hs[m].target / h->tol;
        const double rr = bnorm > 0 ? std::sqrt(acc[m]) / bnorm : std::sqrt(acc[m]);
        const int sm = (hs[m].done == 1 && rr <= h->tol) ? CFM_OK : CFM_NOT_CONVERGED;
        if (iters) iters[m] = hs[m].k;
        if (status) status[m] = sm;
        if (relres) relres[m] = rr;
        if (sm != CFM_OK) worst = sm;
        kmax = std::max(kmax, hs[m].k);
        updates += hs[m].updates;
    }
    h->last_updates = h->mixed ? updates : 0;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->seconds = ms * 1e-3;
        stats->iterations = kmax;
        stats->h2d_bytes = 8.0 * N;
        stats->d2h_bytes = 8.0 * N;
        stats->launches = launches;
        stats->status = worst;
        stats->refinements = h->last_updates;
    }
    if (worst != CFM_OK) set_error("some members did not reach the tolerance");
    return worst;
}

int cfm_fpcg_history(cfm_fpcg *h, double *out, long long max_n, long long *n_out) {
    CFM_ARG_CHECK(h && out && n_out, "null argument");
    const long long n = std::min(max_n, std::min(h->last_k + 1, h->maxiter + 1));
    CFM_CUDA_TRY(cudaMemcpy(out, h->hist, sizeof(double) * n, cudaMemcpyDeviceToHost));
    *n_out = n;
    return CFM_OK;
}

// Training data from plain CG runs (fresh seeds seed0 .. seed0 + nsys - 1)
// and `epochs` passes of Adam over it; loss values of the first and last
// epoch (mean per-sample 1 - cos^2) are returned.
int cfm_unet_train_varcoef(cfm_unet *net, int nsys, int snaps, unsigned long long seed0, int epochs,
                           int batch, float lr, int smooth, int coarsen, double *loss_first,
                           double *loss_last, double *data_seconds, double *train_seconds) {
    const NvtxRange nvtx_range("cfm_unet_train_varcoef");
    clear_error();
    CFM_ARG_CHECK(net && nsys >= 1 && snaps >= 1 && epochs >= 1, "arguments");
    CFM_ARG_CHECK(smooth >= 0 && smooth <= FP_MAX_SMOOTH, "smooth must be in [0, 8]");
    CFM_ARG_CHECK(coarsen == 1 || coarsen == 2, "coarsen must be 1 or 2");
    CFM_ARG_CHECK(batch >= 1 && batch <= net->maxB, "batch must be in [1, max_batch]");
    net->smooth = smooth;
    net->coarsen = coarsen;
    UNetImpl *u = net->u;
    int Hc = 0, Wc = 0;
    unet_shape(u, &Hc, &Wc);
    const int f = coarsen, H = Hc * f, W = Wc * f;  // the systems' grid
    const int n = H * W, nc = Hc * Wc;
    const int per = snaps + 1;  // + the initial residual b
    const long long N = (long long)nsys * per;
    cudaStream_t s = nullptr;
    CFM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct Guard {
        std::vector<void *> p;
        cudaStream_t s;
        ~Guard() {
            if (s) cudaStreamSynchronize(s);
            for (void *q : p) cudaFree(q);
            if (s) cudaStreamDestroy(s);
        }
    } g{{}, s};
    auto alloc = [&](auto **ptr, size_t bytes) -> cudaError_t {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(bytes, 1));
        if (e == cudaSuccess) g.p.push_back(q);
        *ptr = static_cast<std::remove_reference_t<decltype(**ptr)> *>(q);
        return e;
    };
    float *xin_all, *r1_all, *coef_all, *gf, *az_b, *out_b, *dout_b;
    double *bd, *xs, *snap, *r, *e, *acc, *sums, *lossd, *er_all;
    long long *ids_d;
    CFM_CUDA_TRY(alloc(&xin_all, sizeof(float) * 2 * (size_t)nc * N));
    CFM_CUDA_TRY(alloc(&r1_all, sizeof(float) * (size_t)n * N));
    CFM_CUDA_TRY(alloc(&coef_all, sizeof(float) * 3 * (size_t)n * nsys));
    CFM_CUDA_TRY(alloc(&er_all, sizeof(double) * N));
    CFM_CUDA_TRY(alloc(&ids_d, sizeof(long long) * batch));
    CFM_CUDA_TRY(alloc(&gf, sizeof(float) * nc));
    CFM_CUDA_TRY(alloc(&bd, sizeof(double) * n));
    CFM_CUDA_TRY(alloc(&xs, sizeof(double) * n));
    CFM_CUDA_TRY(alloc(&snap, sizeof(double) * (size_t)n * snaps));
    CFM_CUDA_TRY(alloc(&r, sizeof(double) * n));
    CFM_CUDA_TRY(alloc(&e, sizeof(double) * n));
    CFM_CUDA_TRY(alloc(&acc, sizeof(double) * 2));
    double *zs, *r1s;
    CFM_CUDA_TRY(alloc(&zs, sizeof(double) * 2 * n));
    CFM_CUDA_TRY(alloc(&r1s, sizeof(double) * n));
    CFM_CUDA_TRY(alloc(&az_b, sizeof(float) * (size_t)n * batch));
    CFM_CUDA_TRY(alloc(&out_b, sizeof(float) * (size_t)nc * batch));
    CFM_CUDA_TRY(alloc(&dout_b, sizeof(float) * (size_t)nc * batch));
    CFM_CUDA_TRY(alloc(&sums, sizeof(double) * 2 * batch));
    CFM_CUDA_TRY(alloc(&lossd, sizeof(double)));
    // block sums of the data pairs (256 blocks x 2), the loss dots (64 blocks
    // x 2 per batch element) and the batch loss, added in a fixed order; and
    // their counters: [0] pairs, [1] loss, [2 + b] dots of element b
    constexpr int DATA_BLOCKS = 256, LOSS_BLOCKS = 64;
    double *dslots;
    unsigned int *dcount;
    CFM_CUDA_TRY(alloc(&dslots, sizeof(double) * std::max<size_t>(2 * DATA_BLOCKS, 2 * (size_t)LOSS_BLOCKS * batch)));
    CFM_CUDA_TRY(alloc(&dcount, sizeof(unsigned int) * (2 + (size_t)batch)));
    CFM_CUDA_TRY(cudaMemsetAsync(dcount, 0, sizeof(unsigned int) * (2 + (size_t)batch), s));
    double *lslots;
    CFM_CUDA_TRY(alloc(&lslots, sizeof(double) * batch));
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<double> kh(n), fh(n);
    std::vector<float> gh(nc);
    int st = 0;
    nvtxRangePushA("training data: plain-CG pairs");
    struct PopAtExit {
        bool on = true;
        void pop() {
            if (on) nvtxRangePop();
            on = false;
        }
        ~PopAtExit() { pop(); }
    } data_range;
    for (int sy = 0; sy < nsys; ++sy) {
        if ((st = cfm_varcoef_problem(2, W, H, 1, seed0 + sy, kh.data(), fh.data()))) return st;
        for (int ic = 0; ic < nc; ++ic) {  // block-mean log k on the network's grid
            const int cx = ic % Wc, cy = ic / Wc;
            double sum = 0;
            for (int dy = 0; dy < f; ++dy)
                for (int dx = 0; dx < f; ++dx) sum += std::log(kh[(size_t)(cy * f + dy) * W + cx * f + dx]);
            gh[ic] = (float)(sum / (f * f));
        }
        cfm_stencil *S = nullptr;
        if ((st = cfm_stencil_create(2, W, H, 1, kh.data(), &S))) return st;
        CFM_CUDA_TRY(cudaMemcpyAsync(bd, fh.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
        CFM_CUDA_TRY(cudaMemcpyAsync(gf, gh.data(), sizeof(float) * nc, cudaMemcpyHostToDevice, s));
        long long K = 0;
        st = cg_stencil_snapshots(S, bd, xs, 1e-10, 200000, nullptr, 1, 0, &K, nullptr, s);
        int taken = 0;
        if (st == CFM_OK) {
            // snapshots spread over the iterations that reach ~1e-7
            const int every = (int)std::max(1LL, (long long)(0.8 * K) / (snaps + 1));
            st = cg_stencil_snapshots(S, bd, r, 1e-10, (int)(every * (long long)snaps), snap, every,
                                      snaps, nullptr, &taken, s);
            if (st == CFM_NOT_CONVERGED) st = CFM_OK;
        }
        cfm_stencil_destroy(S);
        if (st) return st;
        cfm_stencil *S2 = nullptr;
        if ((st = cfm_stencil_create(2, W, H, 1, kh.data(), &S2))) return st;
        const StencilOp<2> o2 = op2(S2);
        const float *c32 = stencil_coeffs32(S2);  // we | wn | wt | dg
        float *cdst = coef_all + (size_t)sy * 3 * n;
        CFM_CUDA_TRY(cudaMemcpyAsync(cdst, c32, sizeof(float) * 2 * n, cudaMemcpyDeviceToDevice, s));
        CFM_CUDA_TRY(cudaMemcpyAsync(cdst + 2 * (size_t)n, c32 + 3 * (size_t)n, sizeof(float) * n,
                                     cudaMemcpyDeviceToDevice, s));
        for (int j = 0; j < per; ++j) {
            const double *xj = j == 0 ? nullptr : snap + (size_t)(std::min(j, std::max(taken, 1)) - 1) * n;
            const size_t idx = (size_t)sy * per + j;
            CFM_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * 2, s));
            k_pair<<<DATA_BLOCKS, 256, 0, s>>>(o2, n, bd, xs, xj, r, e, acc, dslots, dcount);
            const double *rin = r;
            if (smooth > 0) {
                double *zz[2] = {zs, zs + n};
                const double *cur = nullptr;
                for (int q = 0; q < smooth; ++q) {
                    k_data_jacobi<<<256, 256, 0, s>>>(o2, n, r, cur, zz[q & 1]);
                    cur = zz[q & 1];
                }
                CFM_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * 2, s));
                k_data_smoothed<<<DATA_BLOCKS, 256, 0, s>>>(o2, n, cur, r, e, r1s, acc, dslots, dcount);
                rin = r1s;
            }
            k_pair_store<<<256, 256, 0, s>>>(W, H, f, rin, gf, acc, xin_all + idx * 2 * nc,
                                             r1_all + idx * n, er_all + idx);
        }
        CFM_CUDA_TRY(cudaStreamSynchronize(s));
        cfm_stencil_destroy(S2);
    }
    const auto t1 = std::chrono::steady_clock::now();
    data_range.pop();
    // validation: one held-out system solved by FPCG with the network as it
    // trains; the parameters of the fastest solve are kept
    struct Val {
        cfm_stencil *S = nullptr;
        cfm_fpcg *fp = nullptr;
        std::vector<double> k, b, x;
        std::vector<float> best;
        double best_s = 1e300;
        long long best_it = -1;
        int best_ep = -1;
        ~Val() {
            cfm_fpcg_destroy(fp);
            cfm_stencil_destroy(S);
        }
    } val;
    net->val_best_epoch = -1;
    net->val_best_ms = 0.0;
    if (net->val_every > 0) {
        val.k.resize(n);
        val.b.resize(n);
        val.x.resize(n);
        if ((st = cfm_varcoef_problem(2, W, H, 1, net->val_seed, val.k.data(), val.b.data()))) return st;
        if ((st = cfm_stencil_create(2, W, H, 1, val.k.data(), &val.S))) return st;
        if ((st = cfm_fpcg_create(val.S, val.k.data(), net, smooth, 20000, 1e-8, &val.fp))) return st;
    }
    // The kept checkpoint is the one whose validation solve took the fewest
    // iterations (ties: the earlier epoch): a count, not a time, so the
    // choice, like the training, is the same on every run.
    auto validate = [&](int ep) -> int {
        CFM_CUDA_TRY(cudaStreamSynchronize(s));
        double secs = 1e300;
        long long iters = -1;
        for (int rep = 0; rep < 2; ++rep) {  // the first solve also instantiates the graph
            cfm_stats vs{};
            const int e2 = cfm_fpcg_solve(val.fp, val.b.data(), val.x.data(), &vs);
            if (e2 == CFM_OK) {
                secs = std::min(secs, vs.seconds);
                iters = vs.iterations;
            } else if (e2 != CFM_NOT_CONVERGED && e2 != CFM_BREAKDOWN) {
                return e2;
            }
        }
        if (iters >= 0 && (val.best_ep < 0 || iters < val.best_it)) {
            val.best_it = iters;
            val.best_s = secs;
            val.best_ep = ep;
            val.best.resize(unet_params(u));
            const int e3 = cfm_unet_get_params(net, val.best.data());
            if (e3) return e3;
        }
        return CFM_OK;
    };
    // training
    const NvtxRange train_range("training: Adam epochs");
    std::mt19937_64 rng(seed0 ^ 0x5eedULL);
    std::vector<long long> order(N);
    for (long long i = 0; i < N; ++i) order[i] = i;
    double first = 0, last = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        double ep_loss = 0;
        int nb = 0;
        CFM_CUDA_TRY(cudaMemsetAsync(lossd, 0, sizeof(double), s));
        for (long long i0 = 0; i0 + batch <= N; i0 += batch) {
            for (int bi = 0; bi < batch; ++bi) {
                const long long id = order[i0 + bi];
                CFM_CUDA_TRY(cudaMemcpyAsync(net->xin + (size_t)bi * 2 * nc, xin_all + (size_t)id * 2 * nc,
                                             sizeof(float) * 2 * nc, cudaMemcpyDeviceToDevice, s));
            }
            // the ids are read by the loss kernels queued below: copy synchronously
            CFM_CUDA_TRY(cudaStreamSynchronize(s));
            CFM_CUDA_TRY(cudaMemcpy(ids_d, &order[i0], sizeof(long long) * batch, cudaMemcpyHostToDevice));
            if ((st = unet_forward(u, batch, net->xin, out_b, s))) return st;
            CFM_CUDA_TRY(cudaMemsetAsync(sums, 0, sizeof(double) * 2 * batch, s));
            k_loss_anorm_dots<<<dim3(LOSS_BLOCKS, batch), 256, 0, s>>>(out_b, r1_all, coef_all, ids_d, per,
                                                                      W, H, f, az_b, sums, dslots,
                                                                      dcount + 2);
            k_loss_anorm_grad<<<dim3(LOSS_BLOCKS, batch), 256, 0, s>>>(az_b, r1_all, sums, er_all, ids_d, W,
                                                                      H, f, batch, dout_b, lossd, lslots,
                                                                      dcount + 1);
            CFM_CUDA_TRY(cudaMemsetAsync(unet_grad(u), 0, unet_params(u) * sizeof(float), s));
            if ((st = unet_backward(u, batch, net->xin, dout_b, s))) return st;
            if ((st = unet_adam(u, lr, 1.0f, s))) return st;
            ++nb;
        }
        double l = 0;
        CFM_CUDA_TRY(cudaMemcpyAsync(&l, lossd, sizeof(double), cudaMemcpyDeviceToHost, s));
        CFM_CUDA_TRY(cudaStreamSynchronize(s));
        if ((st = unet_check_err(u))) return st;
        ep_loss = nb ? l / nb : 0;
        if (ep == 0) first = ep_loss;
        last = ep_loss;
        if (net->val_every > 0 && ((ep + 1) % net->val_every == 0 || ep + 1 == epochs))
            if ((st = validate(ep + 1))) return st;
    }
    if (val.best_ep >= 0) {
        if ((st = cfm_unet_set_params(net, val.best.data()))) return st;
        net->val_best_epoch = val.best_ep;
        net->val_best_ms = val.best_s * 1e3;
    }
    const auto t2 = std::chrono::steady_clock::now();
    if (loss_first) *loss_first = first;
    if (loss_last) *loss_last = last;
    if (data_seconds) *data_seconds = std::chrono::duration<double>(t1 - t0).count();
    if (train_seconds) *train_seconds = std::chrono::duration<double>(t2 - t1).count();
    return CFM_OK;
}

int cfm_unet_set_validation(cfm_unet *net, unsigned long long seed, int every) {
    clear_error();
    CFM_ARG_CHECK(net && every >= 0, "arguments");
    net->val_seed = seed;
    net->val_every = every;
    return CFM_OK;
}

int cfm_unet_validation(const cfm_unet *net, int *best_epoch, double *best_ms) {
    CFM_ARG_CHECK(net, "null argument");
    if (best_epoch) *best_epoch = net->val_best_epoch;
    if (best_ms) *best_ms = net->val_best_ms;
    return CFM_OK;
}

}  // extern "C"
