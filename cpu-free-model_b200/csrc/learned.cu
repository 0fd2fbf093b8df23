// The learned preconditioner's U-Net on one B200: forward, backward and an
// Adam step.  No reference counterpart (the reference has no learned or
// tensor-core code).
//
// Architecture (levels L0..L3 at H/2^l x W/2^l, 32/64/128/256 channels):
//   h0 = relu(cin(x))  2->32 | h1 = relu(e1(pool h0)) | h2 = relu(e2(pool h1))
//   h3 = relu(e3(pool h2)) | g3 = relu(d3 h3) | g2 = relu(d2(up g3 + h2))
//   g1 = relu(d1(up g2 + h1)) | g0 = relu(d0(up g1 + h0)) | out = cout(g0) 32->1
// 3x3 convolutions with bias, zero padding; pool = 2x2 mean, up = nearest.
// The seven wide convolutions (e1..d0) and their backward passes run on the
// tensor cores (tc_conv.cuh): BF16 activations and weights, FP32
// accumulation.  cin (2 input channels) and cout (1 output channel) are too
// thin for a 128 x N MMA tile and run on the CUDA cores in FP32.
// Parameters: one flat FP32 vector (master copy, Adam state beside it), per
// layer weight [9][Cout][Cin] (tap = 3 dy + dx) then bias [Cout]; BF16 copies
// of the tensor-core weights and their tap-flipped transposes (the weights
// of the backward-data convolution) are refreshed after every update.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cfm_internal.h"
#include "learned_internal.h"
#include "unet_internal.h"
#include "unet_layers.cuh"

namespace cfm {

using bf16 = __nv_bfloat16;

const UNetLayer UNET_LAYERS[UNET_NLAYERS] = {
    {"cin", 2, 32, 0, false},    {"e1", 32, 64, 1, true},    {"e2", 64, 128, 2, true},
    {"e3", 128, 256, 3, true},   {"d3", 256, 128, 3, true},  {"d2", 128, 64, 2, true},
    {"d1", 64, 32, 1, true},     {"d0", 32, 32, 0, true},    {"cout", 32, 1, 0, false},
};

size_t unet_num_params() {
    size_t n = 0;
    for (const auto &l : UNET_LAYERS) n += 9 * (size_t)l.co * l.ci + l.co;
    return n;
}

// ----------------------------------------------------------------- kernels
namespace {

using unet_dev::CIN_SPAN;
using unet_dev::COUT_SPAN;
using unet_dev::load8;
using unet_dev::PXB;
using unet_dev::store8;

// Capacity (floats) of a net's block-partials buffer for the thin layers'
// and the biases' gradients: blocks x entries of the largest such launch.
constexpr long long GPART_FLOATS = 1LL << 18;

// h0 = relu(cin(x)) (unet_dev::cin_block); grid (ceil(W / (PXB CIN_SPAN 32)), H, B).
__global__ void __launch_bounds__(256, 2) k_cin_fwd(const float *x, const float *w, const float *b,
                                                    bf16 *h0, int H, int W, UNetInputScale in_scale) {
    pdl_enter();
    unet_dev::cin_block(x, w, b, h0, H, W, in_scale, blockIdx.x, blockIdx.y, blockIdx.z);
}

// out = cout(g0) (unet_dev::cout_block); grid (ceil(W / (PXB COUT_SPAN 64)), H, B).
__global__ void __launch_bounds__(256, 2) k_cout_fwd(const bf16 *g0, const float *w, const float *b,
                                                     float *out, int H, int W) {
    pdl_enter();
    unet_dev::cout_block(g0, w, b, out, H, W, blockIdx.x, blockIdx.y, blockIdx.z);
}

// dz = (sum_t w[t][c] dout[q - s_t]) * (g0[q][c] > 0): the backward-data of cout
// fused with the ReLU mask of g0.
__global__ void k_cout_bwd(const float *dout, const float *w, const bf16 *g0, bf16 *dz, int B, int H,
                           int W) {
    __shared__ float sw[288];
    for (int i = threadIdx.x; i < 288; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
    const long long P = (long long)B * H * W;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
         p += (long long)gridDim.x * blockDim.x) {
        const int xx = (int)(p % W), yy = (int)((p / W) % H);
        const long long img0 = p - (long long)yy * W - xx;
        float d[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int y = yy - (t / 3 - 1), xq = xx - (t % 3 - 1);
            d[t] = (y >= 0 && y < H && xq >= 0 && xq < W) ? dout[img0 + (long long)y * W + xq] : 0.f;
        }
#pragma unroll
        for (int c = 0; c < 32; c += 8) {
            float m[8], o[8];
            load8(g0 + p * 32 + c, m);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float acc = 0.f;
#pragma unroll
                for (int t = 0; t < 9; ++t) acc += sw[t * 32 + c + j] * d[t];
                o[j] = m[j] > 0.f ? acc : 0.f;
            }
            store8(dz + p * 32 + c, o);
        }
    }
}

// Cross-block sums that come out the same on every run: a kernel stores its
// blocks' partial sums part[b][e] (nb blocks, ne entries) and
// k_partials_reduce adds them in a fixed order.  A 256-thread block takes 16
// entries and splits the nb blocks into 16 chunks, one thread per (entry,
// chunk); a chunk is summed with four accumulators (block b into b mod 4,
// combined as (a0 + a1) + (a2 + a3)), then the 16 chunks are added in order.
// The totals go to dw[e] (e < nw) and db[e - nw] (+=).
constexpr int PR_ENTRIES = 16, PR_CHUNKS = 16;
__global__ void __launch_bounds__(PR_ENTRIES * PR_CHUNKS)
    k_partials_reduce(const float *part, int nb, int ne, int nw, float *dw, float *db) {
    __shared__ float sc[PR_ENTRIES * PR_CHUNKS];
    const int el = threadIdx.x % PR_ENTRIES, q = threadIdx.x / PR_ENTRIES;
    const int e = blockIdx.x * PR_ENTRIES + el;
    float v = 0.f;
    if (e < ne) {
        const int b0 = (int)((long long)q * nb / PR_CHUNKS), b1 = (int)((long long)(q + 1) * nb / PR_CHUNKS);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        int b = b0;
        for (; b + 3 < b1; b += 4) {
            a0 += part[(size_t)b * ne + e];
            a1 += part[(size_t)(b + 1) * ne + e];
            a2 += part[(size_t)(b + 2) * ne + e];
            a3 += part[(size_t)(b + 3) * ne + e];
        }
        for (; b < b1; ++b) a0 += part[(size_t)b * ne + e];
        v = (a0 + a1) + (a2 + a3);
    }
    sc[threadIdx.x] = v;
    __syncthreads();
    if (q == 0 && e < ne) {
        float t = 0.f;
        for (int c = 0; c < PR_CHUNKS; ++c) t += sc[c * PR_ENTRIES + el];
        if (e < nw) dw[e] += t;
        else db[e - nw] += t;
    }
}

int partials_reduce(const float *part, int nb, int ne, int nw, float *dw, float *db, cudaStream_t s) {
    k_partials_reduce<<<(ne + PR_ENTRIES - 1) / PR_ENTRIES, PR_ENTRIES * PR_CHUNKS, 0, s>>>(part, nb, ne, nw, dw,
                                                                                             db);
    CFM_CUDA_TRY(cudaGetLastError());
    return CFM_OK;
}

// N consecutive values of a BF16 or FP32 row as FP32 (one 8-byte load for
// four BF16 or two FP32; the address is a multiple of N elements).
template <typename T, int N>
__device__ __forceinline__ void load_row(const T *src, float *v) {
    if constexpr (std::is_same<T, float>::value && N == 2) {
        const float2 q = *reinterpret_cast<const float2 *>(src);
        v[0] = q.x, v[1] = q.y;
    } else if constexpr (std::is_same<T, bf16>::value && N == 4) {
        const uint2 q = *reinterpret_cast<const uint2 *>(src);
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
        const float2 a = __bfloat1622float2(h[0]), b = __bfloat1622float2(h[1]);
        v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = (float)src[i];
    }
}

// Weight and bias gradient of a thin layer (the 2 -> 32 input layer and
// the 32 -> 1 output layer, FP32 on the CUDA cores):
//   dw[t][co][ci] = sum_p g[p][co] in[p + s_t][ci],   db[co] = sum_p g[p][co]
// with `in` zero outside the image.  Warp w of a block owns CO_T output and
// CI_T input channels (group w of (CO_N / CO_T) x (CI_N / CI_T) = 8) for
// all nine taps; lane l takes pixels l, l + 32, ... of the block's chunk of
// 32-pixel groups (each inside one row: W is a multiple of 32).  The lanes'
// sums are combined by a fixed xor butterfly and the block's sums go to
// part[block][entry], entry (t CO_N + co) CI_N + ci, then 9 CO_N CI_N + co
// for the bias (k_partials_reduce adds the blocks up).
template <typename GT, typename IT, int CO_N, int CI_N, int CO_T, int CI_T>
__global__ void __launch_bounds__(256, 2)
    k_thin_wgrad(const GT *g, const IT *in, int H, int W, long long ngroups, long long gchunk, float *part) {
    static_assert((CO_N / CO_T) * (CI_N / CI_T) == 8, "eight warps, one channel group each");
    constexpr int NW = 9 * CO_N * CI_N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int co0 = (warp / (CI_N / CI_T)) * CO_T, ci0 = (warp % (CI_N / CI_T)) * CI_T;
    float acc[9][CO_T][CI_T], bacc[CO_T];
#pragma unroll
    for (int t = 0; t < 9; ++t)
#pragma unroll
        for (int i = 0; i < CO_T; ++i)
#pragma unroll
            for (int j = 0; j < CI_T; ++j) acc[t][i][j] = 0.f;
#pragma unroll
    for (int i = 0; i < CO_T; ++i) bacc[i] = 0.f;
    const long long g0 = blockIdx.x * gchunk, g1 = min(ngroups, g0 + gchunk);
    const int gpr = W / 32;
    int x = (int)(g0 % gpr) * 32 + lane;
    int y = (int)((g0 / gpr) % H);
    for (long long gi = g0; gi < g1; ++gi) {
        const long long p = gi * 32 + lane;
        float gv[CO_T];
        load_row<GT, CO_T>(g + p * CO_N + co0, gv);
#pragma unroll
        for (int i = 0; i < CO_T; ++i) bacc[i] += gv[i];
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int sy = t / 3 - 1, sx = t % 3 - 1;
            float iv[CI_T];
            if (y + sy >= 0 && y + sy < H && x + sx >= 0 && x + sx < W) {
                load_row<IT, CI_T>(in + (p + (long long)sy * W + sx) * CI_N + ci0, iv);
            } else {
#pragma unroll
                for (int j = 0; j < CI_T; ++j) iv[j] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < CO_T; ++i)
#pragma unroll
                for (int j = 0; j < CI_T; ++j) acc[t][i][j] = __fmaf_rn(gv[i], iv[j], acc[t][i][j]);
        }
        x += 32;  // the whole group moves to the next row together
        if (x >= W) {
            x -= W;
            if (++y == H) y = 0;
        }
    }
#pragma unroll
    for (int t = 0; t < 9; ++t)
#pragma unroll
        for (int i = 0; i < CO_T; ++i)
#pragma unroll
            for (int j = 0; j < CI_T; ++j)
#pragma unroll
                for (int o = 16; o; o >>= 1) acc[t][i][j] += __shfl_xor_sync(0xffffffffu, acc[t][i][j], o);
#pragma unroll
    for (int i = 0; i < CO_T; ++i)
#pragma unroll
        for (int o = 16; o; o >>= 1) bacc[i] += __shfl_xor_sync(0xffffffffu, bacc[i], o);
    if (lane == 0) {
        float *dst = part + (size_t)blockIdx.x * (NW + CO_N);
#pragma unroll
        for (int t = 0; t < 9; ++t)
#pragma unroll
            for (int i = 0; i < CO_T; ++i)
#pragma unroll
                for (int j = 0; j < CI_T; ++j) dst[(t * CO_N + co0 + i) * CI_N + ci0 + j] = acc[t][i][j];
        if (ci0 == 0)
#pragma unroll
            for (int i = 0; i < CO_T; ++i) dst[NW + co0 + i] = bacc[i];
    }
}

// Launch of k_thin_wgrad over all B H W pixels (about two blocks per SM)
// and the fixed-order sum of its blocks into dw and db.
template <typename GT, typename IT, int CO_N, int CI_N, int CO_T, int CI_T>
int thin_wgrad(const GT *g, const IT *in, int B, int H, int W, float *part, float *dw, float *db,
               cudaStream_t s) {
    CFM_ARG_CHECK(W % 32 == 0, "thin-layer gradient: W must be a multiple of 32");
    const long long ngroups = (long long)B * H * W / 32;
    const long long gchunk = std::max(1LL, (ngroups + 2 * 148 - 1) / (2 * 148));
    const int blocks = (int)((ngroups + gchunk - 1) / gchunk);
    constexpr int NE = 9 * CO_N * CI_N + CO_N;
    CFM_ARG_CHECK((long long)blocks * NE <= GPART_FLOATS, "thin-gradient partials");
    k_thin_wgrad<GT, IT, CO_N, CI_N, CO_T, CI_T><<<blocks, 256, 0, s>>>(g, in, H, W, ngroups, gchunk, part);
    CFM_CUDA_TRY(cudaGetLastError());
    return partials_reduce(part, blocks, NE, 9 * CO_N * CI_N, dw, db, s);
}

// 2x2 mean pool (unet_dev::pool_block); grid (items of a pooled row / blockDim, h, B).
template <int C>
__global__ void k_pool(const bf16 *in, bf16 *out, int h, int w) {
    pdl_enter();
    unet_dev::pool_block<C>(in, out, h, w, blockIdx.x, blockIdx.y, blockIdx.z);
}

// u = up(g) + skip (unet_dev::up_add_block); grid (items of a fine row / blockDim, 2h, B).
template <int C>
__global__ void k_up_add(const bf16 *g, const bf16 *skip, bf16 *u, int h, int w) {
    pdl_enter();
    unet_dev::up_add_block<C>(g, skip, u, h, w, blockIdx.x, blockIdx.y, blockIdx.z);
}

// dz[coarse] = (sum of the 2x2 fine gradients) * (act[coarse] > 0).
__global__ void k_down_sum_mask(const bf16 *d, const bf16 *act, bf16 *dz, int B, int h, int w, int C) {
    const long long n = (long long)B * h * w * (C / 8);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(e % (C / 8)) * 8;
        const long long pix = e / (C / 8);
        const int x = (int)(pix % w), y = (int)((pix / w) % h), img = (int)(pix / ((long long)w * h));
        const long long W2 = 2LL * w;
        const long long base = (((long long)img * 2 * h + 2 * y) * W2 + 2 * x) * C + c8;
        float a[8], b[8], c[8], dd[8], m[8], o[8];
        load8(d + base, a);
        load8(d + base + C, b);
        load8(d + base + W2 * C, c);
        load8(d + base + W2 * C + C, dd);
        load8(act + pix * C + c8, m);
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = m[j] > 0.f ? ((a[j] + b[j]) + c[j]) + dd[j] : 0.f;
        store8(dz + pix * C + c8, o);
    }
}

// dz[fine] = (dskip[fine] + 0.25 dpool[coarse]) * (act[fine] > 0): the skip
// path plus the adjoint of the 2x2 mean pool, through the ReLU of act.
__global__ void k_skip_pool_mask(const bf16 *dskip, const bf16 *dpool, const bf16 *act, bf16 *dz,
                                 int B, int h, int w, int C) {
    const long long n = (long long)B * 4 * h * w * (C / 8);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(e % (C / 8)) * 8;
        const long long pix = e / (C / 8);
        const int x = (int)(pix % (2 * w)), y = (int)((pix / (2 * w)) % (2 * h));
        const int img = (int)(pix / (4LL * h * w));
        const long long cp = ((long long)img * h + y / 2) * w + x / 2;
        float a[8], b[8], m[8];
        load8(dskip + pix * C + c8, a);
        load8(dpool + cp * C + c8, b);
        load8(act + pix * C + c8, m);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = m[j] > 0.f ? a[j] + 0.25f * b[j] : 0.f;
        store8(dz + pix * C + c8, a);
    }
}

// db[c] += sum_p dz[p][c] (NHWC BF16): block-local sums over a chunk of
// pixels into part[block][c] (k_partials_reduce adds them up).
__global__ void k_bias_grad(const bf16 *dz, long long P, int C, long long chunk, float *part) {
    extern __shared__ float red[];  // [blockDim.x]
    const int c = threadIdx.x % C, lane_p = threadIdx.x / C, np = blockDim.x / C;
    const long long p0 = blockIdx.x * chunk, p1 = min(P, p0 + chunk);
    float acc = 0.f;
    for (long long p = p0 + lane_p; p < p1; p += np) acc += __bfloat162float(dz[p * C + c]);
    red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < C) {
        float s = 0.f;
        for (int j = 0; j < np; ++j) s += red[j * C + threadIdx.x];
        part[(size_t)blockIdx.x * C + threadIdx.x] = s;
    }
}

// BF16 weights [9][co][ci] and their tap-flipped transposes [9][ci][co]
// (w'[8 - t][ci][co] = w[t][co][ci]) from the FP32 master copy.
__global__ void k_weights_bf16(const float *w, bf16 *wb, bf16 *wt, int co, int ci) {
    const int n = 9 * co * ci;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int t = e / (co * ci), o = (e / ci) % co, i = e % ci;
        const bf16 v = __float2bfloat16_rn(w[e]);
        wb[e] = v;
        wt[((size_t)(8 - t) * ci + i) * co + o] = v;
    }
}

// Adam (Kingma & Ba 2015) with bias correction; `scale` multiplies the raw
// gradient first (e.g. 1 / batch).
__global__ void k_adam(float *theta, const float *g, float *m, float *v, size_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2, float scale) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i] * scale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int grid_for(long long n, int per = 256) {
    return (int)std::max(1LL, std::min((n + per - 1) / per, 148LL * 16));
}

// One block row per image row: (ceil(items / 256), rows, images).
dim3 row_grid(int items, int rows, int images) { return dim3((items + 255) / 256, rows, images); }

}  // namespace

// --------------------------------------------------------------- the net
struct UNetBuffers {
    // forward
    bf16 *h0, *p1, *h1, *p2, *h2, *p3, *h3, *g3, *u2, *g2, *u1, *g1, *u0, *g0;
    // backward
    bf16 *dz_g0, *du0, *dz_g1, *du1, *dz_g2, *du2, *dz_g3, *dz_h3, *dp3, *dz_h2, *dp2, *dz_h1,
        *dp1, *dz_h0;
};

struct UNetImpl {
    int H = 0, W = 0, maxB = 0;
    size_t nparams = 0;
    size_t woff[UNET_NLAYERS], boff[UNET_NLAYERS];
    float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    bf16 *wb[UNET_NLAYERS] = {}, *wt[UNET_NLAYERS] = {};
    UNetBuffers a{};
    int *err = nullptr;
    float *ws = nullptr;  // split-K workspace of the convolutions and weight gradients
    long long ws_floats = 0;
    // per-block partial sums of the thin layers' and the biases' gradients,
    // added in block order by the last block (deterministic), and the
    // arrival counters of those reductions
    float *gpart = nullptr;
    // grid barrier of the persistent forward, and which forward runs
    // (CFM_UNET_FORWARD_AUTO / _LAYERS / _PERSISTENT)
    UfBarrier *bar = nullptr;
    int fwd_mode = 0;
    long long adam_t = 0;
    std::vector<void *> allocs;
};

namespace {

template <class T>
int dalloc(UNetImpl *u, T **p, size_t count) {
    void *q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("unet allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;
    }
    u->allocs.push_back(q);
    *p = static_cast<T *>(q);
    return CFM_OK;
}

}  // namespace

// Clears the persistent forward's barrier (counters, error word) and sets
// its wait budget.
int unet_reset_barrier(UNetImpl *u) {
    UfBarrier b{};
    b.timeout_ns = barrier_timeout_ns();
    CFM_CUDA_TRY(cudaMemcpy(u->bar, &b, sizeof(b), cudaMemcpyHostToDevice));
    return CFM_OK;
}

int unet_create(int H, int W, int maxB, UNetImpl **out) {
    CFM_ARG_CHECK(out, "null argument");
    *out = nullptr;
    CFM_ARG_CHECK(H >= 8 && H % 8 == 0, "H must be a multiple of 8");
    CFM_ARG_CHECK(W >= 256 && W % 256 == 0, "W must be a multiple of 256");
    CFM_ARG_CHECK(maxB >= 1, "max batch");
    UNetImpl *u = new UNetImpl();
    u->H = H;
    u->W = W;
    u->maxB = maxB;
    size_t o = 0;
    for (int l = 0; l < UNET_NLAYERS; ++l) {
        u->woff[l] = o;
        o += 9 * (size_t)UNET_LAYERS[l].co * UNET_LAYERS[l].ci;
        u->boff[l] = o;
        o += UNET_LAYERS[l].co;
    }
    u->nparams = o;
    const size_t L0 = (size_t)maxB * H * W, L1 = L0 / 4, L2 = L0 / 16, L3 = L0 / 64;
    UNetBuffers &a = u->a;
    int st = 0;
    auto A = [&](bf16 **p, size_t n) {
        if (!st) st = dalloc(u, p, n);
    };
    if (!st) st = dalloc(u, &u->theta, o);
    if (!st) st = dalloc(u, &u->grad, o);
    if (!st) st = dalloc(u, &u->m, o);
    if (!st) st = dalloc(u, &u->v, o);
    if (!st) st = dalloc(u, &u->err, 1);
    if (!st) st = dalloc(u, &u->bar, 1);
    // the split-K workspace: the forward split's TC_WS_FLOATS or the widest
    // weight-gradient split of any tensor-core layer at the largest batch
    u->ws_floats = TC_WS_FLOATS;
    {
        DeviceInfo di;
        if (!st) st = current_device_info(&di);
        for (int l = 0; !st && l < UNET_NLAYERS; ++l)
            if (UNET_LAYERS[l].tc) {
                const int lv = UNET_LAYERS[l].level;
                u->ws_floats = std::max(u->ws_floats,
                                        tc_wgrad_ws_floats(maxB, H >> lv, W >> lv, UNET_LAYERS[l].ci,
                                                           UNET_LAYERS[l].co, di.num_sms));
            }
    }
    if (!st) st = dalloc(u, &u->ws, (size_t)u->ws_floats);
    if (!st) st = dalloc(u, &u->gpart, (size_t)GPART_FLOATS);
    for (int l = 0; l < UNET_NLAYERS; ++l)
        if (UNET_LAYERS[l].tc) {
            const size_t n = 9 * (size_t)UNET_LAYERS[l].co * UNET_LAYERS[l].ci;
            A(&u->wb[l], n);
            A(&u->wt[l], n);
        }
    A(&a.h0, L0 * 32);  A(&a.p1, L1 * 32);  A(&a.h1, L1 * 64);  A(&a.p2, L2 * 64);
    A(&a.h2, L2 * 128); A(&a.p3, L3 * 128); A(&a.h3, L3 * 256); A(&a.g3, L3 * 128);
    A(&a.u2, L2 * 128); A(&a.g2, L2 * 64);  A(&a.u1, L1 * 64);  A(&a.g1, L1 * 32);
    A(&a.u0, L0 * 32);  A(&a.g0, L0 * 32);
    A(&a.dz_g0, L0 * 32); A(&a.du0, L0 * 32); A(&a.dz_g1, L1 * 32); A(&a.du1, L1 * 64);
    A(&a.dz_g2, L2 * 64); A(&a.du2, L2 * 128); A(&a.dz_g3, L3 * 128); A(&a.dz_h3, L3 * 256);
    A(&a.dp3, L3 * 128); A(&a.dz_h2, L2 * 128); A(&a.dp2, L2 * 64); A(&a.dz_h1, L1 * 64);
    A(&a.dp1, L1 * 32); A(&a.dz_h0, L0 * 32);
    if (st) {
        unet_destroy(u);
        return st;
    }
    cudaError_t e;
    if ((e = cudaMemset(u->theta, 0, o * 4)) != cudaSuccess ||
        (e = cudaMemset(u->m, 0, o * 4)) != cudaSuccess ||
        (e = cudaMemset(u->v, 0, o * 4)) != cudaSuccess ||
        (e = cudaMemset(u->err, 0, sizeof(int))) != cudaSuccess) {
        unet_destroy(u);
        CFM_CUDA_TRY(e);
    }
    if ((st = unet_reset_barrier(u))) {
        unet_destroy(u);
        return st;
    }
    *out = u;
    return CFM_OK;
}

void unet_destroy(UNetImpl *u) {
    if (!u) return;
    cudaDeviceSynchronize();
    for (void *p : u->allocs) cudaFree(p);
    delete u;
}

size_t unet_params(const UNetImpl *u) { return u->nparams; }
void unet_shape(const UNetImpl *u, int *H, int *W) {
    *H = u->H;
    *W = u->W;
}
float *unet_theta(UNetImpl *u) { return u->theta; }
float *unet_grad(UNetImpl *u) { return u->grad; }
int *unet_err(UNetImpl *u) { return u->err; }

int unet_refresh_weights(UNetImpl *u, cudaStream_t s) {
    for (int l = 0; l < UNET_NLAYERS; ++l) {
        const UNetLayer &L = UNET_LAYERS[l];
        if (!L.tc) continue;
        const int n = 9 * L.co * L.ci;
        k_weights_bf16<<<grid_for(n), 256, 0, s>>>(u->theta + u->woff[l], u->wb[l], u->wt[l], L.co,
                                                    L.ci);
        CFM_CUDA_TRY(cudaGetLastError());
    }
    return CFM_OK;
}

namespace {

int conv_fwd(UNetImpl *u, int l, const bf16 *x, bf16 *out, int B, int h, int w, cudaStream_t s) {
    const UNetLayer &L = UNET_LAYERS[l];
    ConvArgs c{x, u->wb[l], u->theta + u->boff[l], nullptr, out, u->err, B, h, w, L.ci, L.co, 1};
    c.ws = u->ws;
    c.ws_floats = TC_WS_FLOATS;
    return tc_conv_fwd(c, s);
}

// dx = conv_T(dz) (weights flipped / transposed), optionally masked.
int conv_bwd_data(UNetImpl *u, int l, const bf16 *dz, const bf16 *mask, bf16 *dx, int B, int h,
                  int w, cudaStream_t s) {
    const UNetLayer &L = UNET_LAYERS[l];
    ConvArgs c{dz, u->wt[l], nullptr, mask, dx, u->err, B, h, w, L.co, L.ci, 0};
    c.ws = u->ws;
    c.ws_floats = TC_WS_FLOATS;
    return tc_conv_fwd(c, s);
}

// dW += wgrad(x, dz), db += sum dz.
int conv_bwd_weights(UNetImpl *u, int l, const bf16 *x, const bf16 *dz, int B, int h, int w,
                     cudaStream_t s) {
    const UNetLayer &L = UNET_LAYERS[l];
    WgradArgs g{x, dz, u->grad + u->woff[l], u->err, B, h, w, L.ci, L.co, u->ws, u->ws_floats};
    int st = tc_conv_wgrad(g, s);
    if (st) return st;
    const long long P = (long long)B * h * w;
    const int threads = 256;
    const long long chunk = std::max(64LL, (P + 4 * 148 - 1) / (4 * 148));
    const int blocks = (int)((P + chunk - 1) / chunk);
    CFM_ARG_CHECK((long long)blocks * L.co <= GPART_FLOATS, "bias-gradient partials");
    k_bias_grad<<<blocks, threads, threads * sizeof(float), s>>>(dz, P, L.co, chunk, u->gpart);
    CFM_CUDA_TRY(cudaGetLastError());
    return partials_reduce(u->gpart, blocks, L.co, 0, nullptr, u->grad + u->boff[l], s);
}

}  // namespace

// The persistent forward (one cooperative launch, unet_fused.cuh) with the
// per-layer kernels' buffers and plans.
int forward_persistent(UNetImpl *u, int B, const float *x, float *out, cudaStream_t s,
                       const UNetInputScale *in_scale) {
    UNetBuffers &a = u->a;
    const int H = u->H, W = u->W;
    FusedForwardArgs f{};
    f.B = B;
    f.H = H;
    f.W = W;
    f.x = x;
    f.out = out;
    f.in_scale = in_scale ? *in_scale : UNetInputScale{};
    f.cin_w = u->theta + u->woff[0];
    f.cin_b = u->theta + u->boff[0];
    f.cout_w = u->theta + u->woff[8];
    f.cout_b = u->theta + u->boff[8];
    f.h0 = a.h0;
    f.p1 = a.p1;
    f.h1 = a.h1;
    f.p2 = a.p2;
    f.h2 = a.h2;
    f.p3 = a.p3;
    const bf16 *in[7] = {a.p1, a.p2, a.p3, a.h3, a.u2, a.u1, a.u0};
    bf16 *o[7] = {a.h1, a.h2, a.h3, a.g3, a.g2, a.g1, a.g0};
    for (int l = 0; l < 7; ++l) {
        const UNetLayer &L = UNET_LAYERS[l + 1];
        const int h = H >> L.level, w = W >> L.level;
        f.conv[l] = ConvArgs{in[l], u->wb[l + 1], u->theta + u->boff[l + 1], nullptr, o[l], u->err, B, h, w,
                             L.ci, L.co, 1};
        f.conv[l].ws = u->ws;
        f.conv[l].ws_floats = TC_WS_FLOATS;
    }
    f.skip[3] = a.h2;  // d3: u2 = up(g3) + h2
    f.uout[3] = a.u2;
    f.skip[4] = a.h1;  // d2: u1 = up(g2) + h1
    f.uout[4] = a.u1;
    f.skip[5] = a.h0;  // d1: u0 = up(g1) + h0
    f.uout[5] = a.u0;
    f.bar = u->bar;
    return unet_forward_fused(f, s);
}

int unet_forward(UNetImpl *u, int B, const float *x, float *out, cudaStream_t s,
                 const UNetInputScale *in_scale) {
    CFM_ARG_CHECK(B >= 1 && B <= u->maxB, "batch");
    UNetBuffers &a = u->a;
    const int H = u->H, W = u->W;
    int st;
    if (u->fwd_mode == CFM_UNET_FORWARD_PERSISTENT) return forward_persistent(u, B, x, out, s, in_scale);
    CFM_CUDA_TRY(launch_pdl(k_cin_fwd, dim3((W + PXB * CIN_SPAN * 32 - 1) / (PXB * CIN_SPAN * 32), H, B), dim3(256),
                            0, s, x, (const float *)(u->theta + u->woff[0]),
                            (const float *)(u->theta + u->boff[0]), a.h0, H, W,
                            in_scale ? *in_scale : UNetInputScale{}));
    int h = H, w = W;
    CFM_CUDA_TRY(launch_pdl(k_pool<32>, row_grid(w / 2 * 4, h / 2, B), dim3(256), 0, s, (const bf16 *)a.h0,
                            a.p1, h / 2, w / 2));
    h /= 2, w /= 2;
    if ((st = conv_fwd(u, 1, a.p1, a.h1, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_pool<64>, row_grid(w / 2 * 8, h / 2, B), dim3(256), 0, s, (const bf16 *)a.h1,
                            a.p2, h / 2, w / 2));
    h /= 2, w /= 2;
    if ((st = conv_fwd(u, 2, a.p2, a.h2, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_pool<128>, row_grid(w / 2 * 16, h / 2, B), dim3(256), 0, s,
                            (const bf16 *)a.h2, a.p3, h / 2, w / 2));
    h /= 2, w /= 2;
    if ((st = conv_fwd(u, 3, a.p3, a.h3, B, h, w, s))) return st;
    if ((st = conv_fwd(u, 4, a.h3, a.g3, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_up_add<128>, row_grid(2 * w * 16, 2 * h, B), dim3(256), 0, s,
                            (const bf16 *)a.g3, (const bf16 *)a.h2, a.u2, h, w));
    h *= 2, w *= 2;
    if ((st = conv_fwd(u, 5, a.u2, a.g2, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_up_add<64>, row_grid(2 * w * 8, 2 * h, B), dim3(256), 0, s,
                            (const bf16 *)a.g2, (const bf16 *)a.h1, a.u1, h, w));
    h *= 2, w *= 2;
    if ((st = conv_fwd(u, 6, a.u1, a.g1, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_up_add<32>, row_grid(2 * w * 4, 2 * h, B), dim3(256), 0, s,
                            (const bf16 *)a.g1, (const bf16 *)a.h0, a.u0, h, w));
    h *= 2, w *= 2;
    if ((st = conv_fwd(u, 7, a.u0, a.g0, B, h, w, s))) return st;
    CFM_CUDA_TRY(launch_pdl(k_cout_fwd, dim3((W + PXB * COUT_SPAN * 64 - 1) / (PXB * COUT_SPAN * 64), H, B),
                            dim3(256), 0, s, (const bf16 *)a.g0, (const float *)(u->theta + u->woff[8]),
                            (const float *)(u->theta + u->boff[8]), out, H, W));
    return CFM_OK;
}

// Gradient of sum(out * dout) into u->grad (accumulated; zero it first for a
// fresh gradient).  Needs the activations of the unet_forward just before.
int unet_backward(UNetImpl *u, int B, const float *x, const float *dout, cudaStream_t s) {
    UNetBuffers &a = u->a;
    const int H = u->H, W = u->W;
    const long long P0 = (long long)B * H * W;
    int st;
    const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
    // cout
    {
        if ((st = thin_wgrad<float, bf16, 1, 32, 1, 4>(dout, a.g0, B, H, W, u->gpart, u->grad + u->woff[8],
                                                       u->grad + u->boff[8], s)))
            return st;
        k_cout_bwd<<<grid_for(P0), 256, 0, s>>>(dout, u->theta + u->woff[8], a.g0, a.dz_g0, B, H, W);
        CFM_CUDA_TRY(cudaGetLastError());
    }
    // d0 @L0
    if ((st = conv_bwd_weights(u, 7, a.u0, a.dz_g0, B, H, W, s))) return st;
    if ((st = conv_bwd_data(u, 7, a.dz_g0, nullptr, a.du0, B, H, W, s))) return st;
    k_down_sum_mask<<<grid_for(P0 / 4 * 4), 256, 0, s>>>(a.du0, a.g1, a.dz_g1, B, H1, W1, 32);
    // d1 @L1
    if ((st = conv_bwd_weights(u, 6, a.u1, a.dz_g1, B, H1, W1, s))) return st;
    if ((st = conv_bwd_data(u, 6, a.dz_g1, nullptr, a.du1, B, H1, W1, s))) return st;
    k_down_sum_mask<<<grid_for(P0 / 16 * 8), 256, 0, s>>>(a.du1, a.g2, a.dz_g2, B, H2, W2, 64);
    // d2 @L2
    if ((st = conv_bwd_weights(u, 5, a.u2, a.dz_g2, B, H2, W2, s))) return st;
    if ((st = conv_bwd_data(u, 5, a.dz_g2, nullptr, a.du2, B, H2, W2, s))) return st;
    k_down_sum_mask<<<grid_for(P0 / 64 * 16), 256, 0, s>>>(a.du2, a.g3, a.dz_g3, B, H3, W3, 128);
    // d3 @L3 (its input h3 is a ReLU output: mask the data gradient)
    if ((st = conv_bwd_weights(u, 4, a.h3, a.dz_g3, B, H3, W3, s))) return st;
    if ((st = conv_bwd_data(u, 4, a.dz_g3, a.h3, a.dz_h3, B, H3, W3, s))) return st;
    // e3 @L3
    if ((st = conv_bwd_weights(u, 3, a.p3, a.dz_h3, B, H3, W3, s))) return st;
    if ((st = conv_bwd_data(u, 3, a.dz_h3, nullptr, a.dp3, B, H3, W3, s))) return st;
    k_skip_pool_mask<<<grid_for(P0 / 16 * 16), 256, 0, s>>>(a.du2, a.dp3, a.h2, a.dz_h2, B, H3, W3, 128);
    // e2 @L2
    if ((st = conv_bwd_weights(u, 2, a.p2, a.dz_h2, B, H2, W2, s))) return st;
    if ((st = conv_bwd_data(u, 2, a.dz_h2, nullptr, a.dp2, B, H2, W2, s))) return st;
    k_skip_pool_mask<<<grid_for(P0 / 4 * 8), 256, 0, s>>>(a.du1, a.dp2, a.h1, a.dz_h1, B, H2, W2, 64);
    // e1 @L1
    if ((st = conv_bwd_weights(u, 1, a.p1, a.dz_h1, B, H1, W1, s))) return st;
    if ((st = conv_bwd_data(u, 1, a.dz_h1, nullptr, a.dp1, B, H1, W1, s))) return st;
    k_skip_pool_mask<<<grid_for(P0 * 4), 256, 0, s>>>(a.du0, a.dp1, a.h0, a.dz_h0, B, H1, W1, 32);
    // cin
    {
        if ((st = thin_wgrad<bf16, float, 32, 2, 4, 2>(a.dz_h0, x, B, H, W, u->gpart, u->grad + u->woff[0],
                                                       u->grad + u->boff[0], s)))
            return st;
    }
    return CFM_OK;
}

int unet_adam(UNetImpl *u, float lr, float scale, cudaStream_t s) {
    ++u->adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)u->adam_t), c2 = 1.f - std::pow(b2, (float)u->adam_t);
    k_adam<<<grid_for((long long)u->nparams), 256, 0, s>>>(u->theta, u->grad, u->m, u->v, u->nparams,
                                                            lr, b1, b2, 1e-8f, c1, c2, scale);
    CFM_CUDA_TRY(cudaGetLastError());
    return unet_refresh_weights(u, s);
}

int unet_check_err(UNetImpl *u) {
    int herr = 0;
    UfBarrier b{};
    CFM_CUDA_TRY(cudaMemcpy(&herr, u->err, sizeof(int), cudaMemcpyDeviceToHost));
    CFM_CUDA_TRY(cudaMemcpy(&b, u->bar, sizeof(b), cudaMemcpyDeviceToHost));
    if (herr) {
        set_error("unet: a tensor-core pipeline wait timed out (site %d)", herr);
        return CFM_BARRIER_TIMEOUT;
    }
    if (b.error) {
        set_error("unet: a grid barrier of the persistent forward timed out (barrier %d)", b.where);
        unet_reset_barrier(u);
        return CFM_BARRIER_TIMEOUT;
    }
    return CFM_OK;
}

}  // namespace cfm

// ------------------------------------------------------------------ C ABI
using namespace cfm;


extern "C" {

long long cfm_unet_num_params(void) { return (long long)unet_num_params(); }

int cfm_unet_create(int H, int W, int max_batch, unsigned long long seed, cfm_unet **out) {
    clear_error();
    CFM_ARG_CHECK(out, "null argument");
    *out = nullptr;
    UNetImpl *u = nullptr;
    int st = unet_create(H, W, max_batch, &u);
    if (st) return st;
    cfm_unet *h = new cfm_unet();
    h->u = u;
    h->maxB = max_batch;
    const size_t P = (size_t)max_batch * H * W;
    cudaError_t e;
    if ((e = cudaMalloc(&h->xin, P * 2 * 4)) != cudaSuccess ||
        (e = cudaMalloc(&h->out, P * 4)) != cudaSuccess ||
        (e = cudaMalloc(&h->dout, P * 4)) != cudaSuccess) {
        cfm_unet_destroy(h);
        CFM_CUDA_TRY(e);
    }
    // He-normal weights (std sqrt(2 / (9 Cin))), zero biases; the output layer
    // starts 10x smaller.
    std::vector<float> theta(u->nparams, 0.f);
    std::vector<double> z;
    size_t o = 0;
    for (int l = 0; l < UNET_NLAYERS; ++l) {
        const UNetLayer &L = UNET_LAYERS[l];
        const size_t n = 9 * (size_t)L.co * L.ci;
        z.resize(n);
        cfm_normal(seed, 100u + l, (long long)n, z.data());
        const double sd = std::sqrt(2.0 / (9.0 * L.ci)) * (l == UNET_NLAYERS - 1 ? 0.1 : 1.0);
        for (size_t i = 0; i < n; ++i) theta[o + i] = (float)(sd * z[i]);
        o += n + L.co;
    }
    if ((e = cudaMemcpy(u->theta, theta.data(), theta.size() * 4, cudaMemcpyHostToDevice)) !=
        cudaSuccess) {
        cfm_unet_destroy(h);
        CFM_CUDA_TRY(e);
    }
    if ((st = unet_refresh_weights(u, 0))) {
        cfm_unet_destroy(h);
        return st;
    }
    *out = h;
    return CFM_OK;
}

void cfm_unet_destroy(cfm_unet *h) {
    if (!h) return;
    unet_destroy(h->u);
    cudaFree(h->xin);
    cudaFree(h->out);
    cudaFree(h->dout);
    delete h;
}

int cfm_unet_get_params(cfm_unet *h, float *theta) {
    CFM_ARG_CHECK(h && theta, "null argument");
    CFM_CUDA_TRY(cudaMemcpy(theta, h->u->theta, h->u->nparams * 4, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

int cfm_unet_set_params(cfm_unet *h, const float *theta) {
    CFM_ARG_CHECK(h && theta, "null argument");
    CFM_CUDA_TRY(cudaMemcpy(h->u->theta, theta, h->u->nparams * 4, cudaMemcpyHostToDevice));
    int st = unet_refresh_weights(h->u, 0);
    if (st) return st;
    CFM_CUDA_TRY(cudaDeviceSynchronize());
    return CFM_OK;
}

int cfm_unet_set_training_info(cfm_unet *h, int smooth, int coarsen) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(smooth >= 0 && smooth <= 8, "smooth must be in [0, 8]");
    CFM_ARG_CHECK(coarsen == 1 || coarsen == 2, "coarsen must be 1 or 2");
    h->smooth = smooth;
    h->coarsen = coarsen;
    return CFM_OK;
}

int cfm_unet_forward_host(cfm_unet *h, int B, const float *in, float *out) {
    clear_error();
    CFM_ARG_CHECK(h && in && out, "null argument");
    CFM_ARG_CHECK(B >= 1 && B <= h->maxB, "batch");
    const size_t P = (size_t)B * h->u->H * h->u->W;
    CFM_CUDA_TRY(cudaMemcpy(h->xin, in, P * 2 * 4, cudaMemcpyHostToDevice));
    int st = unet_forward(h->u, B, h->xin, h->out, 0);
    if (st) return st;
    CFM_CUDA_TRY(cudaDeviceSynchronize());
    if ((st = unet_check_err(h->u))) return st;
    CFM_CUDA_TRY(cudaMemcpy(out, h->out, P * 4, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

int cfm_unet_gradient_host(cfm_unet *h, int B, const float *in, const float *dout, float *grad) {
    clear_error();
    CFM_ARG_CHECK(h && in && dout && grad, "null argument");
    CFM_ARG_CHECK(B >= 1 && B <= h->maxB, "batch");
    const size_t P = (size_t)B * h->u->H * h->u->W;
    CFM_CUDA_TRY(cudaMemcpy(h->xin, in, P * 2 * 4, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemcpy(h->dout, dout, P * 4, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemset(h->u->grad, 0, h->u->nparams * 4));
    int st = unet_forward(h->u, B, h->xin, h->out, 0);
    if (st) return st;
    if ((st = unet_backward(h->u, B, h->xin, h->dout, 0))) return st;
    CFM_CUDA_TRY(cudaDeviceSynchronize());
    if ((st = unet_check_err(h->u))) return st;
    CFM_CUDA_TRY(cudaMemcpy(grad, h->u->grad, h->u->nparams * 4, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

// Device time of one forward pass on the net's own input buffer (whatever it
// holds), averaged over `iters` passes after one warm-up: CUDA events.
int cfm_unet_set_forward_mode(cfm_unet *h, int mode) {
    clear_error();
    CFM_ARG_CHECK(h, "null argument");
    CFM_ARG_CHECK(mode == CFM_UNET_FORWARD_AUTO || mode == CFM_UNET_FORWARD_LAYERS ||
                      mode == CFM_UNET_FORWARD_PERSISTENT,
                  "mode must be CFM_UNET_FORWARD_AUTO, _LAYERS or _PERSISTENT");
    h->u->fwd_mode = mode;
    return CFM_OK;
}

int cfm_unet_time_forward(cfm_unet *h, int B, int iters, double *ms_per_forward) {
    clear_error();
    CFM_ARG_CHECK(h && ms_per_forward && iters >= 1, "arguments");
    CFM_ARG_CHECK(B >= 1 && B <= h->maxB, "batch");
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CFM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // one forward captured in a CUDA graph, replayed back to back: the way
    // a solver's graph runs it (no host launch gaps)
    int st = unet_forward(h->u, B, h->xin, h->out, s);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaSuccess;
    if (!st) e = cudaStreamSynchronize(s);
    if (!st && e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (!st && e == cudaSuccess) {
        st = unet_forward(h->u, B, h->xin, h->out, s);
        e = cudaStreamEndCapture(s, &graph);
    }
    if (!st && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (!st && e == cudaSuccess) e = cudaGraphLaunch(exec, s);
    if (!st && e == cudaSuccess) {
        cudaEventRecord(e0, s);
        for (int i = 0; i < iters && e == cudaSuccess; ++i) e = cudaGraphLaunch(exec, s);
        cudaEventRecord(e1, s);
    }
    const cudaError_t es = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = es;
    float ms = 0;
    if (!st && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (st) return st;
    CFM_CUDA_TRY(e);
    if ((st = unet_check_err(h->u))) return st;
    *ms_per_forward = ms / iters;
    return CFM_OK;
}

// Deterministic bounded input and output-gradient patterns for the
// training-step timing.
__global__ void k_train_pattern(float *x, long long nx, float *d, long long nd) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nx;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = (float)((i * 2654435761LL) % 2001 - 1000) * 5e-4f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nd;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = (float)((i * 40503LL) % 2001 - 1000) * 1e-4f;
}

int cfm_unet_time_train_step(cfm_unet *h, int B, int iters, double *ms_per_step) {
    clear_error();
    CFM_ARG_CHECK(h && ms_per_step && iters >= 1, "arguments");
    CFM_ARG_CHECK(B >= 1 && B <= h->maxB, "batch");
    int H = 0, W = 0;
    unet_shape(h->u, &H, &W);
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CFM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const long long px = (long long)B * H * W;
    k_train_pattern<<<1024, 256, 0, s>>>(h->xin, 2 * px, h->dout, px);
    auto step = [&]() -> int {
        int st = unet_forward(h->u, B, h->xin, h->out, s);
        if (st) return st;
        if (cudaMemsetAsync(unet_grad(h->u), 0, unet_params(h->u) * sizeof(float), s) != cudaSuccess)
            return CFM_CUDA_ERROR;
        if ((st = unet_backward(h->u, B, h->xin, h->dout, s))) return st;
        return unet_adam(h->u, 1e-4f, 1.0f, s);
    };
    int st = step();
    if (!st) {
        cudaEventRecord(e0, s);
        for (int i = 0; i < iters && !st; ++i) st = step();
        cudaEventRecord(e1, s);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    float ms = 0;
    if (!st && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (st) return st;
    CFM_CUDA_TRY(e);
    if ((st = unet_check_err(h->u))) return st;
    *ms_per_step = ms / iters;
    return CFM_OK;
}

// BF16 patterns of one activation of the last forward pass, in the order
// h0 p1 h1 p2 h2 p3 h3 g3 u2 g2 u1 g1 u0 g0 (index 0..13), B images.
int cfm_unet_activation_host(cfm_unet *h, int which, int B, unsigned short *out) {
    clear_error();
    CFM_ARG_CHECK(h && out, "null argument");
    CFM_ARG_CHECK(B >= 1 && B <= h->maxB, "batch");
    const UNetBuffers &a = h->u->a;
    const bf16 *bufs[14] = {a.h0, a.p1, a.h1, a.p2, a.h2, a.p3, a.h3, a.g3, a.u2, a.g2, a.u1, a.g1, a.u0, a.g0};
    const int lev[14] = {0, 1, 1, 2, 2, 3, 3, 3, 2, 2, 1, 1, 0, 0};
    const int ch[14] = {32, 32, 64, 64, 128, 128, 256, 128, 128, 64, 64, 32, 32, 32};
    CFM_ARG_CHECK(which >= 0 && which < 14, "activation index");
    const size_t n = (size_t)B * (h->u->H >> lev[which]) * (h->u->W >> lev[which]) * ch[which];
    CFM_CUDA_TRY(cudaMemcpy(out, bufs[which], n * 2, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

}  // extern "C"
