// Device bodies of the U-Net's CUDA-core layers: the first (2 -> 32) and
// last (32 -> 1) convolutions in FP32, the 2x2 mean pool and the
// upsample-and-add of a skip connection.  Each is written for one block of
// 256 threads with its block coordinates (bx, by, bz) as arguments: the
// per-layer kernels (learned.cu) pass blockIdx, the persistent forward
// (unet_fused.cu) the coordinates of the virtual blocks each CTA walks, so
// both compute the same values.
#pragma once

#include <cuda_bf16.h>

#include "cfm_internal.h"
#include "learned_internal.h"

namespace cfm {
namespace unet_dev {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ void load8(const bf16 *p, float *v) {
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 f = __bfloat1622float2(h[i]);
        v[2 * i] = f.x;
        v[2 * i + 1] = f.y;
    }
}

__device__ __forceinline__ void store8(bf16 *p, const float *v) {
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

// Pixels a thread of the first / last layer computes side by side in x: the
// 3 x (PXB + 2) input neighbourhood is loaded once for all of them.
constexpr int PXB = 4;

// h0 = relu(cin(x)): x FP32 [B][H][W][2], w [9][32][2].  Lane = 8 * group +
// q: a group of 8 lanes covers PXB consecutive pixels, lane q their channels
// 4q .. 4q + 3, with its 72 weights and 4 biases in registers; per tap and
// channel o += w0 x0 + w1 x1, taps in order.  Input channel 0 is optionally
// scaled by 1 / rms from a solver's partial sums.  A block walks CIN_SPAN
// pixel groups of one row.  grid: (ceil(W / (PXB CIN_SPAN 32)), H, B), 256 threads.
constexpr int CIN_SPAN = 2;
__device__ __forceinline__ void cin_block(const float *x, const float *w, const float *b, bf16 *h0, int H, int W,
                                          const UNetInputScale &in_scale, int bx, int by, int bz) {
    float sc = 1.f;
    if (in_scale.part) {
        __shared__ double red[8];
        const double *part = in_scale.part + bz * in_scale.part_stride;
        const double cells = in_scale.cells_img ? in_scale.cells_img[bz] : in_scale.cells;
        double acc = 0;
        for (int j = threadIdx.x; j < in_scale.nparts; j += blockDim.x) acc += part[j];
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        double tot = 0;
        for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) tot += red[wi];
        sc = tot > 0 ? (float)sqrt(cells / tot) : 0.f;
        __syncthreads();  // red is read by all before a next call writes it
    }
    const int q = threadIdx.x & 7, c0 = q * 4, grp = threadIdx.x >> 3;  // 32 groups per block
    float wr[9][8];  // [t][(c - c0) * 2 + in]
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        const float4 w0 = *reinterpret_cast<const float4 *>(w + t * 64 + c0 * 2);
        const float4 w1 = *reinterpret_cast<const float4 *>(w + t * 64 + c0 * 2 + 4);
        wr[t][0] = w0.x, wr[t][1] = w0.y, wr[t][2] = w0.z, wr[t][3] = w0.w;
        wr[t][4] = w1.x, wr[t][5] = w1.y, wr[t][6] = w1.z, wr[t][7] = w1.w;
    }
    const float4 bq = *reinterpret_cast<const float4 *>(b + c0);
    const int yy = by, img = bz;
    const float *xi = x + (size_t)img * H * W * 2;
    bf16 *hrow = h0 + ((size_t)img * H + yy) * W * 32;
#pragma unroll 1
    for (int span = 0; span < CIN_SPAN; ++span) {
        const int xs = ((bx * CIN_SPAN + span) * 32 + grp) * PXB;  // first pixel of the group
        if (xs >= W) break;
        float o[PXB][4];
#pragma unroll
        for (int p = 0; p < PXB; ++p) o[p][0] = bq.x, o[p][1] = bq.y, o[p][2] = bq.z, o[p][3] = bq.w;
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
            const int y = yy + dy - 1;
            const bool yin = y >= 0 && y < H;
            const int yc = min(max(y, 0), H - 1);
            float2 v[PXB + 2];
#pragma unroll
            for (int k = 0; k < PXB + 2; ++k) {
                const int xq = xs + k - 1;
                const int xc = min(max(xq, 0), W - 1);
                v[k] = *reinterpret_cast<const float2 *>(xi + 2 * (yc * W + xc));
                if (in_scale.part) v[k].x *= sc;
                if (!(yin && xq >= 0 && xq < W)) v[k] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int t = dy * 3 + dx;
#pragma unroll
                for (int p = 0; p < PXB; ++p)
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        o[p][c] += wr[t][2 * c] * v[p + dx].x + wr[t][2 * c + 1] * v[p + dx].y;
            }
        }
#pragma unroll
        for (int p = 0; p < PXB; ++p) {
            if (xs + p >= W) break;
            __nv_bfloat162 r[2];
            r[0] = __floats2bfloat162_rn(fmaxf(o[p][0], 0.f), fmaxf(o[p][1], 0.f));
            r[1] = __floats2bfloat162_rn(fmaxf(o[p][2], 0.f), fmaxf(o[p][3], 0.f));
            *reinterpret_cast<uint2 *>(hrow + (size_t)(xs + p) * 32 + c0) = *reinterpret_cast<const uint2 *>(r);
        }
    }
}

// out = cout(g0): g0 [B][H][W][32], w [9][1][32], out FP32.  Lane = 4 *
// group + q: a group of 4 lanes covers PXB consecutive pixels, lane q the
// 8-channel group q with its 72 weights in registers, summing over the 9
// taps in order (one 8-term expression per tap); two xor shuffles add the
// groups, (g0 + g1) + (g2 + g3).  A block walks COUT_SPAN pixel groups of
// one row.  grid: (ceil(W / (PXB COUT_SPAN 64)), H, B), 256 threads.
constexpr int COUT_SPAN = 2;
__device__ __forceinline__ void cout_block(const bf16 *g0, const float *w, const float *b, float *out, int H,
                                           int W, int bx, int by, int bz) {
    const int q = threadIdx.x & 3, c0 = q * 8, grp = threadIdx.x >> 2;  // 64 groups per block
    float wr[9][8];
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        const float4 w0 = *reinterpret_cast<const float4 *>(w + t * 32 + c0);
        const float4 w1 = *reinterpret_cast<const float4 *>(w + t * 32 + c0 + 4);
        wr[t][0] = w0.x, wr[t][1] = w0.y, wr[t][2] = w0.z, wr[t][3] = w0.w;
        wr[t][4] = w1.x, wr[t][5] = w1.y, wr[t][6] = w1.z, wr[t][7] = w1.w;
    }
    const float bias = b[0];
    const int yy = by, img = bz;
    const bf16 *gi = g0 + (size_t)img * H * W * 32;
    float *oi = out + ((size_t)img * H + yy) * W;
#pragma unroll 1
    for (int span = 0; span < COUT_SPAN; ++span) {
        // every lane stays to the shuffles; pixels past the row end sum zero
        const int xs = ((bx * COUT_SPAN + span) * 64 + grp) * PXB;
        float acc[PXB];
#pragma unroll
        for (int p = 0; p < PXB; ++p) acc[p] = 0.f;
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
            const int y = yy + dy - 1;
            const bool yin = y >= 0 && y < H;
            const int yc = min(max(y, 0), H - 1);
            float v[PXB + 2][8];
#pragma unroll
            for (int k = 0; k < PXB + 2; ++k) {
                const int xq = xs + k - 1;
                const int xc = min(max(xq, 0), W - 1);
                uint4 raw = *reinterpret_cast<const uint4 *>(gi + (size_t)(yc * W + xc) * 32 + c0);
                if (!(yin && xq >= 0 && xq < W)) raw = make_uint4(0u, 0u, 0u, 0u);
                const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&raw);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float2 f = __bfloat1622float2(h[i]);
                    v[k][2 * i] = f.x;
                    v[k][2 * i + 1] = f.y;
                }
            }
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int t = dy * 3 + dx;
#pragma unroll
                for (int p = 0; p < PXB; ++p) {
                    const float *vv = v[p + dx];
                    acc[p] += wr[t][0] * vv[0] + wr[t][1] * vv[1] + wr[t][2] * vv[2] + wr[t][3] * vv[3] +
                              wr[t][4] * vv[4] + wr[t][5] * vv[5] + wr[t][6] * vv[6] + wr[t][7] * vv[7];
                }
            }
        }
#pragma unroll
        for (int p = 0; p < PXB; ++p) {
            float a = acc[p];
            a += __shfl_xor_sync(0xffffffffu, a, 1);
            a += __shfl_xor_sync(0xffffffffu, a, 2);
            if (q == 0 && xs + p < W) oi[xs + p] = a + bias;
        }
    }
}

// 2x2 mean pool, NHWC, 8 channels per thread; (h, w) is the pooled size.
// grid: (items of a pooled row / blockDim, h, B).
template <int C>
__device__ __forceinline__ void pool_block(const bf16 *in, bf16 *out, int h, int w, int bx, int by, int bz) {
    constexpr int G = C / 8;
    const int e = bx * blockDim.x + threadIdx.x;
    if (e >= w * G) return;
    const int y = by, img = bz;
    const int c8 = (e % G) * 8, x = e / G;
    const size_t W2 = 2 * (size_t)w;
    const size_t base = (((size_t)img * 2 * h + 2 * y) * W2 + 2 * x) * C + c8;
    float a[8], b[8], c[8], d[8], o[8];
    load8(in + base, a);
    load8(in + base + C, b);
    load8(in + base + W2 * C, c);
    load8(in + base + W2 * C + C, d);
#pragma unroll
    for (int j = 0; j < 8; ++j) o[j] = 0.25f * (((a[j] + b[j]) + c[j]) + d[j]);
    store8(out + (((size_t)img * h + y) * w + x) * C + c8, o);
}

// u = up(g) + skip at the finer level (2h x 2w; (h, w) is the coarse size).
// grid: (items of a fine row / blockDim, 2h, B).
template <int C>
__device__ __forceinline__ void up_add_block(const bf16 *g, const bf16 *skip, bf16 *u, int h, int w, int bx, int by,
                                             int bz) {
    constexpr int G = C / 8;
    const int e = bx * blockDim.x + threadIdx.x;
    if (e >= 2 * w * G) return;
    const int y = by, img = bz;
    const int c8 = (e % G) * 8, x = e / G;
    const size_t cp = ((size_t)img * h + y / 2) * w + x / 2;
    const size_t pix = ((size_t)img * 2 * h + y) * 2 * w + x;
    float a[8], b[8];
    load8(g + cp * C + c8, a);
    load8(skip + pix * C + c8, b);
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] += b[j];
    store8(u + pix * C + c8, a);
}

}  // namespace unet_dev
}  // namespace cfm
