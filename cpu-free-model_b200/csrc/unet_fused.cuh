// The U-Net forward as one persistent kernel: one CTA per SM walks the
// layers in order, separated by grid barriers with a bounded wait, and keeps
// its mbarrier ring and 512 TMEM columns for the whole pass.
//
// The per-layer path (learned.cu: k_cin_fwd, k_pool, tc_conv_kernel,
// tc_splitk_epilogue, k_up_add, k_cout_fwd) launches 19 kernels for one
// forward; at the preconditioner's size (256^2, batch 1) each launch is a
// few microseconds of set-up and drain around well under a microsecond of
// tensor-core work.  Here the phases are
//
//   cin | pool | e1 | pool | e2 | pool | e3 | d3 (+ up-add) | d2 (+ up-add)
//   | d1 (+ up-add) | d0 | cout
//
// with a split-K layer adding a reduction phase after its convolution.  Every
// phase computes exactly what its per-layer kernel computes: the CUDA-core
// layers call the same block bodies (unet_layers.cuh) over the same virtual
// block grid, and each convolution uses the per-layer plan (tiling, halo or
// per-tap staging, split-K) of tc_conv_fwd, the same K order and the same
// epilogue arithmetic, so the output is bit-identical to the per-layer
// path.  The upsample-and-add that follows d3, d2 and d1 is folded into
// their epilogue (or split-K reduction): each coarse pixel also writes its
// four fine pixels up(g) + skip.
//
// Measured on B200 (one forward replayed from a CUDA graph): 117 us at
// 256^2 batch 1 against 92 us for the per-layer kernels, 239 against 147 us
// at 512^2, 390 against 251 us at 256^2 batch 8.  A grid barrier costs
// 1.3-1.6 us, and the phases are bound by memory latency on few CTAs: the
// coarse layers' split-K partials (8-9 MB written, then read by the
// reduction phase) make each such pair 7-12 us, and the phase after a
// convolution waits for its epilogue stores to drain.  The per-layer
// kernels overlap those tails with the next launch (programmatic dependent
// launch), so they stay the default.
//
// Warp roles in a convolution phase are those of tc_conv_kernel (warp 0
// TMA, warp 1 TMEM owner and MMA issuer, warps 2-5 epilogue); warps 6 and 7
// only join the CUDA-core phases.  The ring counters carry over from one
// convolution to the next, so no barrier is re-initialised.  Weights stream
// with the operand tiles (no resident copy).  Every wait is bounded: a
// timed-out pipeline wait records the site in `err` and the grid barrier's
// error word, so that every CTA leaves at its next barrier; then the CTA
// lets its copies and MMAs land (bounded) and frees TMEM.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "barrier.cuh"
#include "tc_conv.cuh"
#include "tma.cuh"
#include "unet_internal.h"
#include "unet_layers.cuh"

namespace cfm {

constexpr int UF_CONVS = 7;  // the tensor-core layers e1 e2 e3 d3 d2 d1 d0
constexpr int UF_THREADS = 256;
constexpr int UF_TMEM_COLS = 512;  // two accumulators of up to 256 columns

// One tensor-core convolution of the pass (its tc_conv_fwd plan).
struct UfConv {
    int H, W, N, kc;  // grid, output channels, input channel chunk (32 or 64)
    int bx, by, tiles_x, tiles_y, nch, halo, ksteps, csplit, ntiles;
    int a_region;  // bytes of the A operand in a ring slot; B follows it
    const float *bias;
    int relu;
    __nv_bfloat16 *out;  // [B][H][W][N]
    float *ws;           // csplit > 1: FP32 partials [csplit][B H W][N]
    // optional up-add at the 2H x 2W level: uout = up(out) + skip
    const __nv_bfloat16 *skip;
    __nv_bfloat16 *uout;
};

struct UfParams {
    int B, H, W;
    const float *x;  // [B][H][W][2]
    float *out;      // [B][H][W]
    UNetInputScale in_scale;
    const float *cin_w, *cin_b, *cout_w, *cout_b;
    __nv_bfloat16 *h0, *p1, *h1, *p2, *h2, *p3;
    UfConv conv[UF_CONVS];
    int stages, slot_bytes;
    int *err;
    UfBarrier *bar;
    unsigned long long budget_ns;
};

// Grid barrier of the persistent forward (UfBarrier, unet_internal.h): a
// monotonic 64-bit arrival count.
// A barrier is one release add per CTA and an acquire spin until the count
// reaches the CTA's target (the count at the start of the pass, rounded down
// to a multiple of the grid, plus one grid per barrier so far): no
// last-arriver round trip.  The count stays a multiple of the grid between
// passes because every CTA arrives at every barrier; after a timed-out wait
// (error set) the host resets the whole struct before the next pass.
// All threads of every CTA call it; true when every CTA arrived.
__device__ __forceinline__ bool uf_grid_sync(UfBarrier *b, unsigned long long &target, int site) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        target += gridDim.x;
        asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(&b->count) : "memory");
        int ok = 1;
        const unsigned long long t0 = global_ns();
        for (unsigned n = 1; ld_acquire_u64(&b->count) < target; ++n) {
            if ((n & 63) == 0) {
                if (ld_relaxed_i32(&b->error)) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > b->timeout_ns) {
                    if (atomicCAS(&b->error, 0, 1) == 0) b->where = site;
                    ok = 0;
                    break;
                }
            }
        }
        if (ld_relaxed_i32(&b->error)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Tensor maps of the convolutions: the A operand (halo or per-tap box) and
// the weights of each layer.
struct __align__(64) UfMaps {
    CUtensorMap a[UF_CONVS];
    CUtensorMap b[UF_CONVS];
};

// Dynamic shared memory of the pass: alignment slack, the ring, the
// full/empty/accumulator/drain mbarriers and the TMEM base slot.
__host__ __device__ constexpr size_t uf_smem_bytes(int stages, int slot_bytes) {
    return 1024 + (size_t)stages * slot_bytes + (2 * (size_t)stages + 5) * 8 + 16;
}

// K-major descriptor with a runtime row size (kmajor_desc with SW = sw).
__device__ __forceinline__ uint64_t kmajor_desc_rt(uint32_t saddr, int sw) {
    const uint64_t layout = sw == 128 ? 2 : 4;
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((8 * sw) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= layout << 61;
    return d;
}

struct UfRing {
    unsigned char *ring;
    uint64_t *full, *empty, *acc_full, *acc_empty, *drain;
    uint32_t tmem;
    int stages, slot;
    unsigned long long budget;
};

// Writes out[pixel] (16 channels, BF16) and, with an up-add, the four fine
// pixels up(out) + skip; `g` holds the 16 rounded values.
__device__ __forceinline__ void uf_up_add16(const UfConv &L, int img, int x, int y, int c, const float *g) {
    const int W2 = 2 * L.W, H2 = 2 * L.H;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const size_t fp = (((size_t)img * H2 + 2 * y + i) * W2 + 2 * x + j) * L.N + c;
            float s0[8], s1[8];
            unet_dev::load8(L.skip + fp, s0);
            unet_dev::load8(L.skip + fp + 8, s1);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                s0[k] = g[k] + s0[k];
                s1[k] = g[8 + k] + s1[k];
            }
            unet_dev::store8(L.uout + fp, s0);
            unet_dev::store8(L.uout + fp + 8, s1);
        }
}

// One convolution phase (all threads of the CTA call it).  `it` and `lt`
// are the ring-slot and accumulator counters of the calling role thread.
__device__ __forceinline__ void uf_conv(const UfConv &L, const CUtensorMap *mA, const CUtensorMap *mB,
                                        const UfRing &R, int B, unsigned &it, unsigned &lt,
                                        volatile int *abort_flag, int *err, UfBarrier *bar, float *s_bias) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int S = R.stages;
    const int SW = L.kc * 2, BTAP = L.N * SW;
    auto fail = [&](int code) {
        atomicCAS(err, 0, code);
        atomicCAS(&bar->error, 0, 1);  // every CTA leaves at its next grid barrier
        *abort_flag = 1;
    };
    for (int c = threadIdx.x; c < L.N; c += blockDim.x) s_bias[c] = L.bias ? L.bias[c] : 0.f;
    __syncthreads();
    if (warp == 0) {
        if (lane == 0) {
            fence_proxy_async_global();  // the previous phases' stores, before TMA reads them
            for (int t = blockIdx.x; t < L.ntiles && !*abort_flag; t += gridDim.x) {
                const int pt = t / L.csplit, sp = t % L.csplit;
                const int tx = pt % L.tiles_x, rest = pt / L.tiles_x;
                const int x0 = tx * L.bx, y0 = (rest % L.tiles_y) * L.by, img = rest / L.tiles_y;
                const int q0 = L.ksteps * sp / L.csplit, q1 = L.ksteps * (sp + 1) / L.csplit;
                bool ok = true;
                for (int q = q0; q < q1; ++q, ++it) {
                    const int st = it % S;
                    if (!mbar_wait_bounded(&R.empty[st], ((it / S) & 1) ^ 1, R.budget)) {
                        fail(11);
                        ok = false;
                        break;
                    }
                    unsigned char *a_dst = R.ring + (size_t)st * R.slot;
                    unsigned char *b_dst = a_dst + L.a_region;
                    if (L.halo) {
                        const int ch = q / 3, dy = q % 3;
                        mbar_arrive_expect_tx(&R.full[st], TC_HALO_ROWS * SW + 3 * BTAP);
                        tma_load_4d(a_dst, mA, ch * L.kc, x0 - 1, y0 + dy - 1, img, &R.full[st]);
                        for (int dx = 0; dx < 3; ++dx)
                            tma_load_3d(b_dst + dx * BTAP, mB, ch * L.kc, 0, dy * 3 + dx, &R.full[st]);
                    } else {
                        const int tap = q / L.nch, ch = q % L.nch;
                        const int dy = tap / 3, dx = tap % 3;
                        mbar_arrive_expect_tx(&R.full[st], 128 * SW + BTAP);
                        tma_load_4d(a_dst, mA, ch * L.kc, x0 + dx - 1, y0 + dy - 1, img, &R.full[st]);
                        tma_load_3d(b_dst, mB, ch * L.kc, 0, tap, &R.full[st]);
                    }
                }
                if (!ok) break;
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc =
                (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(L.N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
            bool ok = true;
            for (int t = blockIdx.x; ok && t < L.ntiles && !*abort_flag; t += gridDim.x, ++lt) {
                const int ab = lt & 1;
                if (!mbar_wait_bounded(&R.acc_empty[ab], ((lt >> 1) & 1) ^ 1, R.budget)) {
                    fail(12);
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = R.tmem + ab * 256;
                const int sp = t % L.csplit;
                const int q0 = L.ksteps * sp / L.csplit, q1 = L.ksteps * (sp + 1) / L.csplit;
                for (int q = q0; q < q1; ++q, ++it) {
                    const int st = it % S;
                    if (!mbar_wait_bounded(&R.full[st], (it / S) & 1, R.budget)) {
                        fail(13);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(R.ring + (size_t)st * R.slot);
                    const uint32_t b_addr = a_addr + L.a_region;
                    if (L.halo) {
                        // tap (dy, dx): A = rows dx .. dx + 127 of the halo box
                        for (int dx = 0; dx < 3; ++dx) {
                            const uint32_t a0 = a_addr + dx * SW, b0 = b_addr + dx * BTAP;
                            for (int kk = 0; kk < L.kc / 16; ++kk)
                                umma_bf16(d_tmem, kmajor_desc_rt(a0 + kk * 32, SW), kmajor_desc_rt(b0 + kk * 32, SW),
                                          idesc, (q > q0 || dx > 0 || kk > 0) ? 1u : 0u);
                        }
                    } else {
                        for (int kk = 0; kk < L.kc / 16; ++kk)
                            umma_bf16(d_tmem, kmajor_desc_rt(a_addr + kk * 32, SW),
                                      kmajor_desc_rt(b_addr + kk * 32, SW), idesc, (q > q0 || kk > 0) ? 1u : 0u);
                    }
                    umma_commit(&R.empty[st]);  // frees the slot once these MMAs are done
                }
                if (!ok) break;
                umma_commit(&R.acc_full[ab]);
            }
        }
        __syncwarp();
    } else if (warp < 6) {
        const int q4 = warp & 3;  // TMEM lanes 32 q4 .. 32 q4 + 31
        const int row = q4 * 32 + lane;
        const size_t npix = (size_t)B * L.H * L.W;
        for (int t = blockIdx.x; t < L.ntiles && !*abort_flag; t += gridDim.x, ++lt) {
            const int ab = lt & 1;
            if (!mbar_wait_bounded(&R.acc_full[ab], (lt >> 1) & 1, R.budget)) {
                fail(14);
                break;
            }
            tc_fence_after();
            const uint32_t tbase = R.tmem + ((uint32_t)(q4 * 32) << 16) + ab * 256;
            const int pt = t / L.csplit, sp = t % L.csplit;
            const int tx = pt % L.tiles_x, rest = pt / L.tiles_x;
            const int img = rest / L.tiles_y;
            auto pixel = [&](int r, bool &in, int &x, int &y) {
                x = tx * L.bx + r % L.bx;
                y = (rest % L.tiles_y) * L.by + r / L.bx;
                in = x < L.W && y < L.H;
                return ((size_t)img * L.H + (in ? y : 0)) * L.W + (in ? x : 0);
            };
            bool in_me, in_e, in_o;
            int xm, ym, xt, yt;
            const size_t pix = pixel(row, in_me, xm, ym);
            __nv_bfloat16 *oe = L.out + pixel(row & ~1, in_e, xt, yt) * L.N;
            __nv_bfloat16 *oo = L.out + pixel(row | 1, in_o, xt, yt) * L.N;
            for (int c = 0; c < L.N; c += 16) {
                float acc[16];
                tmem_ld16(tbase + c, acc);
                if (L.csplit > 1) {  // split-K partial: FP32, the reduction phase applies the epilogue
                    if (in_me) {
                        float4 *d = reinterpret_cast<float4 *>(L.ws + ((size_t)sp * npix + pix) * L.N + c);
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            d[j] = make_float4(acc[4 * j], acc[4 * j + 1], acc[4 * j + 2], acc[4 * j + 3]);
                    }
                    continue;
                }
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    v[j] = acc[j] + s_bias[c + j];
                    if (L.relu) v[j] = fmaxf(v[j], 0.f);
                }
                uint4 lo, hi;
                __nv_bfloat162 *l2 = reinterpret_cast<__nv_bfloat162 *>(&lo);
                __nv_bfloat162 *h2 = reinterpret_cast<__nv_bfloat162 *>(&hi);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    l2[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    h2[j] = __floats2bfloat162_rn(v[8 + 2 * j], v[8 + 2 * j + 1]);
                }
                store16_pairs(oe + c, oo + c, in_e, in_o, lane, lo, hi);
                if (L.uout && in_me) {
                    float g[16];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 a = __bfloat1622float2(l2[j]), b = __bfloat1622float2(h2[j]);
                        g[2 * j] = a.x, g[2 * j + 1] = a.y, g[8 + 2 * j] = b.x, g[8 + 2 * j + 1] = b.y;
                    }
                    uf_up_add16(L, img, xm, ym, c, g);
                }
            }
            // accumulator drained: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&R.acc_empty[ab]);
        }
    }
    fence_proxy_async_global();
}

// The split-K reduction of a convolution (all threads of all CTAs): the
// arithmetic of tc_splitk_epilogue (partials added in split order, + bias,
// optional ReLU, BF16), then the optional up-add of 8 channels.
__device__ __forceinline__ void uf_reduce(const UfConv &L, int B) {
    const long long npix = (long long)B * L.H * L.W;
    const int G = L.N / 8;
    const long long items = npix * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < items;
         e += (long long)gridDim.x * blockDim.x) {
        const long long pix = e / G;
        const int c = (int)(e % G) * 8;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.f;
        for (int sp = 0; sp < L.csplit; ++sp) {
            const float4 *src = reinterpret_cast<const float4 *>(L.ws + ((size_t)sp * npix + pix) * L.N + c);
            const float4 a = src[0], b = src[1];
            v[0] += a.x, v[1] += a.y, v[2] += a.z, v[3] += a.w;
            v[4] += b.x, v[5] += b.y, v[6] += b.z, v[7] += b.w;
        }
        uint4 o;
        __nv_bfloat162 *o2 = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            float a = v[j] + (L.bias ? L.bias[c + j] : 0.f), b = v[j + 1] + (L.bias ? L.bias[c + j + 1] : 0.f);
            if (L.relu) a = fmaxf(a, 0.f), b = fmaxf(b, 0.f);
            o2[j / 2] = __floats2bfloat162_rn(a, b);
        }
        *reinterpret_cast<uint4 *>(L.out + pix * L.N + c) = o;
        if (L.uout) {
            const int x = (int)(pix % L.W), y = (int)((pix / L.W) % L.H), img = (int)(pix / ((long long)L.W * L.H));
            float g[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 f = __bfloat1622float2(o2[j]);
                g[2 * j] = f.x, g[2 * j + 1] = f.y;
            }
            const int W2 = 2 * L.W, H2 = 2 * L.H;
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const size_t fp = (((size_t)img * H2 + 2 * y + i) * W2 + 2 * x + j) * L.N + c;
                    float s[8];
                    unet_dev::load8(L.skip + fp, s);
#pragma unroll
                    for (int k = 0; k < 8; ++k) s[k] = g[k] + s[k];
                    unet_dev::store8(L.uout + fp, s);
                }
        }
    }
    fence_proxy_async_global();
}

// 2x2 mean pool (h, w the pooled size) over the per-layer kernel's grid.
template <int C>
__device__ __forceinline__ void uf_pool(const __nv_bfloat16 *in, __nv_bfloat16 *out, int B, int h, int w) {
    const int nbx = (w * (C / 8) + 255) / 256;
    const int nvb = nbx * h * B;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
        unet_dev::pool_block<C>(in, out, h, w, vb % nbx, (vb / nbx) % h, vb / (nbx * h));
    fence_proxy_async_global();
}

__global__ void __launch_bounds__(UF_THREADS, 1)
    unet_fused_fwd(const __grid_constant__ UfMaps maps, const __grid_constant__ UfParams p) {
    extern __shared__ unsigned char uf_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)uf_smem_raw + 1023) & ~(uintptr_t)1023);
    const int S = p.stages;
    UfRing R;
    R.ring = smem;
    R.full = reinterpret_cast<uint64_t *>(smem + (size_t)S * p.slot_bytes);
    R.empty = R.full + S;
    R.acc_full = R.empty + S;
    R.acc_empty = R.acc_full + 2;
    R.drain = R.acc_empty + 2;
    R.stages = S;
    R.slot = p.slot_bytes;
    R.budget = p.budget_ns;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(R.drain + 1);
    __shared__ int s_abort;
    __shared__ float s_bias[256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&R.full[s], 1);
            mbar_init(&R.empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&R.acc_full[b], 1);
            mbar_init(&R.acc_empty[b], 4);
        }
        mbar_init(R.drain, 1);
        s_abort = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, UF_TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    R.tmem = *tmem_slot;
    volatile int *abort_flag = &s_abort;
    unsigned it = 0, lt = 0;
    int site = 0;
    const int B = p.B, H = p.H, W = p.W;
    // the count at the start of this pass: at most gridDim.x - 1 CTAs can
    // have arrived at the first barrier before this one reads it
    unsigned long long target = 0;
    if (threadIdx.x == 0) {
        target = ld_acquire_u64(&p.bar->count);
        target -= target % gridDim.x;
    }
    auto sync = [&]() { return uf_grid_sync(p.bar, target, site++); };
    auto conv = [&](int l) {
        const UfConv &L = p.conv[l];
        uf_conv(L, &maps.a[l], &maps.b[l], R, B, it, lt, abort_flag, p.err, p.bar, s_bias);
        if (L.csplit == 1) return true;
        if (!sync()) return false;
        uf_reduce(L, B);
        return true;
    };
    do {
        {  // cin: x -> h0
            const int nbx = (W + unet_dev::PXB * unet_dev::CIN_SPAN * 32 - 1) / (unet_dev::PXB * unet_dev::CIN_SPAN * 32);
            const int nvb = nbx * H * B;
            for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
                unet_dev::cin_block(p.x, p.cin_w, p.cin_b, p.h0, H, W, p.in_scale, vb % nbx, (vb / nbx) % H,
                                    vb / (nbx * H));
        }
        if (!sync()) break;
        uf_pool<32>(p.h0, p.p1, B, H / 2, W / 2);
        if (!sync()) break;
        if (!conv(0) || !sync()) break;  // e1 -> h1
        uf_pool<64>(p.h1, p.p2, B, H / 4, W / 4);
        if (!sync()) break;
        if (!conv(1) || !sync()) break;  // e2 -> h2
        uf_pool<128>(p.h2, p.p3, B, H / 8, W / 8);
        if (!sync()) break;
        if (!conv(2) || !sync()) break;  // e3 -> h3
        if (!conv(3) || !sync()) break;  // d3 -> g3, u2 = up(g3) + h2
        if (!conv(4) || !sync()) break;  // d2 -> g2, u1 = up(g2) + h1
        if (!conv(5) || !sync()) break;  // d1 -> g1, u0 = up(g1) + h0
        if (!conv(6) || !sync()) break;  // d0 -> g0
        {  // cout: g0 -> out
            const int nbx =
                (W + unet_dev::PXB * unet_dev::COUT_SPAN * 64 - 1) / (unet_dev::PXB * unet_dev::COUT_SPAN * 64);
            const int nvb = nbx * H * B;
            for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
                unet_dev::cout_block(p.conv[6].out, p.cout_w, p.cout_b, p.out, H, W, vb % nbx, (vb / nbx) % H,
                                     vb / (nbx * H));
        }
    } while (0);
    // let every copy and MMA issued here land before TMEM and shared memory go
    if (warp == 0 && lane == 0) {
        const unsigned lo = it > (unsigned)S ? it - S : 0u;
        for (unsigned j = lo; j < it; ++j) mbar_wait_bounded(&R.full[j % S], (j / S) & 1, R.budget);
    }
    if (warp == 1 && lane == 0) {
        umma_commit(R.drain);
        mbar_wait_bounded(R.drain, 0, R.budget);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(R.tmem, UF_TMEM_COLS);
    }
}

}  // namespace cfm
