// 3x3 convolutions on the 5th-generation tensor cores (tcgen05), BF16 in,
// FP32 accumulate in tensor memory (TMEM), for the learned preconditioner.
//
// Both passes are one implicit GEMM, C[m][n] = sum_k A[m][k] B[n][k], with
// K-major BF16 operand tiles brought into shared memory by TMA
// (cp.async.bulk.tensor, single CTA, no multicast) in the swizzled layout
// tcgen05.mma reads, and the FP32 accumulator in TMEM:
//
//  conv (forward, and backward-data with flipped/transposed weights):
//    m = 128 output pixels (a bx x by block of one image), n = output
//    channel, k = (tap, input channel chunk).  Coordinates outside the image
//    read as zero, which is the padding.  Two ways to stage A:
//      halo (bx = 128): per (chunk, dy) one box of the 130 pixels
//        x0 - 1 .. x0 + 128 of row y0 + dy - 1; the three dx taps are the
//        descriptors starting 0, 1 and 2 rows into it (the swizzle follows
//        the absolute shared-memory address, so a row-shifted start reads
//        the shifted rows).  A third of the TMA requests of 9 tap boxes.
//      per tap (bx < 128): the box at (c0, x0 + dx - 1, y0 + dy - 1, img).
//    B (weights) either streams with A or, when a CTA runs several tiles
//    and they fit, stays resident: all 9 x nch tiles loaded once per CTA.
//    Epilogue: + bias, optional ReLU, optional mask (zero where mask <= 0),
//    BF16 store NHWC (lane pairs write whole 32-byte sectors).
//  weight gradient:
//    m = (tap of a tap group, input channel), n = output channel, k = pixels
//    (KC consecutive x of one row per step).  Both operands are MN-major
//    (channels contiguous), read straight from the NHWC tensors: per tap
//    and block of 64 (or 32) channels one box of KC pixels of the layer
//    input at (c0, x + dx - 1, y + dy - 1, img), whose zero fill outside
//    the image is the padding, and per 64 (32) output channels one box of
//    the output gradient at (c0, x, y, img).  Tiles split K; the epilogue
//    stores its partial tile in a workspace [split][tap][ci][co] and
//    tc_wgrad_reduce adds the splits to dW[tap][co][ci] in split order, so
//    the gradient is the same on every run.
//
// Persistent CTAs (one or two per SM, as the host plan says), 6 warps: warp
// 0 issues TMA (one elected lane), warp 1 owns TMEM and issues tcgen05.mma
// (one lane), warps 2-5 drain the accumulator (tcgen05.ld, 32 TMEM lanes
// each).  A ring of operand slots (full/empty mbarriers) and two TMEM
// accumulators (acc_full / acc_empty) overlap loads, MMAs and the epilogue
// of the previous tile.  Every wait is bounded; on a timeout the CTA
// records an error, lets its in-flight copies and MMAs land (bounded),
// frees TMEM and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "cfm_internal.h"
#include "tma.cuh"

namespace cfm {

// ------------------------------------------------------- tcgen05 wrappers
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, M = 128, kind::f16 (BF16 operands here).
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                          uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
// mbarrier arrive once every tcgen05 op this thread issued so far has completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}
// 32 TMEM lanes x 16 consecutive 32-bit columns: thread l of the warp gets lane l.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tma_load_4d(void *dst_smem, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst_smem)),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor of a K-major, swizzled operand tile whose
// rows are SW bytes (SW = 64 or 128) and whose 8-row groups are 8 * SW bytes
// apart: start >> 4 (bits 0-13), leading offset 1 (16 B, bits 16-29), stride
// offset 8 * SW >> 4 (bits 32-45), version 1 (bits 46-47), layout type at
// bits 61-63 (2 = 128-byte swizzle, 4 = 64-byte swizzle).
template <int SW>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
    constexpr uint64_t layout = SW == 128 ? 2 : 4;
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((8 * SW) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= layout << 61;
    return d;
}

// Shared-memory matrix descriptor of an MN-major, swizzled operand tile:
// rows of SW bytes (SW / 2 channels, SW = 64 or 128) along K, 8-row groups
// `sbo` bytes apart, blocks of SW / 2 channels along M (or N) `lbo` bytes
// apart.  Field positions as in kmajor_desc.
__device__ __forceinline__ uint64_t mnmajor_desc(uint32_t saddr, int sw, uint32_t lbo, uint32_t sbo) {
    const uint64_t layout = sw == 128 ? 2 : 4;
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= layout << 61;
    return d;
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, N >> 3 at bits
// 17-22, M >> 4 at bits 24-28 (M = 128); A and B K-major, or both MN-major
// (bits 15 and 16).
template <int N, bool MN = false>
__host__ __device__ constexpr uint32_t idesc_bf16_m128() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (MN ? (1u << 15) | (1u << 16) : 0u) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

struct TcConvParams {
    int mode;  // 0 conv, 1 weight gradient
    int B, H, W;
    int Cin, Cout;  // of the convolution this pass belongs to (conv mode: Cin -> Cout = N)
    int ntiles;
    int ksteps;  // conv: 3 * nch (halo) or 9 * nch; wgrad: steps per split
    // conv mode tiling
    int bx, by, tiles_x, tiles_y;
    int nch;   // Cin / KC
    int halo;  // one (bx + 2)-pixel box per (chunk, dy); the dx taps are row offsets into it
    int wres;  // every weight tile resident in shared memory, loaded once per CTA
    int csplit;  // split-K: work item t = (pixel tile t / csplit, k range t % csplit)
    float *ws;   // csplit > 1: FP32 partials [csplit][B H W][N], reduced by tc_splitk_epilogue
    long long ws_floats;  // capacity of ws (0: no split)
    // wgrad mode tiling
    int ci_rows, ci_tiles, taps_per_tile, tap_groups, ksplit;
    int a_cb, b_cb;     // channels of one operand box (64, or 32 for 32-channel tensors)
    long long total_k;  // B * H * (W / KC)
    // shared-memory plan
    int stages;       // operand ring depth
    int stage_bytes;  // one ring slot (a multiple of 1024)
    int a_region;     // bytes of the A part of a slot; B (if streamed) follows it
    int wres_bytes;   // resident weight region in front of the ring (a multiple of 1024)
    // epilogue
    const float *bias;
    int relu;
    const __nv_bfloat16 *mask;  // [B][H][W][N]; zero the output where mask <= 0
    __nv_bfloat16 *out;         // [B][H][W][N]
    float *dw;                  // [9][Cout][Cin]
    float *wpart;               // wgrad partial tiles [ksplit][9][Cin][Cout] (FP32)
    int *err;
    unsigned long long budget_ns;
};

// Rows of a halo box: the 128 output pixels of a tile plus one on each side.
constexpr int TC_HALO_ROWS = 130;
// Shared-memory bytes of a conv pass with this plan: 1024 alignment slack,
// the resident weights, the ring, the full/empty/acc/drain/weight mbarriers
// and the TMEM base slot.
__host__ __device__ constexpr size_t tc_conv_smem(int wres_bytes, int stages, int stage_bytes) {
    return 1024 + (size_t)wres_bytes + (size_t)stages * stage_bytes + (2 * (size_t)stages + 8) * 8 + 16;
}

template <int N>
__host__ __device__ constexpr uint32_t tc_tmem_cols() {
    return 2 * N < 32 ? 32 : 2 * N;
}

// Stores 16 BF16 channels of pixel pairs (lanes 2i, 2i + 1) so that each
// store instruction writes whole 32-byte sectors: the even lane writes the
// first 16 bytes and the odd lane the second 16 bytes of one pixel, first
// for the even lane's pixel, then for the odd lane's.
__device__ __forceinline__ void store16_pairs(__nv_bfloat16 *pix_even, __nv_bfloat16 *pix_odd,
                                              bool in_even, bool in_odd, int lane, const uint4 &lo,
                                              const uint4 &hi) {
    const bool odd = lane & 1;
    const uint4 give = odd ? lo : hi;  // the half the partner lane needs
    uint4 got;
    got.x = __shfl_xor_sync(0xffffffffu, give.x, 1);
    got.y = __shfl_xor_sync(0xffffffffu, give.y, 1);
    got.z = __shfl_xor_sync(0xffffffffu, give.z, 1);
    got.w = __shfl_xor_sync(0xffffffffu, give.w, 1);
    const int half = odd ? 8 : 0;
    if (in_even) *reinterpret_cast<uint4 *>(pix_even + half) = odd ? got : lo;
    if (in_odd) *reinterpret_cast<uint4 *>(pix_odd + half) = odd ? hi : got;
}

template <int KC, int N>
__global__ void __launch_bounds__(192, N <= 128 ? 2 : 1)
    tc_conv_kernel(const __grid_constant__ CUtensorMap mapA0, const __grid_constant__ CUtensorMap mapA1,
                   const __grid_constant__ CUtensorMap mapB, TcConvParams p) {
    constexpr int SW = KC * 2;              // bytes of one operand row (the swizzle span)
    constexpr int BTAP = N * SW;            // one weight tile (N rows)
    constexpr uint32_t TMEM_COLS = tc_tmem_cols<N>();
    const int STAGES = p.stages;
    extern __shared__ unsigned char tc_smem_raw[];
    unsigned char *smem =
        (unsigned char *)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *wres = smem;                  // [9][nch] weight tiles (when p.wres)
    unsigned char *ring = smem + p.wres_bytes;   // STAGES slots of p.stage_bytes
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)STAGES * p.stage_bytes);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;   // [2]
    uint64_t *acc_empty = acc_full + 2;    // [2]
    uint64_t *drain = acc_empty + 2;       // [1]
    uint64_t *wbar = drain + 1;            // [1]
    uint32_t *tmem_base_slot = reinterpret_cast<uint32_t *>(wbar + 1);
    __shared__ int s_abort;
    __shared__ float s_bias[N];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);
        }
        mbar_init(drain, 1);
        mbar_init(wbar, 1);
        s_abort = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_base_slot, TMEM_COLS);
        tmem_relinquish();
    }
    // everything above is on-chip set-up; global memory only after the
    // predecessor kernel has completed (programmatic dependent launch)
    pdl_enter();
    for (int c = threadIdx.x; c < N; c += blockDim.x) s_bias[c] = p.bias ? p.bias[c] : 0.f;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_base_slot;
    const unsigned long long budget = p.budget_ns;
    volatile int *abort_flag = &s_abort;
    auto fail = [&](int code) {
        atomicCAS(p.err, 0, code);
        *abort_flag = 1;
    };
    const bool conv = p.mode == 0;
    const bool use_wres = conv && p.wres;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA
        if (lane == 0) {
            bool wres_loaded = false;
            if (use_wres) {
                // all 9 * nch weight tiles, once, on their own barrier
                mbar_arrive_expect_tx(wbar, (unsigned)(9 * p.nch * BTAP));
                for (int tap = 0; tap < 9; ++tap)
                    for (int ch = 0; ch < p.nch; ++ch)
                        tma_load_3d(wres + (size_t)(tap * p.nch + ch) * BTAP, &mapB, ch * KC, 0, tap, wbar);
                wres_loaded = true;
            }
            unsigned it = 0;
            for (int t = blockIdx.x; t < p.ntiles && !*abort_flag; t += gridDim.x) {
                int img = 0, y0 = 0, x0 = 0, g = 0, ct = 0;
                long long k0 = 0;
                int q0 = 0, q1 = 0;
                int wxc = 0, wy = 0, wim = 0;  // wgrad: x chunk, row and image of the next K step
                if (conv) {
                    const int pt = t / p.csplit, sp = t % p.csplit;
                    const int tx = pt % p.tiles_x, rest = pt / p.tiles_x;
                    x0 = tx * p.bx;
                    y0 = (rest % p.tiles_y) * p.by;
                    img = rest / p.tiles_y;
                    q0 = p.ksteps * sp / p.csplit;
                    q1 = p.ksteps * (sp + 1) / p.csplit;
                } else {
                    const int s = t % p.ksplit, rest = t / p.ksplit;
                    ct = rest % p.ci_tiles;
                    g = rest / p.ci_tiles;
                    k0 = p.total_k * s / p.ksplit;
                    q1 = (int)(p.total_k * ((t % p.ksplit) + 1) / p.ksplit - k0);
                    const int xchunks = p.W / KC;
                    wxc = (int)(k0 % xchunks);
                    const long long r2 = k0 / xchunks;
                    wy = (int)(r2 % p.H);
                    wim = (int)(r2 / p.H);
                }
                for (int q = q0; q < q1; ++q, ++it) {
                    const int st = it % STAGES;
                    if (!mbar_wait_bounded(&empty[st], ((it / STAGES) & 1) ^ 1, budget)) {
                        fail(1);
                        break;
                    }
                    unsigned char *a_dst = ring + (size_t)st * p.stage_bytes;
                    unsigned char *b_dst = a_dst + p.a_region;
                    if (conv && p.halo) {
                        const int ch = q / 3, dy = q % 3;
                        mbar_arrive_expect_tx(&full[st], TC_HALO_ROWS * SW + (use_wres ? 0 : 3 * BTAP));
                        tma_load_4d(a_dst, &mapA1, ch * KC, x0 - 1, y0 + dy - 1, img, &full[st]);
                        if (!use_wres)
                            for (int dx = 0; dx < 3; ++dx)
                                tma_load_3d(b_dst + dx * BTAP, &mapB, ch * KC, 0, dy * 3 + dx, &full[st]);
                    } else if (conv) {
                        const int tap = q / p.nch, ch = q % p.nch;
                        const int dy = tap / 3, dx = tap % 3;
                        mbar_arrive_expect_tx(&full[st], 128 * SW + (use_wres ? 0 : BTAP));
                        tma_load_4d(a_dst, &mapA0, ch * KC, x0 + dx - 1, y0 + dy - 1, img, &full[st]);
                        if (!use_wres) tma_load_3d(b_dst, &mapB, ch * KC, 0, tap, &full[st]);
                    } else {
                        const int px0 = wxc * KC, y = wy, im = wim;
                        if (++wxc == p.W / KC) {  // step along the row, then rows, then images
                            wxc = 0;
                            if (++wy == p.H) {
                                wy = 0;
                                ++wim;
                            }
                        }
                        int ntap = 9 - g * p.taps_per_tile;
                        if (ntap > p.taps_per_tile) ntap = p.taps_per_tile;
                        const unsigned bytes = (unsigned)ntap * p.ci_rows * KC * 2 + (unsigned)BTAP;
                        mbar_arrive_expect_tx(&full[st], bytes);
                        const int nab = p.ci_rows / p.a_cb;
                        const int abox = KC * p.a_cb * 2, bbox = KC * p.b_cb * 2;
                        for (int j = 0; j < ntap; ++j) {
                            const int tap = g * p.taps_per_tile + j;
                            const int dy = tap / 3, dx = tap % 3;
                            for (int b = 0; b < nab; ++b)
                                tma_load_4d(a_dst + (j * nab + b) * abox, &mapA0, ct * p.ci_rows + b * p.a_cb,
                                            px0 + dx - 1, y + dy - 1, im, &full[st]);
                        }
                        for (int b = 0; b < N / p.b_cb; ++b)
                            tma_load_4d(b_dst + b * bbox, &mapB, b * p.b_cb, px0, y, im, &full[st]);
                    }
                }
            }
            // let every issued load land before shared memory goes away
            const unsigned lo = it > (unsigned)STAGES ? it - STAGES : 0u;
            for (unsigned j = lo; j < it; ++j)
                mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, budget);
            if (wres_loaded) mbar_wait_bounded(wbar, 0, budget);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16_m128<N>();
            constexpr uint32_t idesc_mn = idesc_bf16_m128<N, true>();
            const uint32_t wres_addr = smem_u32(wres);
            bool ok = true;
            if (use_wres && !mbar_wait_bounded(wbar, 0, budget)) {
                fail(5);
                ok = false;
            }
            unsigned it = 0, lt = 0;
            for (int t = blockIdx.x; ok && t < p.ntiles && !*abort_flag; t += gridDim.x, ++lt) {
                const int ab = lt & 1;
                if (!mbar_wait_bounded(&acc_empty[ab], ((lt >> 1) & 1) ^ 1, budget)) {
                    fail(2);
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem + ab * N;
                int q0 = 0, q1;
                if (conv) {
                    const int sp = t % p.csplit;
                    q0 = p.ksteps * sp / p.csplit;
                    q1 = p.ksteps * (sp + 1) / p.csplit;
                } else {
                    q1 = (int)(p.total_k * ((t % p.ksplit) + 1) / p.ksplit -
                               p.total_k * (t % p.ksplit) / p.ksplit);
                }
                for (int q = q0; q < q1; ++q, ++it) {
                    const int st = it % STAGES;
                    if (!mbar_wait_bounded(&full[st], (it / STAGES) & 1, budget)) {
                        fail(3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(ring + (size_t)st * p.stage_bytes);
                    const uint32_t b_addr = a_addr + p.a_region;
                    if (conv && p.halo) {
                        // tap (dy, dx): A = rows dx .. dx + 127 of the halo box
                        const int ch = q / 3, dy = q % 3;
#pragma unroll
                        for (int dx = 0; dx < 3; ++dx) {
                            const uint32_t a0 = a_addr + dx * SW;
                            const uint32_t b0 =
                                use_wres ? wres_addr + (uint32_t)((dy * 3 + dx) * p.nch + ch) * BTAP
                                         : b_addr + dx * BTAP;
#pragma unroll
                            for (int kk = 0; kk < KC / 16; ++kk)
                                umma_bf16(d_tmem, kmajor_desc<SW>(a0 + kk * 32), kmajor_desc<SW>(b0 + kk * 32),
                                          idesc, (q > q0 || dx > 0 || kk > 0) ? 1u : 0u);
                        }
                    } else if (!conv) {
                        // MN-major: a K step of 16 pixels is 16 rows of each box
                        const uint32_t ra = p.a_cb * 2, rb = p.b_cb * 2;
#pragma unroll
                        for (int kk = 0; kk < KC / 16; ++kk)
                            umma_bf16(d_tmem, mnmajor_desc(a_addr + kk * 16 * ra, ra, KC * ra, 8 * ra),
                                      mnmajor_desc(b_addr + kk * 16 * rb, rb, KC * rb, 8 * rb), idesc_mn,
                                      (q > q0 || kk > 0) ? 1u : 0u);
                    } else {
                        uint32_t b0 = b_addr;
                        if (use_wres) {
                            const int tap = q / p.nch, ch = q % p.nch;
                            b0 = wres_addr + (uint32_t)(tap * p.nch + ch) * BTAP;
                        }
#pragma unroll
                        for (int kk = 0; kk < KC / 16; ++kk)
                            umma_bf16(d_tmem, kmajor_desc<SW>(a_addr + kk * 32), kmajor_desc<SW>(b0 + kk * 32),
                                      idesc, (q > q0 || kk > 0) ? 1u : 0u);
                    }
                    umma_commit(&empty[st]);  // frees the slot once these MMAs are done
                }
                if (!ok) break;
                umma_commit(&acc_full[ab]);
            }
            // wait for every MMA issued here before TMEM is freed
            umma_commit(drain);
            mbar_wait_bounded(drain, 0, budget);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------- epilogue
        const int q4 = warp & 3;  // TMEM lanes 32 q4 .. 32 q4 + 31
        const int row = q4 * 32 + lane;
        unsigned lt = 0;
        for (int t = blockIdx.x; t < p.ntiles && !*abort_flag; t += gridDim.x, ++lt) {
            const int ab = lt & 1;
            if (!mbar_wait_bounded(&acc_full[ab], (lt >> 1) & 1, budget)) {
                fail(4);
                break;
            }
            tc_fence_after();
            const uint32_t tbase = tmem + ((uint32_t)(q4 * 32) << 16) + ab * N;
            if (conv) {
                const int pt = t / p.csplit, sp = t % p.csplit;
                const int tx = pt % p.tiles_x, rest = pt / p.tiles_x;
                const int img = rest / p.tiles_y;
                // this lane's pixel and those of the even/odd lanes of its pair
                auto pixel = [&](int r, bool &in) {
                    const int x = tx * p.bx + r % p.bx;
                    const int y = (rest % p.tiles_y) * p.by + r / p.bx;
                    in = x < p.W && y < p.H;
                    return ((size_t)img * p.H + (in ? y : 0)) * p.W + (in ? x : 0);
                };
                bool in_me, in_e, in_o;
                const size_t pix = pixel(row, in_me);
                __nv_bfloat16 *oe = p.out + pixel(row & ~1, in_e) * N;
                __nv_bfloat16 *oo = p.out + pixel(row | 1, in_o) * N;
                const __nv_bfloat16 *mk = p.mask ? p.mask + pix * N : nullptr;
                float *wsrow = p.csplit > 1
                                   ? p.ws + ((size_t)sp * p.B * p.H * p.W + pix) * N
                                   : nullptr;
                auto emit16 = [&](int c, const float *acc) {
                    if (wsrow) {  // split-K partial: FP32, the reduction applies the epilogue
                        if (in_me) {
                            float4 *d = reinterpret_cast<float4 *>(wsrow + c);
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                d[j] = make_float4(acc[4 * j], acc[4 * j + 1], acc[4 * j + 2], acc[4 * j + 3]);
                        }
                        return;
                    }
                    float v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        v[j] = acc[j] + s_bias[c + j];
                        if (p.relu) v[j] = fmaxf(v[j], 0.f);
                    }
                    if (mk && in_me) {
                        const uint4 m0 = reinterpret_cast<const uint4 *>(mk + c)[0];
                        const uint4 m1 = reinterpret_cast<const uint4 *>(mk + c)[1];
                        const __nv_bfloat16 *mb0 = reinterpret_cast<const __nv_bfloat16 *>(&m0);
                        const __nv_bfloat16 *mb1 = reinterpret_cast<const __nv_bfloat16 *>(&m1);
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            if (!(__bfloat162float(mb0[j]) > 0.f)) v[j] = 0.f;
                            if (!(__bfloat162float(mb1[j]) > 0.f)) v[8 + j] = 0.f;
                        }
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
                };
                if constexpr (N <= 64) {
                    // narrow tile: drain TMEM first and hand the accumulator back
                    // to the MMA warp before the global stores
                    float accall[N];
#pragma unroll
                    for (int c = 0; c < N; c += 16) tmem_ld16(tbase + c, accall + c);
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[ab]);
#pragma unroll
                    for (int c = 0; c < N; c += 16) emit16(c, accall + c);
                    continue;
                } else {
#pragma unroll 1
                    for (int c = 0; c < N; c += 16) {
                        float acc[16];
                        tmem_ld16(tbase + c, acc);
                        emit16(c, acc);
                    }
                }
            } else {
                const int rest = t / p.ksplit;
                const int ct = rest % p.ci_tiles, g = rest / p.ci_tiles;
                const int j = row / p.ci_rows;
                const int tap = g * p.taps_per_tile + j;
                const int ci = ct * p.ci_rows + row % p.ci_rows;
                const bool in = j < p.taps_per_tile && tap < 9 && ci < p.Cin;
                // this split's partial row (tap, ci): Cout consecutive floats
                float *d = p.wpart + (((size_t)(t % p.ksplit) * 9 + (in ? tap : 0)) * p.Cin + ci) * p.Cout;
#pragma unroll 1
                for (int c = 0; c < N; c += 16) {
                    float acc[16];
                    tmem_ld16(tbase + c, acc);
                    if (in && c + 16 <= p.Cout) {
                        float4 *d4 = reinterpret_cast<float4 *>(d + c);
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            d4[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
                    }
                }
            }
            // accumulator drained: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[ab]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace cfm

namespace cfm {

// Weight-gradient splits of tc_conv_kernel: dw[tap][co][ci] += the sum of
// part[s][tap][ci][co] over the splits s, in a fixed order (the same sum on
// every run).  A block takes WR_ENTRIES consecutive partial entries and
// splits the ksplit splits into WR_CHUNKS chunks, one thread per (entry,
// chunk): a chunk is summed with four accumulators (split s into s mod 4,
// combined as (a0 + a1) + (a2 + a3)), then the chunks are added in order.
// Reads are coalesced over the entries of a split.
constexpr int WR_ENTRIES = 32, WR_CHUNKS = 8;
__global__ void __launch_bounds__(WR_ENTRIES * WR_CHUNKS)
    tc_wgrad_reduce(const float *part, int ksplit, int Cin, int Cout, float *dw) {
    pdl_enter();
    __shared__ float sc[WR_CHUNKS][WR_ENTRIES];
    const long long n = 9LL * Cin * Cout;
    const int el = threadIdx.x % WR_ENTRIES, q = threadIdx.x / WR_ENTRIES;
    const long long e = (long long)blockIdx.x * WR_ENTRIES + el;
    float v = 0.f;
    if (e < n) {
        const int s0 = ksplit * q / WR_CHUNKS, s1 = ksplit * (q + 1) / WR_CHUNKS;
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        int sp = s0;
        for (; sp + 3 < s1; sp += 4) {
            a0 += part[(size_t)sp * n + e];
            a1 += part[(size_t)(sp + 1) * n + e];
            a2 += part[(size_t)(sp + 2) * n + e];
            a3 += part[(size_t)(sp + 3) * n + e];
        }
        for (; sp < s1; ++sp) a0 += part[(size_t)sp * n + e];
        v = (a0 + a1) + (a2 + a3);
    }
    sc[q][el] = v;
    __syncthreads();
    if (q == 0 && e < n) {
        float t = 0.f;
        for (int c = 0; c < WR_CHUNKS; ++c) t += sc[c][el];
        const int co = (int)(e % Cout);
        const long long r = e / Cout;
        const int ci = (int)(r % Cin), tap = (int)(r / Cin);
        dw[((size_t)tap * Cout + co) * Cin + ci] += t;
    }
}

// Split-K reduction and epilogue of tc_conv_kernel: out[p][c] =
// act(sum_j ws[j][p][c] + bias[c]) [* (mask > 0)], the partials summed in
// split order (deterministic).  One thread per (pixel, 8 channels).
template <int N>
__global__ void tc_splitk_epilogue(const float *ws, int csplit, long long npix, const float *bias, int relu,
                                   const __nv_bfloat16 *mask, __nv_bfloat16 *out) {
    pdl_enter();
    constexpr int G = N / 8;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < npix * G;
         e += (long long)gridDim.x * blockDim.x) {
        const long long pix = e / G;
        const int c = (int)(e % G) * 8;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.f;
        for (int sp = 0; sp < csplit; ++sp) {
            const float4 *src = reinterpret_cast<const float4 *>(ws + ((size_t)sp * npix + pix) * N + c);
            const float4 a = src[0], b = src[1];
            v[0] += a.x, v[1] += a.y, v[2] += a.z, v[3] += a.w;
            v[4] += b.x, v[5] += b.y, v[6] += b.z, v[7] += b.w;
        }
        uint4 m = make_uint4(0u, 0u, 0u, 0u);
        if (mask) m = *reinterpret_cast<const uint4 *>(mask + pix * N + c);
        const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&m);
        uint4 o;
        __nv_bfloat162 *o2 = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            float a = v[j] + (bias ? bias[c + j] : 0.f), b = v[j + 1] + (bias ? bias[c + j + 1] : 0.f);
            if (relu) a = fmaxf(a, 0.f), b = fmaxf(b, 0.f);
            if (mask) {
                if (!(__bfloat162float(mb[j]) > 0.f)) a = 0.f;
                if (!(__bfloat162float(mb[j + 1]) > 0.f)) b = 0.f;
            }
            o2[j / 2] = __floats2bfloat162_rn(a, b);
        }
        *reinterpret_cast<uint4 *>(out + pix * N + c) = o;
    }
}

}  // namespace cfm
