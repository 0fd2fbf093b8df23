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
//    channel, k = (tap, input channel chunk).  A tile for tap (dy, dx) is the
//    activation box at (c0, x0 + dx - 1, y0 + dy - 1, img) of the NHWC tensor;
//    coordinates outside the image read as zero, which is the padding.
//    Epilogue: + bias, optional ReLU, optional mask (zero where mask <= 0),
//    BF16 store NHWC.
//  weight gradient:
//    m = (tap of a tap group, input channel), n = output channel, k = pixels
//    (KC consecutive x of one row per step).  A rows come from x-shifted
//    channel-major copies of the layer input (XT_dx[img][c][y][x] =
//    X[img][y][x + dx - 1][c]; the y shift is a TMA coordinate), B rows from
//    the channel-major output gradient.  Tiles split K; the epilogue adds
//    its partial tile to dW[tap][co][ci] (FP32 atomics).
//
// One persistent CTA per SM, 6 warps: warp 0 issues TMA (one elected lane),
// warp 1 owns TMEM and issues tcgen05.mma (one lane), warps 2-5 drain the
// accumulator (tcgen05.ld, 32 TMEM lanes each).  A ring of STAGES operand
// buffers (full/empty mbarriers) and two TMEM accumulators (acc_full /
// acc_empty) overlap loads, MMAs and the epilogue of the previous tile.
// Every wait is bounded; on a timeout the CTA records an error, lets its
// in-flight copies and MMAs land (bounded), frees TMEM and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

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

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28 (M = 128).
template <int N>
__host__ __device__ constexpr uint32_t idesc_bf16_m128() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(128 >> 4) << 24);
}

struct TcConvParams {
    int mode;  // 0 conv, 1 weight gradient
    int B, H, W;
    int Cin, Cout;  // of the convolution this pass belongs to (conv mode: Cin -> Cout = N)
    int ntiles;
    int ksteps;  // conv: 9 * Cin / KC; wgrad: steps per split
    // conv mode tiling
    int bx, by, tiles_x, tiles_y;
    // wgrad mode tiling
    int ci_rows, ci_tiles, taps_per_tile, tap_groups, ksplit;
    long long total_k;  // B * H * (W / KC)
    // epilogue
    const float *bias;
    int relu;
    const __nv_bfloat16 *mask;  // [B][H][W][N]; zero the output where mask <= 0
    __nv_bfloat16 *out;         // [B][H][W][N]
    float *dw;                  // [9][Cout][Cin]
    int *err;
    unsigned long long budget_ns;
};

template <int KC, int N>
struct TcGeom {
    static constexpr int SW = KC * 2;
    static constexpr int A_BYTES = 128 * SW;
    static constexpr int B_BYTES = N * SW;
    static constexpr int STAGE = (A_BYTES + B_BYTES + 1023) / 1024 * 1024;
    // Narrow tiles (N <= 64) keep the ring near 100 KB so two CTAs share an
    // SM (two independent load / MMA / epilogue pipelines, 2 x 2N TMEM
    // columns); wide ones take up to 200 KB alone.  At most 16 stages.
    static constexpr int BUDGET = (N <= 64 ? 100 : 200) * 1024;
    static constexpr int STAGES = BUDGET / STAGE > 16 ? 16 : BUDGET / STAGE;
    // + 1024 alignment slack + full/empty/acc/drain mbarriers and the TMEM base slot
    static constexpr size_t SMEM = (size_t)STAGES * STAGE + 1024 + (2 * STAGES + 8) * 8;
    static constexpr uint32_t TMEM_COLS = 2 * N < 32 ? 32 : 2 * N;
};

template <int KC, int N>
__global__ void __launch_bounds__(192, N <= 64 ? 2 : 1)
    tc_conv_kernel(const __grid_constant__ CUtensorMap mapA0, const __grid_constant__ CUtensorMap mapA1,
                   const __grid_constant__ CUtensorMap mapA2, const __grid_constant__ CUtensorMap mapB,
                   TcConvParams p) {
    using G = TcGeom<KC, N>;
    constexpr int STAGES = G::STAGES;
    extern __shared__ unsigned char tc_smem_raw[];
    unsigned char *smem =
        (unsigned char *)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * G::STAGE);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;   // [2]
    uint64_t *acc_empty = acc_full + 2;    // [2]
    uint64_t *drain = acc_empty + 2;       // [1]
    uint32_t *tmem_base_slot = reinterpret_cast<uint32_t *>(drain + 1);
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
        s_abort = 0;
        mbar_fence_init();
    }
    for (int c = threadIdx.x; c < N; c += blockDim.x) s_bias[c] = p.bias ? p.bias[c] : 0.f;
    if (warp == 1) {
        tmem_alloc(tmem_base_slot, G::TMEM_COLS);
        tmem_relinquish();
    }
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

    if (warp == 0) {
        // ------------------------------------------------------------ TMA
        if (lane == 0) {
            unsigned it = 0;
            for (int t = blockIdx.x; t < p.ntiles && !*abort_flag; t += gridDim.x) {
                int img = 0, y0 = 0, x0 = 0, g = 0, ct = 0;
                long long k0 = 0;
                if (p.mode == 0) {
                    const int tx = t % p.tiles_x, rest = t / p.tiles_x;
                    x0 = tx * p.bx;
                    y0 = (rest % p.tiles_y) * p.by;
                    img = rest / p.tiles_y;
                } else {
                    const int s = t % p.ksplit, rest = t / p.ksplit;
                    ct = rest % p.ci_tiles;
                    g = rest / p.ci_tiles;
                    k0 = p.total_k * s / p.ksplit;
                }
                const int nsteps = p.mode == 0 ? p.ksteps
                                               : (int)(p.total_k * ((t % p.ksplit) + 1) / p.ksplit - k0);
                for (int q = 0; q < nsteps; ++q, ++it) {
                    const int st = it % STAGES;
                    if (!mbar_wait_bounded(&empty[st], ((it / STAGES) & 1) ^ 1, budget)) {
                        fail(1);
                        break;
                    }
                    unsigned char *a_dst = smem + st * G::STAGE;
                    unsigned char *b_dst = a_dst + G::A_BYTES;
                    if (p.mode == 0) {
                        const int nch = p.Cin / KC;
                        const int tap = q / nch, c0 = (q % nch) * KC;
                        const int dy = tap / 3, dx = tap % 3;
                        mbar_arrive_expect_tx(&full[st], G::A_BYTES + G::B_BYTES);
                        tma_load_4d(a_dst, &mapA0, c0, x0 + dx - 1, y0 + dy - 1, img, &full[st]);
                        tma_load_3d(b_dst, &mapB, c0, 0, tap, &full[st]);
                    } else {
                        const long long kq = k0 + q;
                        const int xchunks = p.W / KC;
                        const int xc = (int)(kq % xchunks);
                        const long long r2 = kq / xchunks;
                        const int y = (int)(r2 % p.H), im = (int)(r2 / p.H);
                        int ntap = 9 - g * p.taps_per_tile;
                        if (ntap > p.taps_per_tile) ntap = p.taps_per_tile;
                        const unsigned bytes =
                            (unsigned)ntap * p.ci_rows * KC * 2 + (unsigned)G::B_BYTES;
                        mbar_arrive_expect_tx(&full[st], bytes);
                        for (int j = 0; j < ntap; ++j) {
                            const int tap = g * p.taps_per_tile + j;
                            const int dy = tap / 3, dx = tap % 3;
                            const CUtensorMap *m = dx == 0 ? &mapA0 : (dx == 1 ? &mapA1 : &mapA2);
                            tma_load_4d(a_dst + j * p.ci_rows * KC * 2, m, xc * KC, y + dy - 1,
                                        ct * p.ci_rows, im, &full[st]);
                        }
                        tma_load_4d(b_dst, &mapB, xc * KC, y, 0, im, &full[st]);
                    }
                }
            }
            // let every issued load land before shared memory goes away
            const unsigned lo = it > (unsigned)STAGES ? it - STAGES : 0u;
            for (unsigned j = lo; j < it; ++j)
                mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, budget);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16_m128<N>();
            unsigned it = 0, lt = 0;
            for (int t = blockIdx.x; t < p.ntiles && !*abort_flag; t += gridDim.x, ++lt) {
                const int ab = lt & 1;
                if (!mbar_wait_bounded(&acc_empty[ab], ((lt >> 1) & 1) ^ 1, budget)) {
                    fail(2);
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem + ab * N;
                const int nsteps =
                    p.mode == 0 ? p.ksteps
                                : (int)(p.total_k * ((t % p.ksplit) + 1) / p.ksplit -
                                        p.total_k * (t % p.ksplit) / p.ksplit);
                bool ok = true;
                for (int q = 0; q < nsteps; ++q, ++it) {
                    const int st = it % STAGES;
                    if (!mbar_wait_bounded(&full[st], (it / STAGES) & 1, budget)) {
                        fail(3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + st * G::STAGE);
                    const uint32_t b_addr = a_addr + G::A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < KC / 16; ++kk) {
                        umma_bf16(d_tmem, kmajor_desc<G::SW>(a_addr + kk * 32),
                                  kmajor_desc<G::SW>(b_addr + kk * 32), idesc,
                                  (q > 0 || kk > 0) ? 1u : 0u);
                    }
                    umma_commit(&empty[st]);  // frees the stage once these MMAs are done
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
            if (p.mode == 0) {
                const int tx = t % p.tiles_x, rest = t / p.tiles_x;
                const int x = tx * p.bx + row % p.bx;
                const int y = (rest % p.tiles_y) * p.by + row / p.bx;
                const int img = rest / p.tiles_y;
                const bool in = x < p.W && y < p.H;
                const size_t pix = ((size_t)img * p.H + (in ? y : 0)) * p.W + (in ? x : 0);
                __nv_bfloat16 *o = p.out + pix * N;
                const __nv_bfloat16 *mk = p.mask ? p.mask + pix * N : nullptr;
                auto emit16 = [&](int c, const float *acc) {
                    if (!in) return;
                    __align__(16) __nv_bfloat16 v16[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        float v = acc[j] + s_bias[c + j];
                        if (p.relu) v = fmaxf(v, 0.f);
                        if (mk && !(__bfloat162float(mk[c + j]) > 0.f)) v = 0.f;
                        v16[j] = __float2bfloat16_rn(v);
                    }
                    reinterpret_cast<uint4 *>(o + c)[0] = reinterpret_cast<const uint4 *>(v16)[0];
                    reinterpret_cast<uint4 *>(o + c)[1] = reinterpret_cast<const uint4 *>(v16)[1];
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
                float *d = p.dw + (size_t)(in ? tap : 0) * p.Cout * p.Cin + ci;
#pragma unroll 1
                for (int c = 0; c < N; c += 16) {
                    float acc[16];
                    tmem_ld16(tbase + c, acc);
                    if (in) {
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj)
                            if (c + jj < p.Cout) atomicAdd(d + (size_t)(c + jj) * p.Cin, acc[jj]);
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
        tmem_dealloc(tmem, G::TMEM_COLS);
    }
}

}  // namespace cfm
