// 3D Jacobi sweep fed by the tensor memory accelerator (TMA), persistent.
//
// Work units, their order and the arithmetic are those of j3d_sweeps_kernel
// (jacobi.cu): units (z-chunk, tile) dealt round-robin to the blocks, sum
// order ((((E + W) + N) + S) + T) + B times fl(1/6).  What changes is how the
// data arrives: one producer warp streams each plane of the current unit's
// tile, with its x and y halos, into a ring of STAGES shared-memory buffers
// by cp.async.bulk.tensor (box (32 VN + 2 VN) x (TY + 2) x 1, x starting VN
// elements early so the box is 16-byte aligned; out-of-range cells read as
// zero and are never used).  CW consumer warps each own RPW rows of the tile
// and VN consecutive points per lane (one 16-byte vector); they keep the z-1
// and z values of their points in registers, read the z+1 plane and the
// N/S/E/W neighbours from shared memory, and store the new values straight to
// global memory.  A stage is released (a proxy fence by every consumer lane,
// then one mbarrier arrive per consumer warp) after the last step that reads
// it, so up to STAGES planes are in flight per block.  All mbarrier and grid-barrier waits are bounded.
//
// Sweeps are ordered either by a grid barrier after each sweep (udone null)
// or, with udone (one counter per unit, zero at launch), by the units'
// neighbourhoods alone: when the consumers of a block finish unit u of
// sweep t they set udone[u] = t + 1 (release, after a consumer-only barrier
// that also ORs their error flags), and the producer loads unit u of sweep
// t only after every unit of its 3 x 3 x 3 neighbourhood -- chunks and
// tiles at distance one, z chunks wrapping around and y tiles too when y is
// periodic, since those write the periodic images u reads -- has reached t
// (27 lanes poll one neighbour each; bounded).  Those neighbours are all of
// u's readers and writers in sweep t - 1, so both the values u reads and
// the cells it overwrites are settled, and a block that finishes a sweep
// early goes straight on with its next unit instead of waiting for the
// slowest block.  Every wait is on an earlier sweep, so the units complete
// in (sweep, unit) order at worst and the waits cannot form a cycle.
#pragma once

#include "barrier.cuh"
#include "tma.cuh"

namespace cfm {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
    using type = double2;
    static constexpr int N = 2;
};
template <>
struct Vec16<float> {
    using type = float4;
    static constexpr int N = 4;
};

template <typename T, int CW, int RPW, int STAGES>
struct TmaGeom {
    static constexpr int VN = Vec16<T>::N;
    static constexpr int TY = CW * RPW;
    static constexpr int TX = 32 * VN;
    static constexpr int BXW = TX + 2 * VN;
    static constexpr int BYH = TY + 2;
    static constexpr unsigned TX_BYTES = BXW * BYH * sizeof(T);
    static constexpr unsigned STRIDE = (TX_BYTES + 127) / 128 * 128;
    static constexpr size_t SMEM = (size_t)STAGES * STRIDE + 2 * STAGES * sizeof(uint64_t);
    static constexpr int THREADS = 32 * (CW + 1);
};

// Consumer-warp barrier (named barrier 1, `nthreads` threads) that also
// returns the OR of every participant's `pred`.
__device__ __forceinline__ int bar_red_or(int nthreads, int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\t"
        "selp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(pred), "r"(nthreads)
        : "memory");
    return r;
}

__device__ __forceinline__ unsigned int ld_relaxed_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ double tma_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float tma_add(float a, float b) { return __fadd_rn(a, b); }

__device__ __forceinline__ double tma_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float tma_mul(float a, float b) { return __fmul_rn(a, b); }

template <typename T, int CW, int RPW, int STAGES, bool PY>
__global__ void __launch_bounds__(32 * (CW + 1))
    j3d_tma_kernel(const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
                   T *g0, T *g1, int nx, int ny, int nz, int niter, int zchunk, BarrierState *bar,
                   unsigned int *udone) {
    using G = TmaGeom<T, CW, RPW, STAGES>;
    using V = typename Vec16<T>::type;
    constexpr int VN = G::VN, TX = G::TX, BXW = G::BXW, TY = G::TY;
    extern __shared__ __align__(128) unsigned char tsm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(tsm + STAGES * G::STRIDE);
    uint64_t *empty = full + STAGES;
    __shared__ int s_err;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CW);
        }
        s_err = 0;
        mbar_fence_init();
    }
    __syncthreads();

    const int ntx = (nx + TX - 1) / TX;
    const int nty = (ny - 2 + TY - 1) / TY;
    const long long ntiles = (long long)ntx * nty;
    const int nzi = nz - 2;
    const int nch = (nzi + zchunk - 1) / zchunk;
    const long long U = ntiles * nch;
    const long long NB = gridDim.x;
    const unsigned long long budget = bar->timeout_ns;
    const size_t P = (size_t)nx * ny;
    const size_t zimg = (size_t)(nz - 2) * P;
    const size_t yimg = (size_t)(ny - 2) * nx;
    const T c6 = T(1) / T(6);
    unsigned k = 0;  // plane loads issued (producer) / consumed (consumers) so far

    int cerr = 0;  // consumers: an error seen by any consumer warp (dataflow order)
    for (int it = 0; it < niter; ++it) {
        const CUtensorMap *tm = (it & 1) ? &tm1 : &tm0;
        T *out = (it & 1) ? g0 : g1;
        if (warp == CW) {
            // ---------------------------------------------------- producer
            if (lane == 0) fence_proxy_async_global();
            for (long long u = blockIdx.x; u < U; u += NB) {
                if (__shfl_sync(0xffffffffu, lane == 0 ? *(volatile int *)&s_err : 0, 0)) break;
                const int ch = (int)(u / ntiles), tile = (int)(u - ch * ntiles);
                if (udone && it > 0) {
                    // the unit's neighbourhood must have finished sweep it - 1
                    const int tx = tile % ntx, ty = tile / ntx;
                    long long nb = -1;
                    if (lane < 27) {
                        int c2 = ch + lane / 9 - 1, y2 = ty + (lane / 3) % 3 - 1;
                        const int x2 = tx + lane % 3 - 1;
                        c2 = c2 < 0 ? nch - 1 : (c2 >= nch ? 0 : c2);
                        bool valid = x2 >= 0 && x2 < ntx;
                        if (PY) y2 = y2 < 0 ? nty - 1 : (y2 >= nty ? 0 : y2);
                        else valid = valid && y2 >= 0 && y2 < nty;
                        if (valid) nb = (long long)c2 * ntiles + (long long)y2 * ntx + x2;
                    }
                    const unsigned long long t0 = global_ns();
                    bool waited_out = false;
                    for (;;) {
                        const bool ready = nb < 0 || ld_relaxed_u32(udone + nb) >= (unsigned)it;
                        if (__all_sync(0xffffffffu, ready)) break;
                        const bool stop = lane == 0 && (global_ns() - t0 > budget || ld_relaxed_i32(&bar->error));
                        if (__shfl_sync(0xffffffffu, stop, 0)) {
                            waited_out = true;
                            break;
                        }
                    }
                    if (waited_out) {
                        if (lane == 0) {
                            if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = 3000000 + it;
                            s_err = 1;
                        }
                        break;
                    }
                    __threadfence();  // acquire the neighbours' stores ...
                    if (lane == 0) fence_proxy_async_global();  // ... for the TMA reads below
                }
                if (lane == 0) {
                    const int x0 = (tile % ntx) * TX, y0 = 1 + (tile / ntx) * TY;
                    const int z0 = 1 + ch * zchunk, z1 = min(z0 + zchunk, nz - 1);
                    for (int z = z0 - 1; z <= z1; ++z) {
                        const int s = k % STAGES;
                        if (!mbar_wait_bounded(&empty[s], ((k / STAGES) & 1) ^ 1, budget)) {
                            if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = 1000000 + it;
                            s_err = 1;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[s], G::TX_BYTES);
                        tma_load_3d(tsm + s * G::STRIDE, tm, x0 - VN, y0 - 1, z, &full[s]);
                        ++k;
                    }
                }
                __syncwarp();
            }
            __syncwarp();
            if (udone && __shfl_sync(0xffffffffu, lane == 0 ? *(volatile int *)&s_err : 0, 0)) break;
        } else {
            // ---------------------------------------------------- consumers
            for (long long u = blockIdx.x; u < U; u += NB) {
                const int ch = (int)(u / ntiles), tile = (int)(u - ch * ntiles);
                const int x0 = (tile % ntx) * TX, y0 = 1 + (tile / ntx) * TY;
                const int z0 = 1 + ch * zchunk, z1 = min(z0 + zchunk, nz - 1);
                const int xb = x0 + lane * VN;
                const int r0 = warp * RPW;  // first tile row of this warp
                // smem offset of this lane's first element in tile row r0
                const int own0 = (r0 + 1) * BXW + VN + lane * VN;
                const bool full_vec = xb >= 1 && xb + VN - 1 <= nx - 2;
                bool row_ok[RPW];
                size_t gbase[RPW];
#pragma unroll
                for (int j = 0; j < RPW; ++j) {
                    const int y = y0 + r0 + j;
                    row_ok[j] = y <= ny - 2;
                    gbase[j] = (size_t)(row_ok[j] ? y : 1) * nx + xb;
                }
                T prev[RPW][VN], cur[RPW][VN];
                bool ok = true;
                {  // plane z0 - 1: own values only
                    const int s = k % STAGES;
                    ok = mbar_wait_bounded(&full[s], (k / STAGES) & 1, budget);
                    const T *pp = reinterpret_cast<const T *>(tsm + s * G::STRIDE);
#pragma unroll
                    for (int j = 0; j < RPW; ++j) {
                        const V v = *reinterpret_cast<const V *>(pp + own0 + j * BXW);
                        memcpy(prev[j], &v, sizeof(v));
                    }
                    fence_proxy_async_shared();  // reads of the slot before its refill
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[s]);
                    ++k;
                }
                int scur = k % STAGES;
                if (ok) ok = mbar_wait_bounded(&full[scur], (k / STAGES) & 1, budget);
                {
                    const T *pc = reinterpret_cast<const T *>(tsm + scur * G::STRIDE);
#pragma unroll
                    for (int j = 0; j < RPW; ++j) {
                        const V v = *reinterpret_cast<const V *>(pc + own0 + j * BXW);
                        memcpy(cur[j], &v, sizeof(v));
                    }
                }
                ++k;
                size_t zoff = (size_t)z0 * P;
                for (int z = z0; z < z1 && ok; ++z, zoff += P) {
                    const int snx = k % STAGES;
                    if (!mbar_wait_bounded(&full[snx], (k / STAGES) & 1, budget)) {
                        ok = false;
                        break;
                    }
                    ++k;
                    const T *pc = reinterpret_cast<const T *>(tsm + scur * G::STRIDE) + own0;
                    const T *pn = reinterpret_cast<const T *>(tsm + snx * G::STRIDE) + own0;
                    T nxt[RPW][VN], nn[RPW][VN], ss[RPW][VN], wl[RPW], er[RPW];
#pragma unroll
                    for (int j = 0; j < RPW; ++j) {
                        const V a = *reinterpret_cast<const V *>(pn + j * BXW);
                        const V b = *reinterpret_cast<const V *>(pc + (j + 1) * BXW);
                        const V c = *reinterpret_cast<const V *>(pc + (j - 1) * BXW);
                        memcpy(nxt[j], &a, sizeof(a));
                        memcpy(nn[j], &b, sizeof(b));
                        memcpy(ss[j], &c, sizeof(c));
                        wl[j] = pc[j * BXW - 1];
                        er[j] = pc[j * BXW + VN];
                    }
                    fence_proxy_async_shared();  // reads of the slot before its refill
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[scur]);
                    const bool zspecial = (z == 1) || (z == nz - 2);
#pragma unroll
                    for (int j = 0; j < RPW; ++j) {
                        T res[VN];
#pragma unroll
                        for (int i = 0; i < VN; ++i) {
                            const T e = (i == VN - 1) ? er[j] : cur[j][i + 1];
                            const T w = (i == 0) ? wl[j] : cur[j][i - 1];
                            T s = tma_add(e, w);
                            s = tma_add(s, nn[j][i]);
                            s = tma_add(s, ss[j][i]);
                            s = tma_add(s, nxt[j][i]);
                            s = tma_add(s, prev[j][i]);
                            res[i] = tma_mul(c6, s);
                        }
                        if (row_ok[j]) {
                            const size_t idx = zoff + gbase[j];
                            V v;
                            memcpy(&v, res, sizeof(v));
                            if (full_vec) {
                                // evict-first: the output must not push the input
                                // planes other tiles still need out of L2
                                __stcs(reinterpret_cast<V *>(out + idx), v);
                            } else {
#pragma unroll
                                for (int i = 0; i < VN; ++i)
                                    if (xb + i >= 1 && xb + i <= nx - 2) __stcs(out + idx + i, res[i]);
                            }
                            const int y = y0 + r0 + j;
                            const bool yspecial = PY && (y == 1 || y == ny - 2);
                            if (zspecial || yspecial) {
                                // periodic images of this value (see the file comment of jacobi.cu)
                                auto put = [&](size_t at) {
                                    if (full_vec) {
                                        *reinterpret_cast<V *>(out + at) = v;
                                    } else {
#pragma unroll
                                        for (int i = 0; i < VN; ++i)
                                            if (xb + i >= 1 && xb + i <= nx - 2) out[at + i] = res[i];
                                    }
                                };
                                const bool zlo = z == 1, zhi = z == nz - 2;
                                const bool ylo = PY && y == 1, yhi = PY && y == ny - 2;
                                if (zlo) put(idx + zimg);
                                if (zhi) put(idx - zimg);
                                if (ylo) {
                                    put(idx + yimg);
                                    if (zlo) put(idx + yimg + zimg);
                                    if (zhi) put(idx + yimg - zimg);
                                }
                                if (yhi) {
                                    put(idx - yimg);
                                    if (zlo) put(idx - yimg + zimg);
                                    if (zhi) put(idx - yimg - zimg);
                                }
                            }
                        }
#pragma unroll
                        for (int i = 0; i < VN; ++i) {
                            prev[j][i] = cur[j][i];
                            cur[j][i] = nxt[j][i];
                        }
                    }
                    scur = snx;
                }
                fence_proxy_async_shared();  // reads of the slot before its refill
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[scur]);
                if (udone) {
                    // the unit's stores, then one consumer barrier: publish
                    // the unit, or leave together if any consumer failed
                    __threadfence();
                    cerr = bar_red_or(32 * CW, !ok);
                    if (!cerr && warp == 0 && lane == 0) st_release_gpu_u32(udone + u, (unsigned)(it + 1));
                    if (cerr) {
                        if (!ok && lane == 0) {
                            if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = 2000000 + it;
                            s_err = 1;
                        }
                        break;
                    }
                } else if (!ok) {
                    if (lane == 0) {
                        if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = 2000000 + it;
                        s_err = 1;
                    }
                    break;
                }
            }
            if (cerr) break;
        }
        if (!udone && it + 1 < niter) {
            if (!grid_barrier(bar, gridDim.x, it)) break;
        }
    }
    // On an error exit, let the loads this block issued land before its
    // shared memory is released (bounded).
    if (warp == CW && lane == 0 && s_err) {
        const unsigned lo = k > (unsigned)STAGES ? k - STAGES : 0u;
        for (unsigned j = lo; j < k; ++j) mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, budget);
    }
}

}  // namespace cfm
