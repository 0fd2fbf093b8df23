// 3D Jacobi, two sweeps per pass over the grid (temporal blocking), fed by
// the tensor memory accelerator, persistent.
//
// Same units, unit order and per-sweep arithmetic as j3d_tma_kernel (sum
// order ((((E + W) + N) + S) + T) + B times fl(1/6)), so every sweep is bit
// for bit the reference's; what changes is that each pass reads the grid once
// and writes it once for two sweeps.  For output planes [z0, z1) of a tile,
// the consumers first compute sweep-1 values on the tile plus a one-cell ring
// for planes z0 - 1 .. z1 ("windows", one per plane, each reading three input
// planes) into a three-plane ring in shared memory, then sweep 2 of plane
// p - 1 from the ring as soon as window p is done.
//
// Periodic images.  Rows y = 0, ny - 1 (periodic y) and planes z = 0,
// nz - 1 hold copies of the opposite interior values; the x faces are fixed.
// A sweep-1 value at an image cell is the sweep-1 value of its source cell,
// computed from the source's own neighbourhood (a copy of the neighbourhood
// would differ at the fixed x faces):
//  - window p = 0 reads input planes nz - 3 .. nz - 1 (source plane nz - 2),
//    window p = nz - 1 reads planes 0 .. 2 (source plane 1); the producer
//    streams those planes as a fresh three-plane window;
//  - tiles that need sweep-1 row 0 (y0 = 1) or row ny - 1 also load, per
//    plane, the three source rows ny - 3 .. ny - 1 or 0 .. 2 into extra rows
//    of the stage.
// Without periodic y, rows 0 and ny - 1 are fixed like the x faces.
//
// One producer warp streams planes (box (32 VN + 2 VN) x (TY + 4), x
// starting VN elements early so it is 16-byte aligned, rows y0 - 2 ..
// y0 + TY + 1; out-of-range cells read as zero and are never used) into a
// ring of STAGES stages; CW consumer warps share the windows through named
// barriers.  Every mbarrier and grid-barrier wait is bounded; after a
// timeout the consumers skip the remaining waits, finish their loops
// without meaning (the result is reported invalid) and leave together.
#pragma once

#include "barrier.cuh"
#include "j3d_tma.cuh"
#include "tma.cuh"

namespace cfm {

template <typename T, int CW, int RPW, int STAGES>
struct Tma2Geom {
    static constexpr int VN = Vec16<T>::N;
    static constexpr int TY = CW * RPW;
    static constexpr int TX = 32 * VN;
    static constexpr int BXW = TX + 2 * VN;  // columns x0 - VN .. x0 + TX + VN - 1
    static constexpr int BYH = TY + 4;       // rows y0 - 2 .. y0 + TY + 1
    static constexpr int XR = 3;             // rows of one far-row box
    static constexpr unsigned MAIN_BYTES = BXW * BYH * sizeof(T);
    static constexpr unsigned XR_BYTES = BXW * XR * sizeof(T);
    // stage: main box, then the two far-row boxes, each 128-byte aligned
    static constexpr unsigned FLO = (MAIN_BYTES + 127) / 128 * 128;
    static constexpr unsigned FHI = FLO + (XR_BYTES + 127) / 128 * 128;
    static constexpr unsigned STRIDE = (FHI + XR_BYTES + 127) / 128 * 128;
    static constexpr int S1_ROWS = TY + 2;  // sweep-1 rows y0 - 1 .. y0 + TY
    static constexpr unsigned S1_PLANE = (BXW * S1_ROWS * sizeof(T) + 127) / 128 * 128;
    static constexpr size_t SMEM = (size_t)STAGES * STRIDE + 3 * (size_t)S1_PLANE + 2 * STAGES * sizeof(uint64_t);
    static constexpr int THREADS = 32 * (CW + 1);
};

// Source plane of sweep-1 window p (the image planes map to their sources).
__device__ __forceinline__ int tma2_src(int p, int nz) { return p == 0 ? nz - 2 : (p == nz - 1 ? 1 : p); }

// Named barrier of the consumer warps (warps 0 .. CW - 1).
template <int CW>
__device__ __forceinline__ void consumers_sync() {
    asm volatile("bar.sync 1, %0;" ::"r"(32 * CW) : "memory");
}

template <typename T, int CW, int RPW, int STAGES, bool PY>
__global__ void __launch_bounds__(32 * (CW + 1))
    j3d_tma2_kernel(const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
                    const __grid_constant__ CUtensorMap tx0, const __grid_constant__ CUtensorMap tx1,
                    T *g0, T *g1, int nx, int ny, int nz, int npairs, int zchunk, BarrierState *bar) {
    using G = Tma2Geom<T, CW, RPW, STAGES>;
    using V = typename Vec16<T>::type;
    constexpr int VN = G::VN, TX = G::TX, BXW = G::BXW, TY = G::TY;
    extern __shared__ __align__(128) unsigned char tsm[];
    T *s1 = reinterpret_cast<T *>(tsm + STAGES * G::STRIDE);  // [3][S1_ROWS][BXW]
    constexpr int S1N = G::S1_PLANE / sizeof(T);
    uint64_t *full = reinterpret_cast<uint64_t *>(tsm + STAGES * G::STRIDE + 3 * G::S1_PLANE);
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
    volatile int *err = &s_err;

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

    for (int it = 0; it < npairs; ++it) {
        const CUtensorMap *tm = (it & 1) ? &tm1 : &tm0;
        const CUtensorMap *tx = (it & 1) ? &tx1 : &tx0;
        T *out = (it & 1) ? g0 : g1;
        if (warp == CW) {
            // ---------------------------------------------------- producer
            if (lane == 0) {
                fence_proxy_async_global();
                for (long long u = blockIdx.x; u < U && !*err; u += NB) {
                    const int ch = (int)(u / ntiles), tile = (int)(u - ch * ntiles);
                    const int x0 = (tile % ntx) * TX, y0 = 1 + (tile / ntx) * TY;
                    const int z0 = 1 + ch * zchunk, z1 = min(z0 + zchunk, nz - 1);
                    const bool need_lo = PY && y0 == 1, need_hi = PY && y0 + TY >= ny - 1;
                    const unsigned bytes = G::MAIN_BYTES + (need_lo ? G::XR_BYTES : 0u) + (need_hi ? G::XR_BYTES : 0u);
                    auto emit = [&](int plane) -> bool {
                        const int s = k % STAGES;
                        if (!mbar_wait_bounded(&empty[s], ((k / STAGES) & 1) ^ 1, budget)) {
                            if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = 3000000 + it;
                            *err = 1;
                            return false;
                        }
                        unsigned char *dst = tsm + s * G::STRIDE;
                        mbar_arrive_expect_tx(&full[s], bytes);
                        tma_load_3d(dst, tm, x0 - VN, y0 - 2, plane, &full[s]);
                        if (need_lo) tma_load_3d(dst + G::FLO, tx, x0 - VN, ny - 3, plane, &full[s]);
                        if (need_hi) tma_load_3d(dst + G::FHI, tx, x0 - VN, 0, plane, &full[s]);
                        ++k;
                        return true;
                    };
                    int qprev = -100;
                    for (int p = z0 - 1; p <= z1; ++p) {
                        const int q = tma2_src(p, nz);
                        bool ok = true;
                        if (q != qprev + 1) {
                            ok = emit(q - 1) && emit(q) && emit(q + 1);
                        } else {
                            ok = emit(q + 1);
                        }
                        if (!ok) break;
                        qprev = q;
                    }
                }
            }
            __syncwarp();
        } else {
            // ---------------------------------------------------- consumers
            for (long long u = blockIdx.x; u < U; u += NB) {
                const int ch = (int)(u / ntiles), tile = (int)(u - ch * ntiles);
                const int x0 = (tile % ntx) * TX, y0 = 1 + (tile / ntx) * TY;
                const int z0 = 1 + ch * zchunk, z1 = min(z0 + zchunk, nz - 1);
                int slo = 0, smid = 0, shi = 0, qprev = -100;
                for (int p = z0 - 1; p <= z1; ++p) {
                    const int q = tma2_src(p, nz);
                    const bool fresh = q != qprev + 1;
                    if (fresh) {
                        slo = k % STAGES;
                        smid = (k + 1) % STAGES;
                        shi = (k + 2) % STAGES;
                        for (int j = 0; j < 3; ++j, ++k)
                            if (!*err && !mbar_wait_bounded(&full[k % STAGES], (k / STAGES) & 1, budget))
                                *err = 1;
                    } else {
                        slo = smid;
                        smid = shi;
                        shi = k % STAGES;
                        if (!*err && !mbar_wait_bounded(&full[k % STAGES], (k / STAGES) & 1, budget)) *err = 1;
                        ++k;
                    }
                    qprev = q;
                    // ---- sweep 1 of window p (source plane q) into ring slot p % 3:
                    // rows y0 - 1 .. y0 + TY, one row per warp at a time; the
                    // TX central columns as VN-vectors (lane: x0 + lane VN ..),
                    // the two edge columns x0 - 1, x0 + TX by lanes 0 and 1
                    {
                        const T *ib = reinterpret_cast<const T *>(tsm + slo * G::STRIDE);  // plane q - 1
                        const T *ic = reinterpret_cast<const T *>(tsm + smid * G::STRIDE);  // plane q
                        const T *ia = reinterpret_cast<const T *>(tsm + shi * G::STRIDE);  // plane q + 1
                        T *so = s1 + (p % 3) * S1N;
                        for (int r = warp; r < G::S1_ROWS; r += CW) {
                            const int y = y0 - 1 + r;
                            if (y > ny - 1) break;  // rows only grow
                            const bool fixed_row = !PY && (y == 0 || y == ny - 1);
                            // the source cell's row in the stage: main box row r + 1,
                            // or the middle far row (source row ny - 2 or 1)
                            int ro;
                            if (PY && y == 0) ro = (int)(G::FLO / sizeof(T)) + BXW;
                            else if (PY && y == ny - 1) ro = (int)(G::FHI / sizeof(T)) + BXW;
                            else ro = (r + 1) * BXW;
                            // central columns
                            {
                                const int col = VN + lane * VN;  // x = x0 + lane VN
                                const int xb = x0 + lane * VN;
                                T own[VN], nn[VN], ss[VN], tt[VN], bb[VN], res[VN];
                                {
                                    const V a0 = *reinterpret_cast<const V *>(ic + ro + col);
                                    const V a1 = *reinterpret_cast<const V *>(ic + ro + col + BXW);
                                    const V a2 = *reinterpret_cast<const V *>(ic + ro + col - BXW);
                                    const V a3 = *reinterpret_cast<const V *>(ia + ro + col);
                                    const V a4 = *reinterpret_cast<const V *>(ib + ro + col);
                                    memcpy(own, &a0, sizeof(a0));
                                    memcpy(nn, &a1, sizeof(a1));
                                    memcpy(ss, &a2, sizeof(a2));
                                    memcpy(tt, &a3, sizeof(a3));
                                    memcpy(bb, &a4, sizeof(a4));
                                }
                                const T wl = ic[ro + col - 1], er = ic[ro + col + VN];
#pragma unroll
                                for (int i = 0; i < VN; ++i) {
                                    const T e = (i == VN - 1) ? er : own[i + 1];
                                    const T w = (i == 0) ? wl : own[i - 1];
                                    T sum = tma_add(e, w);
                                    sum = tma_add(sum, nn[i]);
                                    sum = tma_add(sum, ss[i]);
                                    sum = tma_add(sum, tt[i]);
                                    sum = tma_add(sum, bb[i]);
                                    const int x = xb + i;
                                    // fixed cells keep their value (read at the
                                    // row itself, not at a far source row)
                                    res[i] = (fixed_row || x == 0 || x == nx - 1) ? ic[(r + 1) * BXW + col + i]
                                                                                  : tma_mul(c6, sum);
                                }
                                V v;
                                memcpy(&v, res, sizeof(v));
                                *reinterpret_cast<V *>(so + r * BXW + col) = v;
                            }
                            // edge columns
                            if (lane < 2) {
                                const int col = lane == 0 ? VN - 1 : VN + TX;
                                const int x = x0 - 1 + (lane == 0 ? 0 : TX + 1);
                                if (x >= 0 && x <= nx - 1) {
                                    T v;
                                    if (fixed_row || x == 0 || x == nx - 1) {
                                        v = ic[(r + 1) * BXW + col];
                                    } else {
                                        const T *cc = ic + ro + col;
                                        T sum = tma_add(cc[1], cc[-1]);
                                        sum = tma_add(sum, cc[BXW]);
                                        sum = tma_add(sum, cc[-BXW]);
                                        sum = tma_add(sum, ia[ro + col]);
                                        sum = tma_add(sum, ib[ro + col]);
                                        v = tma_mul(c6, sum);
                                    }
                                    so[r * BXW + col] = v;
                                }
                            }
                        }
                    }
                    fence_proxy_async_shared();  // reads of the stages before their refill
                    consumers_sync<CW>();
                    // stages no later window reads: all three before a fresh
                    // window (or after the last), else the oldest
                    {
                        const bool last = p == z1;
                        const bool next_fresh = !last && tma2_src(p + 1, nz) != q + 1;
                        if (lane == 0) {
                            mbar_arrive(&empty[slo]);
                            if (last || next_fresh) {
                                mbar_arrive(&empty[smid]);
                                mbar_arrive(&empty[shi]);
                            }
                        }
                    }
                    // ---- sweep 2 of plane z = p - 1 from ring slots z - 1, z, z + 1
                    const int z = p - 1;
                    if (z >= z0) {
                        const T *sb = s1 + ((z + 2) % 3) * S1N;  // z - 1
                        const T *sc = s1 + (z % 3) * S1N;
                        const T *sa = s1 + ((z + 1) % 3) * S1N;
                        const int xb = x0 + lane * VN;
                        const bool full_vec = xb >= 1 && xb + VN - 1 <= nx - 2;
                        const bool zspecial = (z == 1) || (z == nz - 2);
                        const size_t zoff = (size_t)z * P;
#pragma unroll
                        for (int j = 0; j < RPW; ++j) {
                            const int y = y0 + warp * RPW + j;
                            if (y > ny - 2) continue;
                            const int o = (warp * RPW + j + 1) * BXW + VN + lane * VN;
                            T own[VN], nn[VN], ss[VN], tt[VN], bb[VN];
                            {
                                const V a = *reinterpret_cast<const V *>(sc + o);
                                const V b = *reinterpret_cast<const V *>(sc + o + BXW);
                                const V c = *reinterpret_cast<const V *>(sc + o - BXW);
                                const V d = *reinterpret_cast<const V *>(sa + o);
                                const V e = *reinterpret_cast<const V *>(sb + o);
                                memcpy(own, &a, sizeof(a));
                                memcpy(nn, &b, sizeof(b));
                                memcpy(ss, &c, sizeof(c));
                                memcpy(tt, &d, sizeof(d));
                                memcpy(bb, &e, sizeof(e));
                            }
                            const T wl = sc[o - 1], er = sc[o + VN];
                            T res[VN];
#pragma unroll
                            for (int i = 0; i < VN; ++i) {
                                const T e = (i == VN - 1) ? er : own[i + 1];
                                const T w = (i == 0) ? wl : own[i - 1];
                                T s = tma_add(e, w);
                                s = tma_add(s, nn[i]);
                                s = tma_add(s, ss[i]);
                                s = tma_add(s, tt[i]);
                                s = tma_add(s, bb[i]);
                                res[i] = tma_mul(c6, s);
                            }
                            const size_t idx = zoff + (size_t)y * nx + xb;
                            V v;
                            memcpy(&v, res, sizeof(v));
                            if (full_vec) {
                                __stcs(reinterpret_cast<V *>(out + idx), v);
                            } else {
#pragma unroll
                                for (int i = 0; i < VN; ++i)
                                    if (xb + i >= 1 && xb + i <= nx - 2) __stcs(out + idx + i, res[i]);
                            }
                            const bool yspecial = PY && (y == 1 || y == ny - 2);
                            if (zspecial || yspecial) {
                                // periodic images of this value, as j3d_tma_kernel writes them
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
                    }
                    consumers_sync<CW>();  // ring slot (p + 1) % 3 is free again
                }
            }
        }
        if (it + 1 < npairs) {
            if (!grid_barrier(bar, gridDim.x, it)) break;
        }
    }
    // On an error exit, let the loads this block issued land before its
    // shared memory is released (bounded).
    if (warp == CW && lane == 0 && *err) {
        const unsigned lo = k > (unsigned)STAGES ? k - STAGES : 0u;
        for (unsigned j = lo; j < k; ++j) mbar_wait_bounded(&full[j % STAGES], (j / STAGES) & 1, budget);
    }
}

}  // namespace cfm
