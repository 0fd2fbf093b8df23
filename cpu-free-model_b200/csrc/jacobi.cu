// Jacobi 2d5p / 3d7p sweeps on one GPU: kernels and the cfm_jacobi handle.
//
// Arithmetic (bit-exact with the reference's single-GPU run):
//   2D  a' = 0.25 * (((a[x+1] + a[x-1]) + a[y+1]) + a[y-1])
//        Stencil/jacobi2D/src/common.cu:28-42
//   3D  a' = (T(1)/T(6)) * (((((a[x+1] + a[x-1]) + a[y+1]) + a[y-1]) + a[z+1]) + a[z-1])
//        Stencil/jacobi3D/src/common.cu:31-57
// Halo semantics: after every sweep the reference copies row ny-2 -> row 0 and
// row 1 -> row ny-1 (planes in 3D), full width (Stencil/jacobi2D/src/common.cu:
// 234-242, Stencil/jacobi3D/src/common.cu:198-207).  The kernels here write
// each periodic image together with the interior value it copies (as
// jacobi_kernel_single_gpu_persistent does, Stencil/jacobi3D/src/common.cu:82-88),
// and the few cells no sweep reads or writes (the box edges of the halo
// rows/planes) are set to their images once before the first sweep
// (edge_preset_kernel), which gives the same grid after >= 1 sweeps.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cudaTypedefs.h>

#include "barrier.cuh"
#include "cfm_internal.h"
#include "j3d_tma.cuh"
#include "j3d_tma2.cuh"
#include "tma.cuh"

namespace cfm {

constexpr unsigned FULL = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T quarter(T s);
template <>
__device__ __forceinline__ double quarter<double>(double s) {
    return __dmul_rn(0.25, s);
}
template <>
__device__ __forceinline__ float quarter<float>(float s) {
    // The reference multiplies by the double literal 0.25 and stores a float;
    // scaling by a power of two is exact in double, so the single rounding to
    // float equals the correctly rounded float product.
    return __fmul_rn(0.25f, s);
}

template <typename T>
__device__ __forceinline__ T add_rn(T a, T b);
template <>
__device__ __forceinline__ double add_rn<double>(double a, double b) {
    return __dadd_rn(a, b);
}
template <>
__device__ __forceinline__ float add_rn<float>(float a, float b) {
    return __fadd_rn(a, b);
}
template <typename T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) {
    return __dmul_rn(a, b);
}
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) {
    return __fmul_rn(a, b);
}

// ------------------------------------------------------------------ 2D sweep
// One warp handles one 32-wide segment of one interior row; x neighbours come
// from warp shuffles, y neighbours from the (L1/L2-resident) rows above/below.
// Used for the persistent kernel (niter sweeps, barrier between) and, with
// niter = 1 and a plain launch, for the host-loop comparators.
template <typename T, bool IMAGES>
__global__ void __launch_bounds__(256) j2d_sweeps_kernel(T *g0, T *g1, int nx, int ny, int niter,
                                                         BarrierState *bar) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int ntx = (nx + 31) >> 5;
    const long long nseg = (long long)ntx * (ny - 2);
    T *in = g0, *out = g1;
    for (int it = 0; it < niter; ++it) {
        for (long long s = warp; s < nseg; s += nwarps) {
            const int y = 1 + (int)(s / ntx);
            const int x = (int)(s % ntx) * 32 + lane;
            const bool ld = x < nx;
            const size_t idx = (size_t)y * nx + x;
            T cur = ld ? in[idx] : T(0);
            T e = __shfl_down_sync(FULL, cur, 1);
            T w = __shfl_up_sync(FULL, cur, 1);
            if (lane == 31) e = (x + 1 < nx) ? in[idx + 1] : T(0);
            if (lane == 0) w = (x >= 1 && ld) ? in[idx - 1] : T(0);
            if (x >= 1 && x <= nx - 2) {
                const T n = in[idx + nx];
                const T so = in[idx - nx];
                const T v = quarter<T>(add_rn(add_rn(add_rn(e, w), n), so));
                out[idx] = v;
                if (IMAGES) {
                    if (y == 1) out[idx + (size_t)(ny - 2) * nx] = v;
                    if (y == ny - 2) out[idx - (size_t)(ny - 2) * nx] = v;
                }
            }
        }
        if (it + 1 < niter) {
            if (!grid_barrier(bar, gridDim.x, it)) return;
        }
        T *t = in;
        in = out;
        out = t;
    }
}

// 2D sweep with the mirror x boundary of the reference's PERKS comparator
// (jacobi_kernel_single_gpu_mirror, Stencil/jacobi2D/src/common.cu:44-66):
// every column of the interior rows is updated, the east and west neighbours
// clamped to the cell itself at x = nx-1 and x = 0, summed as
// 0.25 * (((N + S) + E) + W) with N the row below in memory (iy + 1).  One
// warp per 32-column segment as in j2d_sweeps_kernel; with IMAGES the
// periodic halo rows are written in-kernel (whole rows, corners included).
template <typename T, bool IMAGES>
__global__ void __launch_bounds__(256) j2d_mirror_kernel(T *g0, T *g1, int nx, int ny, int niter,
                                                         BarrierState *bar) {
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int ntx = (nx + 31) >> 5;
    const long long nseg = (long long)ntx * (ny - 2);
    T *in = g0, *out = g1;
    for (int it = 0; it < niter; ++it) {
        for (long long s = warp; s < nseg; s += nwarps) {
            const int y = 1 + (int)(s / ntx);
            const int x = (int)(s % ntx) * 32 + lane;
            const bool ld = x < nx;
            const size_t idx = (size_t)y * nx + x;
            const T cur = ld ? in[idx] : T(0);
            T e = __shfl_down_sync(FULL, cur, 1);
            T w = __shfl_up_sync(FULL, cur, 1);
            if (lane == 31 && x + 1 < nx) e = in[idx + 1];
            if (lane == 0 && x >= 1 && ld) w = in[idx - 1];
            if (x == nx - 1) e = cur;
            if (x == 0) w = cur;
            if (ld) {
                const T n = in[idx + nx];
                const T so = in[idx - nx];
                const T v = quarter<T>(add_rn(add_rn(add_rn(n, so), e), w));
                out[idx] = v;
                if (IMAGES) {
                    if (y == 1) out[idx + (size_t)(ny - 2) * nx] = v;
                    if (y == ny - 2) out[idx - (size_t)(ny - 2) * nx] = v;
                }
            }
        }
        if (it + 1 < niter) {
            if (!grid_barrier(bar, gridDim.x, it)) return;
        }
        T *t = in;
        in = out;
        out = t;
    }
}

// 2D sweep for rows whose byte length is a multiple of 16 (nx a multiple of
// V = 16 / sizeof(T)).  Work unit = (row chunk, column tile of 32 V columns),
// one warp per unit, units chunk-major and dealt to warps round-robin (the
// warps at work hold neighbouring tiles of one chunk, so the one-column x
// halo of a tile is an L1/L2 hit).  Each lane owns V consecutive columns
// (16-byte loads and stores) and marches down the chunk keeping a window of
// U + 2 rows in registers; U rows are loaded per step (4 in FP32, 2 in
// FP64), so each value is read from HBM once per sweep.  At most 64
// registers (four blocks per SM): with 91 the kernel ran at 452 GLUP/s FP32
// at 16384^2, with 64 at 689 (0.84 of the copy bandwidth).  x neighbours come from the lane's
// own vector, the neighbouring lanes (shuffles) or, at the warp's edges, one
// scalar load.  Boundary columns are stored unchanged.  The arithmetic per
// cell is the reference's: 0.25 * (((E + W) + N) + S).
template <typename T>
__device__ __forceinline__ void vload(const T *p, T (&v)[16 / sizeof(T)]) {
    const typename Vec16<T>::type q = *reinterpret_cast<const typename Vec16<T>::type *>(p);
    const T *e = reinterpret_cast<const T *>(&q);
#pragma unroll
    for (int j = 0; j < Vec16<T>::N; ++j) v[j] = e[j];
}
template <typename T>
__device__ __forceinline__ void vstore(T *p, const T (&v)[16 / sizeof(T)]) {
    typename Vec16<T>::type q;
    T *e = reinterpret_cast<T *>(&q);
#pragma unroll
    for (int j = 0; j < Vec16<T>::N; ++j) e[j] = v[j];
    *reinterpret_cast<typename Vec16<T>::type *>(p) = q;
}

template <typename T, bool IMAGES>
__global__ void __launch_bounds__(256, 4) j2d_march_kernel(T *g0, T *g1, int nx, int ny, int niter,
                                                           BarrierState *bar) {
    constexpr int V = Vec16<T>::N, W = 32 * V, U = sizeof(T) == 4 ? 4 : 2;
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const int ntx = (nx + W - 1) / W;
    // row chunk: about six units per warp, 8 to 256 rows, a multiple of the step
    const long long want = ((long long)(ny - 2) * ntx + 6 * nw - 1) / (6 * nw);
    const int rc = (int)((min(256LL, max(8LL, want)) + U - 1) / U * U);
    const int nrc = (ny - 2 + rc - 1) / rc;
    const long long nunits = (long long)ntx * nrc;
    T *in = g0, *out = g1;
    for (int it = 0; it < niter; ++it) {
        for (long long u = gw; u < nunits; u += nw) {
            const int tx = (int)(u % ntx), c = (int)(u / ntx);
            const int x0 = tx * W + lane * V;
            const bool on = x0 < nx;  // nx is a multiple of V: the whole vector is in the row
            const int yb = 1 + c * rc, ye = min(ny - 1, yb + rc);
            T win[U + 2][V];
            auto load_row = [&](int y, T (&v)[V]) {
                if (on) {
                    vload(in + (size_t)y * nx + x0, v);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j) v[j] = T(0);
                }
            };
            load_row(yb - 1, win[0]);
            load_row(yb, win[1]);
            for (int y = yb; y < ye; y += U) {
#pragma unroll
                for (int k = 0; k < U; ++k)
                    if (y + 1 + k <= ny - 1) load_row(y + 1 + k, win[k + 2]);
#pragma unroll
                for (int k = 0; k < U; ++k) {
                    const int r = y + k;
                    if (r >= ye) break;
                    const T(&cen)[V] = win[k + 1];
                    // x neighbours of the lane's first and last columns
                    T w0 = __shfl_up_sync(FULL, cen[V - 1], 1);
                    T eV = __shfl_down_sync(FULL, cen[0], 1);
                    const size_t row = (size_t)r * nx;
                    if (lane == 0 && on) w0 = x0 >= 1 ? in[row + x0 - 1] : T(0);
                    if (lane == 31 && on) eV = x0 + V < nx ? in[row + x0 + V] : T(0);
                    T o[V];
#pragma unroll
                    for (int j = 0; j < V; ++j) {
                        const int x = x0 + j;
                        const T e = j + 1 < V ? cen[j + 1] : eV;
                        const T w = j > 0 ? cen[j - 1] : w0;
                        const T nn = win[k + 2][j], so = win[k][j];
                        o[j] = (x >= 1 && x <= nx - 2) ? quarter<T>(add_rn(add_rn(add_rn(e, w), nn), so))
                                                       : cen[j];
                    }
                    if (on) {
                        vstore(out + row + x0, o);
                        if (IMAGES) {
                            if (r == 1) vstore(out + (size_t)(ny - 1) * nx + x0, o);
                            if (r == ny - 2) vstore(out + x0, o);
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    win[0][j] = win[U][j];
                    win[1][j] = win[U + 1][j];
                }
            }
        }
        if (it + 1 < niter) {
            if (!grid_barrier(bar, gridDim.x, it)) return;
        }
        T *t = in;
        in = out;
        out = t;
    }
}

// ------------------------------------------------------------------ 3D sweep
// Work unit = (z-chunk, tile) with the tile 32 (x, aligned at x = 0) by TY
// interior rows; units are ordered chunk-major and dealt to blocks round-robin
// (block b takes units b, b + G, b + 2G, ...), so at any moment the G blocks
// work on G consecutive units -- neighbouring tiles of the same z-chunk at the
// same plane -- and the tile-edge rows they share are L2 hits.  Inside a unit
// each thread marches along z keeping the z-1, z, z+1 values in registers:
// every interior value is read from HBM once per sweep.
constexpr int J3_ZSTEP = 2;  // z planes loaded ahead per step (2 measured best of 2, 4, 8)
template <typename T, int TY, bool PY, bool IMAGES>
__global__ void __launch_bounds__(32 * TY, 4) j3d_sweeps_kernel(T *g0, T *g1, int nx, int ny, int nz,
                                                                int niter, int zchunk,
                                                                BarrierState *bar) {
    constexpr int K = J3_ZSTEP;  // planes loaded ahead per step
    const int lane = threadIdx.x;
    const int wy = threadIdx.y;
    const int ntx = (nx + 31) >> 5;
    const int nty = (ny - 2 + TY - 1) / TY;
    const long long ntiles = (long long)ntx * nty;
    const int nzi = nz - 2;
    const int nch = (nzi + zchunk - 1) / zchunk;
    const long long U = ntiles * nch;
    const size_t P = (size_t)nx * ny;
    const T c6 = T(1) / T(6);
    const size_t zimg = (size_t)(nz - 2) * P;
    const size_t yimg = (size_t)(ny - 2) * nx;
    T *in = g0, *out = g1;
    for (int it = 0; it < niter; ++it) {
        // the two grids of a sweep never alias: loads may pass stores
        const T *__restrict__ src = in;
        T *__restrict__ dst = out;
        for (long long u = blockIdx.x; u < U; u += gridDim.x) {
            const int ch = (int)(u / ntiles);
            const int tile = (int)(u - (long long)ch * ntiles);
            const int x = (tile % ntx) * 32 + lane;
            const int y = 1 + (tile / ntx) * TY + wy;
            const int z0 = 1 + ch * zchunk;
            const int z1 = min(z0 + zchunk, nz - 1);
            const bool ld = (y <= ny - 2) && (x < nx);
            const bool comp = ld && x >= 1 && x <= nx - 2;
            size_t idx = ((size_t)z0 * ny + (ld ? y : 1)) * nx + (ld ? x : 0);
            T win[K + 2];  // planes z-1 .. z+K at this (x, y)
            win[0] = ld ? src[idx - P] : T(0);
            win[1] = ld ? src[idx] : T(0);
            for (int z = z0; z < z1; z += K, idx += K * P) {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    win[k + 2] = (ld && z + 1 + k <= z1) ? src[idx + (size_t)(k + 1) * P] : T(0);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const int zz = z + k;
                    if (zz >= z1) break;
                    const size_t i = idx + (size_t)k * P;
                    const T cur = win[k + 1];
                    T e = __shfl_down_sync(FULL, cur, 1);
                    T w = __shfl_up_sync(FULL, cur, 1);
                    if (lane == 31) e = (ld && x + 1 < nx) ? src[i + 1] : T(0);
                    if (lane == 0) w = (ld && x >= 1) ? src[i - 1] : T(0);
                    if (comp) {
                        const T n = src[i + nx];
                        const T so = src[i - nx];
                        T sum = add_rn(add_rn(add_rn(add_rn(add_rn(e, w), n), so), win[k + 2]), win[k]);
                        const T v = mul_rn(c6, sum);
                        dst[i] = v;
                        if (IMAGES) {
                            const bool zlo = (zz == 1), zhi = (zz == nz - 2);
                            if (zlo) dst[i + zimg] = v;
                            if (zhi) dst[i - zimg] = v;
                            if (PY) {
                                if (y == 1) {
                                    dst[i + yimg] = v;
                                    if (zlo) dst[i + yimg + zimg] = v;
                                    if (zhi) dst[i + yimg - zimg] = v;
                                }
                                if (y == ny - 2) {
                                    dst[i - yimg] = v;
                                    if (zlo) dst[i - yimg + zimg] = v;
                                    if (zhi) dst[i - yimg - zimg] = v;
                                }
                            }
                        }
                    }
                }
                win[0] = win[K];
                win[1] = win[K + 1];
            }
        }
        if (it + 1 < niter) {
            if (!grid_barrier(bar, gridDim.x, it)) return;
        }
        T *t = in;
        in = out;
        out = t;
    }
}

// ---------------------------------------------------------- 2D resident sweep
// PERKS-style temporal residency (the design of Stencil/jacobi2D/PERKS/
// jacobi-general-kernel.cuh:22-505, re-derived): block b owns the interior
// rows [r0, r1) and keeps them, plus one halo row above and below, in shared
// memory for all sweeps (two copies, ping-pong).  Per sweep the only global
// traffic is the block's first and last new rows, published to a
// double-buffered exchange area, and its two halo rows read back from the
// ring neighbours (b-1, b+1 mod B; the ring closes through the periodic rows,
// so block 0's upper halo is the last block's last row).  Synchronisation is
// point-to-point: a per-block sweep counter, bounded waits on the two
// neighbours only, no grid-wide barrier.
__device__ __forceinline__ void st_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T, bool MIRROR>
__global__ void __launch_bounds__(1024, 1)
    j2d_resident_kernel(const T *in, T *final_out, int nx, int ny, int niter, T *xbuf,
                        unsigned int *flags, BarrierState *bar) {
    extern __shared__ __align__(16) unsigned char j2d_smem[];
    const int B = gridDim.x, b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const int nrows = ny - 2;
    const int r0 = 1 + (int)((long long)b * nrows / B);
    const int r1 = 1 + (int)((long long)(b + 1) * nrows / B);
    const int h = r1 - r0;
    const int up_blk = (b + B - 1) % B, dn_blk = (b + 1) % B;
    const size_t band = (size_t)(h + 2) * nx;
    T *cur = reinterpret_cast<T *>(j2d_smem);
    T *nxt = cur + band;
    for (size_t i = tid; i < band; i += nth) {
        const T v = in[(size_t)(r0 - 1) * nx + i];
        cur[i] = v;
        nxt[i] = v;
    }
    __syncthreads();
    __shared__ int s_ok;
    // updated columns: 1 .. nx-2, or with the mirror boundary 0 .. nx-1
    const int x0 = MIRROR ? 0 : 1;
    const int inner = MIRROR ? nx : nx - 2;
    // rows [ra, rb) of the band as a flat run of cells, row r / column x of
    // the first cell of each thread stepped without a division per cell
    const int dr = nth / inner, dx = nth % inner;
    auto sweep_rows = [&](int ra, int rb, T *pub) {
        int r = ra + tid / inner, x = x0 + tid % inner;
        for (; r < rb; r += dr, x += dx) {
            if (x >= x0 + inner) {
                x -= inner;
                ++r;
                if (r >= rb) break;
            }
            const T *c = cur + (size_t)r * nx + x;
            T v;
            if (MIRROR)  // Stencil/jacobi2D/src/common.cu:57-63
                v = quarter<T>(add_rn(add_rn(add_rn(c[nx], c[-nx]), c[x < nx - 1 ? 1 : 0]),
                                      c[x > 0 ? -1 : 0]));
            else
                v = quarter<T>(add_rn(add_rn(add_rn(c[1], c[-1]), c[nx]), c[-nx]));
            nxt[(size_t)r * nx + x] = v;
            if (pub) {  // the rows the neighbours read: first to slot 0, last to slot 1
                if (r == 1) __stcg(pub + x, v);
                if (r == h) __stcg(pub + nx + x, v);
            }
        }
    };
    for (int t = 0; t < niter; ++t) {
        T *xb = xbuf + ((size_t)(t & 1) * B + b) * 2 * nx;
        // 1. the first and last rows, published as they are computed (a
        //    one-row band publishes its row in both slots)
        sweep_rows(1, 2, xb);
        if (h > 1) sweep_rows(h, h + 1, xb);
        // the slot columns 0 and nx-1 carry the band's boundary cells
        if (!MIRROR && tid == 0) {  // (mirror: sweep_rows published them)
            __stcg(xb, nxt[nx]);
            __stcg(xb + nx - 1, nxt[2 * (size_t)nx - 1]);
            __stcg(xb + nx, nxt[(size_t)h * nx]);
            __stcg(xb + 2 * nx - 1, nxt[(size_t)(h + 1) * nx - 1]);
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release_u32(flags + b, (unsigned)(t + 1));
        }
        // 2. the inner rows while the neighbours' counters move
        if (h > 2) sweep_rows(2, h, nullptr);
        // 3. wait for the two ring neighbours' rows of this sweep
        if (tid == 0) {
            int ok = 1;
            const unsigned long long t0 = global_ns();
            const unsigned long long budget = bar->timeout_ns;
            while (ld_acquire_u32(flags + up_blk) < (unsigned)(t + 1) ||
                   ld_acquire_u32(flags + dn_blk) < (unsigned)(t + 1)) {
                if (ld_relaxed_i32(&bar->error)) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > budget) {
                    if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = t;
                    ok = 0;
                    break;
                }
            }
            __threadfence();
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return;
        const T *up = xbuf + ((size_t)(t & 1) * B + up_blk) * 2 * nx + nx;  // last row above
        const T *dn = xbuf + ((size_t)(t & 1) * B + dn_blk) * 2 * nx;       // first row below
        for (int x = tid; x < nx; x += nth) {
            nxt[x] = __ldcg(up + x);
            nxt[(size_t)(h + 1) * nx + x] = __ldcg(dn + x);
        }
        __syncthreads();
        T *tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    // write the band back; the owners of rows 1 and ny-2 also write their
    // periodic images (full rows, so the corner cells become images too)
    for (size_t i = tid; i < (size_t)h * nx; i += nth) final_out[(size_t)r0 * nx + i] = cur[nx + i];
    if (r0 == 1)
        for (int x = tid; x < nx; x += nth) final_out[(size_t)(ny - 1) * nx + x] = cur[nx + x];
    if (r1 == ny - 1)
        for (int x = tid; x < nx; x += nth) final_out[x] = cur[(size_t)h * nx + x];
}

// The resident kernel with two sweeps per exchange (halo two rows deep): the
// band lives in shared memory with two halo rows on each side (h + 4 rows,
// twice).  The first sweep runs alone (the initial halo rows need not be
// periodic images yet) and ends with an exchange of the block's first two
// and last two rows; from then on each period is sweep A over rows r0 - 1 ..
// r1 (the extra row on each side computed from the deeper halo, with the
// same inputs and arithmetic as the neighbour that owns it, so the same
// bits) and sweep B over the block's own rows r0 .. r1 - 1, then one
// exchange; an odd last sweep runs alone.  Half the neighbour handshakes of
// j2d_resident_kernel for 2 / h more computed rows.  Needs h >= 2.
template <typename T, bool MIRROR>
__global__ void __launch_bounds__(1024, 1)
    j2d_resident2_kernel(const T *in, T *final_out, int nx, int ny, int niter, T *xbuf,
                         unsigned int *flags, BarrierState *bar) {
    extern __shared__ __align__(16) unsigned char j2d_smem[];
    const int B = gridDim.x, b = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
    const int nrows = ny - 2;
    const int r0 = 1 + (int)((long long)b * nrows / B);
    const int r1 = 1 + (int)((long long)(b + 1) * nrows / B);
    const int h = r1 - r0;  // >= 2
    const int up_blk = (b + B - 1) % B, dn_blk = (b + 1) % B;
    // local row l of the band is global row r0 - 2 + l; own rows are 2 .. h + 1
    const size_t band = (size_t)(h + 4) * nx;
    T *cur = reinterpret_cast<T *>(j2d_smem);
    T *nxt = cur + band;
    // initial rows r0 - 1 .. r1 (local 1 .. h + 2) in both copies
    for (size_t i = tid; i < (size_t)(h + 2) * nx; i += nth) {
        const T v = in[(size_t)(r0 - 1) * nx + i];
        cur[nx + i] = v;
        nxt[nx + i] = v;
    }
    __syncthreads();
    __shared__ int s_ok;
    const int x0 = MIRROR ? 0 : 1;
    const int inner = MIRROR ? nx : nx - 2;
    const int dr = nth / inner, dx = nth % inner;
    // rows [ra, rb) (local) of dst from src
    auto sweep_rows = [&](const T *src, T *dst, int ra, int rb) {
        if (ra >= rb) return;
        int r = ra + tid / inner, x = x0 + tid % inner;
        for (; r < rb; r += dr, x += dx) {
            if (x >= x0 + inner) {
                x -= inner;
                ++r;
                if (r >= rb) break;
            }
            const T *c = src + (size_t)r * nx + x;
            T v;
            if (MIRROR)
                v = quarter<T>(add_rn(add_rn(add_rn(c[nx], c[-nx]), c[x < nx - 1 ? 1 : 0]),
                                      c[x > 0 ? -1 : 0]));
            else
                v = quarter<T>(add_rn(add_rn(add_rn(c[1], c[-1]), c[nx]), c[-nx]));
            dst[(size_t)r * nx + x] = v;
        }
    };
    // The block's own rows of one sweep src -> dst: first its two edge rows
    // at each end, published (full rows) to exchange slot `e`; then, when
    // `publish`, the block's counter; then the inner rows; then, when
    // `publish`, the neighbours' rows into dst's halo rows.  Returns false
    // when a wait ran out.
    auto own_sweep = [&](const T *src, T *dst, unsigned e, bool publish) -> bool {
        const int ea = min(4, h + 2), eb = max(ea, h);
        sweep_rows(src, dst, 2, ea);
        sweep_rows(src, dst, eb, h + 2);
        if (!publish) {
            sweep_rows(src, dst, ea, eb);
            return true;
        }
        __syncthreads();
        T *xb = xbuf + ((size_t)(e & 1) * B + b) * 4 * nx;  // first two, last two rows
        for (int i = tid; i < 2 * nx; i += nth) {
            __stcg(xb + i, dst[2 * (size_t)nx + i]);
            __stcg(xb + 2 * nx + i, dst[(size_t)h * nx + i]);
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release_u32(flags + b, e);
        }
        sweep_rows(src, dst, ea, eb);
        if (tid == 0) {
            int ok = 1;
            const unsigned long long t0 = global_ns();
            const unsigned long long budget = bar->timeout_ns;
            while (ld_acquire_u32(flags + up_blk) < e || ld_acquire_u32(flags + dn_blk) < e) {
                if (ld_relaxed_i32(&bar->error)) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > budget) {
                    if (atomicCAS(&bar->error, 0, 1) == 0) bar->where = (int)e;
                    ok = 0;
                    break;
                }
            }
            __threadfence();
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return false;
        const T *up = xbuf + ((size_t)(e & 1) * B + up_blk) * 4 * nx + 2 * nx;  // its last two rows
        const T *dn = xbuf + ((size_t)(e & 1) * B + dn_blk) * 4 * nx;           // its first two rows
        for (int i = tid; i < 2 * nx; i += nth) {
            dst[i] = __ldcg(up + i);
            dst[(size_t)(h + 2) * nx + i] = __ldcg(dn + i);
        }
        __syncthreads();
        return true;
    };
    int t = 0;
    unsigned e = 0;  // exchanges so far
    if (niter > 0) {  // the first sweep alone, from the initial halo rows
        if (!own_sweep(cur, nxt, ++e, niter > 1)) return;
        T *tmp = cur;
        cur = nxt;
        nxt = tmp;
        t = 1;
    }
    while (t < niter) {
        if (niter - t >= 2) {
            sweep_rows(cur, nxt, 1, h + 3);  // sweep A: own rows and one more each side
            __syncthreads();
            if (!own_sweep(nxt, cur, ++e, t + 2 < niter)) return;  // sweep B, back into cur
            t += 2;
        } else {
            if (!own_sweep(cur, nxt, ++e, false)) return;
            __syncthreads();
            T *tmp = cur;
            cur = nxt;
            nxt = tmp;
            t += 1;
        }
    }
    __syncthreads();
    // write the band back; the owners of rows 1 and ny-2 also write their
    // periodic images (full rows)
    for (size_t i = tid; i < (size_t)h * nx; i += nth) final_out[(size_t)r0 * nx + i] = cur[2 * nx + i];
    if (r0 == 1)
        for (int x = tid; x < nx; x += nth) final_out[(size_t)(ny - 1) * nx + x] = cur[2 * nx + x];
    if (r1 == ny - 1)
        for (int x = tid; x < nx; x += nth) final_out[x] = cur[(size_t)(h + 1) * nx + x];
}

// Cells on the edges of the box (two or more coordinates on the boundary) are
// neither read nor written by a sweep.  The reference's full-row/plane halo
// copies leave each such cell equal to its periodic image after the first
// sweep; set that once in both buffers.  Images always have their periodic
// coordinates moved inside, so no cell read here is written here.
template <typename T>
__global__ void edge_preset_kernel(const T *cur, T *b0, T *b1, int dims, int nx, int ny, int nz,
                                   int py) {
    const long long n_edge = 4LL * nx + 4LL * ny + (dims == 3 ? 4LL * nz : 0);
    const int zmax = dims == 3 ? nz : 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_edge;
         i += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        long long k = i;
        if (k < 4LL * nx) {  // edges running along x
            const int c = (int)(k / nx);
            x = (int)(k % nx);
            y = (c & 1) ? ny - 1 : 0;
            z = (c & 2) ? zmax - 1 : 0;
        } else if ((k -= 4LL * nx) < 4LL * ny) {  // edges along y
            const int c = (int)(k / ny);
            y = (int)(k % ny);
            x = (c & 1) ? nx - 1 : 0;
            z = (c & 2) ? zmax - 1 : 0;
        } else {  // edges along z (3D only)
            k -= 4LL * ny;
            const int c = (int)(k / nz);
            z = (int)(k % nz);
            x = (c & 1) ? nx - 1 : 0;
            y = (c & 2) ? ny - 1 : 0;
        }
        const int onb = (x == 0 || x == nx - 1) + (y == 0 || y == ny - 1) +
                        (dims == 3 && (z == 0 || z == nz - 1));
        if (onb < 2) continue;
        int iy = y, iz = z;
        if (dims == 2 || py) iy = (y == 0) ? ny - 2 : (y == ny - 1 ? 1 : y);
        if (dims == 3) iz = (z == 0) ? nz - 2 : (z == nz - 1 ? 1 : z);
        if (iy == y && iz == z) continue;
        const size_t dst = ((size_t)z * ny + y) * nx + x;
        const size_t src = ((size_t)iz * ny + iy) * nx + x;
        const T v = cur[src];
        b0[dst] = v;
        b1[dst] = v;
    }
}

// Device-side initial state (same values as cfm_jacobi_problem_host):
// sy/sz hold the host-computed sin(2 pi i/(n-1)) factors.
template <typename T>
__global__ void load_problem_kernel(T *a, int dims, int nx, int ny, int nz, int problem,
                                    const double *sy, const double *sz) {
    const size_t N = (size_t)nx * ny * (dims == 3 ? nz : 1);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const size_t r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        T v = T(0);
        if (dims == 2) {
            if (x == 0 || x == nx - 1) v = (T)sy[y];
        } else if (problem == CFM_PROBLEM_REF) {
            if (x == 0) v = (T)((T)z - (T)y) - (T)(nx - 1);
        } else {
            if (x == 0 || x == nx - 1) v = (T)(sy[y] * sz[z]);
        }
        a[i] = v;
    }
}

}  // namespace cfm

using namespace cfm;

namespace cfm {
// One configuration of the 3D TMA pipeline: tensor maps over both grids
// (main boxes and, for two sweeps per pass, the 3-row far-row boxes), the
// kernel and its launch shape.
struct TmaConfig {
    bool ok = false;
    CUtensorMap map[2], xmap[2];
    const void *fn = nullptr;
    int var = 0, sweeps = 1, blocks = 0, zchunk = 0, threads = 0;
    long long units = 0;
    size_t smem = 0;
};
}  // namespace cfm

struct cfm_jacobi {
    cfm_jacobi_params p;
    size_t elems = 0, esize = 0;
    void *buf[2] = {nullptr, nullptr};
    int cur = 0;
    BarrierState *bar = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int blocks = 0, threads = 0, zchunk = 0;
    int num_sms = 0;
    // 2D resident kernel: exchange rows, per-block sweep counters, shape
    void *xbuf = nullptr;
    unsigned int *flags = nullptr;
    int res_blocks = 0;
    size_t res_smem = 0;
    bool res_two = false;  // two sweeps per exchange (j2d_resident2_kernel)
    bool resident = false;
    // 3D TMA pipeline: the chosen shape, and (for a two-sweep shape) the
    // one-sweep shape that does the last sweep of an odd count
    bool tma = false;
    cfm::TmaConfig tc, tail;
    size_t smem_optin = 0;
    // 2D: the mirror x boundary of the reference's PERKS comparator
    bool mirror = false;
    // 3D TMA pipeline: sweeps ordered by unit neighbourhoods (true) or a
    // grid barrier per sweep (the default: measured 3% faster at 512^3, the
    // lockstep keeps the halo rows that neighbouring tiles share in L2); the
    // per-unit counters and their capacity
    bool dataflow = false;
    unsigned int *udone = nullptr;
    long long udone_cap = 0;
};

namespace {

// Units are dealt round-robin to G blocks, so a sweep takes ceil(U / G)
// rounds, each as long as one unit: zc planes plus the two planes every unit
// reloads at its start.  Pick the z-chunk that minimises rounds * (zc + 2)
// (ties: the longer chunk).  Returns the chunk and lowers *blocks when there
// are fewer units than blocks.
long long units_of(long long ntiles, int nzi, int zc) { return ntiles * ((nzi + zc - 1) / zc); }

int pick_zchunk(long long ntiles, int nzi, int *blocks) {
    int best = std::min(8, nzi);
    double best_cost = 1e300;
    const int cand[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256};
    for (int zc0 : cand) {
        const int zc = std::min(zc0, nzi);
        const long long U = units_of(ntiles, nzi, zc);
        const long long G = std::min<long long>(*blocks, U);
        const double cost = (double)((U + G - 1) / G) * (zc + 2) * ((double)*blocks / G);
        if (cost <= best_cost) {
            best_cost = cost;
            best = zc;
        }
    }
    const long long U = units_of(ntiles, nzi, best);
    if (U < *blocks) *blocks = (int)std::max(1LL, U);
    return best;
}

constexpr int J3_TY = 8;

// Shapes of the TMA pipeline compiled into the library: consumer warps, rows
// per consumer warp, ring stages.  Entry 0 is the default; the autotuner
// (cfm_jacobi_autotune) times them all; the environment variable
// CFM_J3D_TMA_VARIANT (an index into this table) overrides the choice.
struct TmaVariant {
    int cw, rpw, stages;
    int sweeps;            // sweeps per pass over the grid (2: j3d_tma2_kernel)
    const void *fn[2][2];  // [precision][periodic_y]
    size_t smem[2];        // [precision]
    int tx[2];             // [precision]
};

template <int CW, int RPW, int S>
TmaVariant make_tma_variant() {
    TmaVariant v{CW, RPW, S, 1, {}, {}, {}};
    v.fn[CFM_FP64][0] = (const void *)j3d_tma_kernel<double, CW, RPW, S, false>;
    v.fn[CFM_FP64][1] = (const void *)j3d_tma_kernel<double, CW, RPW, S, true>;
    v.fn[CFM_FP32][0] = (const void *)j3d_tma_kernel<float, CW, RPW, S, false>;
    v.fn[CFM_FP32][1] = (const void *)j3d_tma_kernel<float, CW, RPW, S, true>;
    v.smem[CFM_FP64] = TmaGeom<double, CW, RPW, S>::SMEM;
    v.smem[CFM_FP32] = TmaGeom<float, CW, RPW, S>::SMEM;
    v.tx[CFM_FP64] = TmaGeom<double, CW, RPW, S>::TX;
    v.tx[CFM_FP32] = TmaGeom<float, CW, RPW, S>::TX;
    return v;
}

template <int CW, int RPW, int S>
TmaVariant make_tma2_variant() {
    TmaVariant v{CW, RPW, S, 2, {}, {}, {}};
    v.fn[CFM_FP64][0] = (const void *)j3d_tma2_kernel<double, CW, RPW, S, false>;
    v.fn[CFM_FP64][1] = (const void *)j3d_tma2_kernel<double, CW, RPW, S, true>;
    v.fn[CFM_FP32][0] = (const void *)j3d_tma2_kernel<float, CW, RPW, S, false>;
    v.fn[CFM_FP32][1] = (const void *)j3d_tma2_kernel<float, CW, RPW, S, true>;
    v.smem[CFM_FP64] = Tma2Geom<double, CW, RPW, S>::SMEM;
    v.smem[CFM_FP32] = Tma2Geom<float, CW, RPW, S>::SMEM;
    v.tx[CFM_FP64] = Tma2Geom<double, CW, RPW, S>::TX;
    v.tx[CFM_FP32] = Tma2Geom<float, CW, RPW, S>::TX;
    return v;
}

// Variants 0-11 take one sweep per pass, 12-15 two (temporal blocking).
const TmaVariant *tma_variants(int *count) {
    static const TmaVariant v[] = {
        make_tma_variant<8, 2, 6>(), make_tma_variant<4, 2, 8>(),  make_tma_variant<4, 4, 6>(),
        make_tma_variant<8, 1, 8>(), make_tma_variant<4, 2, 12>(), make_tma_variant<2, 4, 8>(),
        make_tma_variant<8, 4, 4>(), make_tma_variant<16, 2, 4>(),  make_tma_variant<16, 2, 6>(),
        make_tma_variant<16, 2, 8>(), make_tma_variant<8, 4, 8>(),  make_tma_variant<16, 4, 4>(),
        make_tma2_variant<16, 2, 4>(), make_tma2_variant<16, 2, 6>(), make_tma2_variant<8, 4, 5>(),
        make_tma2_variant<8, 2, 4>(),
    };
    *count = (int)(sizeof(v) / sizeof(v[0]));
    return v;
}

const TmaVariant &tma_variant(int i) {
    int n = 0;
    const TmaVariant *v = tma_variants(&n);
    return v[(i >= 0 && i < n) ? i : 0];
}


// Tensor maps over both grids: dims (nx, ny, nz), box (TX + 2 VN, TY + 2, 1)
// for one sweep per pass, (TX + 2 VN, TY + 4, 1) plus the 3-row far-row box
// for two; zero fill outside.  Needs the row pitch nx * esize to be a
// multiple of 16.  Leaves c->ok false when the pipeline does not apply.
int build_tma(cfm_jacobi *h, int var, int zchunk, TmaConfig *c) {
    const cfm_jacobi_params &p = h->p;
    c->ok = false;
    if (p.dims != 3 || ((size_t)p.nx * h->esize) % 16 != 0) return CFM_OK;
    auto enc = tensor_map_encoder();
    if (!enc) return CFM_OK;
    const TmaVariant &V = tma_variant(var);
    const int ty = V.cw * V.rpw, tx = V.tx[p.precision];
    const int vn = (int)(16 / h->esize);
    const cuuint64_t dims[3] = {(cuuint64_t)p.nx, (cuuint64_t)p.ny, (cuuint64_t)p.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)p.nx * h->esize, (cuuint64_t)p.nx * p.ny * h->esize};
    const cuuint32_t box[3] = {(cuuint32_t)(tx + 2 * vn), (cuuint32_t)(ty + (V.sweeps == 2 ? 4 : 2)), 1u};
    const cuuint32_t xbox[3] = {(cuuint32_t)(tx + 2 * vn), 3u, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt =
        p.precision == CFM_FP64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    for (int i = 0; i < 2; ++i) {
        CUresult r = enc(&c->map[i], dt, 3, h->buf[i], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r == CUDA_SUCCESS && V.sweeps == 2)
            r = enc(&c->xmap[i], dt, 3, h->buf[i], dims, strides, xbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return CFM_OK;  // stay on the register kernel
    }
    const void *fn = V.fn[p.precision][p.periodic_y ? 1 : 0];
    const size_t smem = V.smem[p.precision];
    if (smem > h->smem_optin) return CFM_OK;
    const int threads = 32 * (V.cw + 1);
    CFM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // all of the SM's shared memory for the ring (two rings per SM when they fit)
    CFM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    int per_sm = 0;
    CFM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    if (per_sm < 1) return CFM_OK;
    c->blocks = per_sm * h->num_sms;
    const long long ntiles = (long long)((p.nx + tx - 1) / tx) * ((p.ny - 2 + ty - 1) / ty);
    if (zchunk <= 0)
        if (const char *zc = std::getenv("CFM_J3D_ZCHUNK")) zchunk = std::atoi(zc);
    if (zchunk >= 1) {
        c->zchunk = std::min(zchunk, p.nz - 2);
        const long long U = units_of(ntiles, p.nz - 2, c->zchunk);
        if (U < c->blocks) c->blocks = (int)std::max(1LL, U);
    } else {
        c->zchunk = pick_zchunk(ntiles, p.nz - 2, &c->blocks);
    }
    // one completion counter per unit for the neighbourhood-ordered sweeps
    const long long U = units_of(ntiles, p.nz - 2, c->zchunk);
    if (V.sweeps == 1 && U > h->udone_cap) {
        unsigned int *q = nullptr;
        CFM_CUDA_TRY(cudaMalloc(&q, sizeof(unsigned int) * U));
        if (h->udone) {
            cudaStreamSynchronize(h->stream);
            cudaFree(h->udone);
        }
        h->udone = q;
        h->udone_cap = U;
    }
    c->units = U;
    c->var = var;
    c->sweeps = V.sweeps;
    c->threads = threads;
    c->fn = fn;
    c->smem = smem;
    c->ok = true;
    return CFM_OK;
}

int default_tma_variant();

// The pipeline shape `var` (and, for two sweeps per pass, the default
// one-sweep shape for the last sweep of an odd count).
int setup_tma(cfm_jacobi *h, int var, int zchunk = 0) {
    h->tma = false;
    int st = build_tma(h, var, zchunk, &h->tc);
    if (st || !h->tc.ok) return st;
    if (h->tc.sweeps == 2) {
        int dv = default_tma_variant();
        if (tma_variant(dv).sweeps != 1) dv = 0;
        if ((st = build_tma(h, dv, 0, &h->tail))) return st;
        if (!h->tail.ok) return CFM_OK;
    }
    h->tma = true;
    return CFM_OK;
}

int default_tma_variant() {
    int n = 0;
    tma_variants(&n);
    if (const char *e = std::getenv("CFM_J3D_TMA_VARIANT")) {
        const int v = std::atoi(e);
        if (v >= 0 && v < n) return v;
    }
    return 0;
}

int check_params(const cfm_jacobi_params *p) {
    CFM_ARG_CHECK(p, "params is null");
    CFM_ARG_CHECK(p->dims == 2 || p->dims == 3, "dims must be 2 or 3");
    CFM_ARG_CHECK(p->nx >= 3 && p->ny >= 3, "nx, ny must be >= 3");
    CFM_ARG_CHECK(p->dims == 2 || p->nz >= 3, "nz must be >= 3");
    CFM_ARG_CHECK(p->precision == CFM_FP64 || p->precision == CFM_FP32, "precision");
    CFM_ARG_CHECK(p->impl >= CFM_JACOBI_HOST_LOOP && p->impl <= CFM_JACOBI_RESIDENT, "impl");
    const double cells = (double)p->nx * p->ny * (p->dims == 3 ? p->nz : 1);
    CFM_ARG_CHECK(cells < 9.0e18, "grid too large");
    CFM_ARG_CHECK((double)p->nx * p->ny < 2.0e9, "plane too large");
    return CFM_OK;
}

size_t grid_elems(const cfm_jacobi_params *p) {
    return (size_t)p->nx * p->ny * (p->dims == 3 ? (size_t)p->nz : 1);
}

template <typename T>
const void *sweep_fn(const cfm_jacobi_params &p, bool images, bool mirror) {
    if (p.dims == 2 && mirror)
        return images ? (const void *)j2d_mirror_kernel<T, true>
                      : (const void *)j2d_mirror_kernel<T, false>;
    if (p.dims == 2 && p.nx % (16 / (int)sizeof(T)) == 0)
        return images ? (const void *)j2d_march_kernel<T, true>
                      : (const void *)j2d_march_kernel<T, false>;
    if (p.dims == 2)
        return images ? (const void *)j2d_sweeps_kernel<T, true>
                      : (const void *)j2d_sweeps_kernel<T, false>;
    if (p.periodic_y)
        return images ? (const void *)j3d_sweeps_kernel<T, J3_TY, true, true>
                      : (const void *)j3d_sweeps_kernel<T, J3_TY, true, false>;
    return images ? (const void *)j3d_sweeps_kernel<T, J3_TY, false, true>
                  : (const void *)j3d_sweeps_kernel<T, J3_TY, false, false>;
}

const void *sweep_fn_any(const cfm_jacobi_params &p, bool images, bool mirror) {
    return p.precision == CFM_FP64 ? sweep_fn<double>(p, images, mirror)
                                   : sweep_fn<float>(p, images, mirror);
}

const void *resident_fn(const cfm_jacobi_params &p, bool mirror, bool two) {
    if (two) {
        if (p.precision == CFM_FP64)
            return mirror ? (const void *)j2d_resident2_kernel<double, true>
                          : (const void *)j2d_resident2_kernel<double, false>;
        return mirror ? (const void *)j2d_resident2_kernel<float, true>
                      : (const void *)j2d_resident2_kernel<float, false>;
    }
    if (p.precision == CFM_FP64)
        return mirror ? (const void *)j2d_resident_kernel<double, true>
                      : (const void *)j2d_resident_kernel<double, false>;
    return mirror ? (const void *)j2d_resident_kernel<float, true>
                  : (const void *)j2d_resident_kernel<float, false>;
}

dim3 block_of(const cfm_jacobi_params &p) { return p.dims == 2 ? dim3(256) : dim3(32, J3_TY); }

// Host-side sin factors shared by the host and device initial states.
void sin_factors(int n, std::vector<double> &out) {
    const double pi = 2.0 * std::asin(1.0);
    out.resize(n);
    for (int i = 0; i < n; ++i) out[i] = std::sin(2.0 * pi * (double)i / (double)(n - 1));
}

template <typename T>
void host_problem(const cfm_jacobi_params *p, int problem, T *a) {
    const int nx = p->nx, ny = p->ny, nz = p->dims == 3 ? p->nz : 1;
    std::memset(a, 0, sizeof(T) * grid_elems(p));
    if (p->dims == 2) {
        // 2D: the reference rounds pi to the grid type before the double sin
        // (Stencil/jacobi2D/include/common.h:24, src/common.cu:19).
        const T pi = (T)(2.0 * std::asin(1.0));
        for (int y = 0; y < ny; ++y) {
            const T v = (T)std::sin(2.0 * (double)pi * (double)y / (double)(ny - 1));
            a[(size_t)y * nx] = v;
            a[(size_t)y * nx + nx - 1] = v;
        }
        return;
    }
    std::vector<double> sy, sz;
    sin_factors(ny, sy);
    sin_factors(nz, sz);
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            const size_t row = ((size_t)z * ny + y) * nx;
            if (problem == CFM_PROBLEM_REF) {
                a[row] = (T)((T)z - (T)y) - (T)(nx - 1);
            } else {
                const T v = (T)(sy[y] * sz[z]);
                a[row] = v;
                a[row + nx - 1] = v;
            }
        }
}

int choose_launch(cfm_jacobi *h) {
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    h->num_sms = di.num_sms;
    h->smem_optin = di.smem_optin;
    const cfm_jacobi_params &p = h->p;
    const void *fn = sweep_fn_any(p, true, h->mirror);
    dim3 b = block_of(p);
    const int threads = (int)(b.x * b.y);
    int per_sm = 0;
    CFM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
    if (per_sm < 1) {
        set_error("sweep kernel cannot be resident");
        return CFM_UNSUPPORTED;
    }
    h->threads = threads;
    h->blocks = per_sm * di.num_sms;
    if (p.dims == 3) {
        const long long ntiles = (long long)((p.nx + 31) / 32) * ((p.ny - 2 + J3_TY - 1) / J3_TY);
        h->zchunk = pick_zchunk(ntiles, p.nz - 2, &h->blocks);
    } else {
        // no more blocks than there are warp work units (more only lengthen
        // the grid barrier): row segments of 32 columns, or for the
        // row-marching kernel tiles of 16-byte lanes over row chunks of at
        // least 8 rows
        const int vec = 16 / (int)h->esize;
        const bool march = p.nx % vec == 0 && !h->mirror;
        const long long units = march ? (long long)((p.nx + 32 * vec - 1) / (32 * vec)) * ((p.ny - 2 + 7) / 8)
                                      : (long long)((p.nx + 31) / 32) * (p.ny - 2);
        const long long need = (units * 32 + threads - 1) / threads;
        if (need < h->blocks) h->blocks = (int)std::max(1LL, need);
    }
    if (p.dims == 2 && p.impl == CFM_JACOBI_RESIDENT) {
        // One 1024-thread block per SM, each holding its band twice in shared
        // memory; used only when that fits on chip.  Preferred: two sweeps
        // per exchange (bands of >= 2 rows plus 2 halo rows each side), else
        // one (any band, 1 halo row each side).
        h->resident = false;
        for (int two = 1; two >= 0 && !h->resident; --two) {
            const int B = std::min(di.num_sms, two ? (p.ny - 2) / 2 : p.ny - 2);
            if (B < 1) continue;
            const int hmax = (p.ny - 2 + B - 1) / B;
            const size_t smem = 2 * (size_t)(hmax + (two ? 4 : 2)) * p.nx * h->esize;
            const void *rfn = resident_fn(p, h->mirror, two != 0);
            if (smem > di.smem_optin) continue;
            CFM_CUDA_TRY(cudaFuncSetAttribute(rfn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
            int rper = 0;
            CFM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rper, rfn, 1024, smem));
            if (rper >= 1) {
                h->resident = true;
                h->res_two = two != 0;
                h->res_blocks = B;
                h->res_smem = smem;
            }
        }
    }
    return CFM_OK;
}

template <typename T>
int launch_edge_preset(cfm_jacobi *h) {
    const cfm_jacobi_params &p = h->p;
    T *cur = (T *)h->buf[h->cur];
    const long long n = 4LL * p.nx + 4LL * p.ny + (p.dims == 3 ? 4LL * p.nz : 0);
    const int blocks = (int)std::min<long long>((n + 255) / 256, 1024);
    edge_preset_kernel<T><<<blocks, 256, 0, h->stream>>>(cur, (T *)h->buf[0], (T *)h->buf[1],
                                                         p.dims, p.nx, p.ny, p.dims == 3 ? p.nz : 1,
                                                         p.periodic_y);
    CFM_CUDA_TRY(cudaGetLastError());
    return CFM_OK;
}

// Reference single_gpu() host loop: sweep kernel, then the periodic halo
// copies with cudaMemcpyAsync (Stencil/jacobi3D/src/common.cu:174-215).
int host_loop_copy(cfm_jacobi *h, int niter, int *launches) {
    const cfm_jacobi_params &p = h->p;
    const void *fn = sweep_fn_any(p, false, h->mirror);
    const size_t es = h->esize;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    int one = 1;
    const dim3 block = block_of(p);
    for (int it = 0; it < niter; ++it) {
        void *in = h->buf[h->cur], *out = h->buf[h->cur ^ 1];
        void *args3[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, (void *)&p.nz, &one,
                         &h->zchunk, &h->bar};
        void *args2[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, &one, &h->bar};
        CFM_CUDA_TRY(cudaLaunchKernel(fn, dim3(h->blocks), block, p.dims == 3 ? args3 : args2, 0,
                                      h->stream));
        char *o = (char *)out;
        if (p.dims == 2) {
            const size_t row = (size_t)nx * es;
            CFM_CUDA_TRY(cudaMemcpyAsync(o, o + (size_t)(ny - 2) * row, row,
                                         cudaMemcpyDeviceToDevice, h->stream));
            CFM_CUDA_TRY(cudaMemcpyAsync(o + (size_t)(ny - 1) * row, o + row, row,
                                         cudaMemcpyDeviceToDevice, h->stream));
        } else {
            const size_t row = (size_t)nx * es, plane = row * ny;
            if (p.periodic_y) {
                CFM_CUDA_TRY(cudaMemcpy2DAsync(o + plane, plane, o + plane + (size_t)(ny - 2) * row,
                                               plane, row, nz - 2, cudaMemcpyDeviceToDevice,
                                               h->stream));
                CFM_CUDA_TRY(cudaMemcpy2DAsync(o + plane + (size_t)(ny - 1) * row, plane,
                                               o + plane + row, plane, row, nz - 2,
                                               cudaMemcpyDeviceToDevice, h->stream));
            }
            CFM_CUDA_TRY(cudaMemcpyAsync(o, o + (size_t)(nz - 2) * plane, plane,
                                         cudaMemcpyDeviceToDevice, h->stream));
            CFM_CUDA_TRY(cudaMemcpyAsync(o + (size_t)(nz - 1) * plane, o + plane, plane,
                                         cudaMemcpyDeviceToDevice, h->stream));
        }
        h->cur ^= 1;
        ++*launches;
    }
    return CFM_OK;
}

int host_loop_images(cfm_jacobi *h, int niter, int *launches) {
    const cfm_jacobi_params &p = h->p;
    const void *fn = sweep_fn_any(p, true, h->mirror);
    int one = 1;
    const dim3 block = block_of(p);
    for (int it = 0; it < niter; ++it) {
        void *in = h->buf[h->cur], *out = h->buf[h->cur ^ 1];
        void *args3[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, (void *)&p.nz, &one,
                         &h->zchunk, &h->bar};
        void *args2[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, &one, &h->bar};
        CFM_CUDA_TRY(cudaLaunchKernel(fn, dim3(h->blocks), block, p.dims == 3 ? args3 : args2, 0,
                                      h->stream));
        h->cur ^= 1;
        ++*launches;
    }
    return CFM_OK;
}

int resident2d(cfm_jacobi *h, int niter, int *launches) {
    const cfm_jacobi_params &p = h->p;
    CFM_CUDA_TRY(cudaMemsetAsync(h->flags, 0, sizeof(unsigned int) * h->res_blocks, h->stream));
    const void *in = h->buf[h->cur];
    void *fin = h->buf[h->cur ^ (niter & 1)];
    int n = niter;
    void *args[] = {(void *)&in, &fin, (void *)&p.nx, (void *)&p.ny, &n, &h->xbuf, &h->flags,
                    &h->bar};
    const void *fn = resident_fn(p, h->mirror, h->res_two);
    CFM_CUDA_TRY(launch_cooperative(fn, dim3(h->res_blocks), dim3(1024), args, h->res_smem,
                                    h->stream));
    h->cur ^= (niter & 1);
    ++*launches;
    return CFM_OK;
}

int launch_tma(cfm_jacobi *h, const TmaConfig &c, int count, int *launches) {
    const cfm_jacobi_params &p = h->p;
    // map[cur] / g0 is the grid read by the first pass
    const int cu = h->cur;
    void *g0 = h->buf[cu], *g1 = h->buf[cu ^ 1];
    int n = count, zc = c.zchunk;
    if (c.sweeps == 2) {
        void *args[] = {(void *)&c.map[cu], (void *)&c.map[cu ^ 1], (void *)&c.xmap[cu], (void *)&c.xmap[cu ^ 1],
                        &g0, &g1, (void *)&p.nx, (void *)&p.ny, (void *)&p.nz, &n, &zc, &h->bar};
        CFM_CUDA_TRY(launch_cooperative(c.fn, dim3(c.blocks), dim3(c.threads), args, c.smem, h->stream));
    } else {
        unsigned int *ud = h->dataflow && count > 1 ? h->udone : nullptr;
        if (ud) CFM_CUDA_TRY(cudaMemsetAsync(ud, 0, sizeof(unsigned int) * c.units, h->stream));
        void *args[] = {(void *)&c.map[cu], (void *)&c.map[cu ^ 1], &g0, &g1, (void *)&p.nx, (void *)&p.ny,
                        (void *)&p.nz, &n, &zc, &h->bar, &ud};
        CFM_CUDA_TRY(launch_cooperative(c.fn, dim3(c.blocks), dim3(c.threads), args, c.smem, h->stream));
    }
    h->cur ^= (count & 1);
    ++*launches;
    return CFM_OK;
}

// niter sweeps: one launch, or for two sweeps per pass niter / 2 passes and,
// for an odd count, one more launch of the one-sweep shape.
int persistent_tma(cfm_jacobi *h, int niter, int *launches) {
    if (h->tc.sweeps == 1) return launch_tma(h, h->tc, niter, launches);
    int st = CFM_OK;
    if (niter / 2 > 0 && (st = launch_tma(h, h->tc, niter / 2, launches))) return st;
    if (niter & 1) st = launch_tma(h, h->tail, 1, launches);
    return st;
}

int persistent(cfm_jacobi *h, int niter, int *launches) {
    const cfm_jacobi_params &p = h->p;
    if (h->resident) return resident2d(h, niter, launches);
    if (h->tma) return persistent_tma(h, niter, launches);
    const void *fn = sweep_fn_any(p, true, h->mirror);
    void *in = h->buf[h->cur], *out = h->buf[h->cur ^ 1];
    int n = niter;
    void *args3[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, (void *)&p.nz, &n, &h->zchunk,
                     &h->bar};
    void *args2[] = {&in, &out, (void *)&p.nx, (void *)&p.ny, &n, &h->bar};
    CFM_CUDA_TRY(launch_cooperative(fn, dim3(h->blocks), block_of(p),
                                    p.dims == 3 ? args3 : args2, 0, h->stream));
    h->cur ^= (niter & 1);
    ++*launches;
    return CFM_OK;
}

int reset_barrier(cfm_jacobi *h) {
    BarrierState s{};
    s.timeout_ns = barrier_timeout_ns();
    CFM_CUDA_TRY(cudaMemcpyAsync(h->bar, &s, sizeof(s), cudaMemcpyHostToDevice, h->stream));
    return CFM_OK;
}

// Enqueues the sweeps (no synchronisation).
int enqueue_sweeps(cfm_jacobi *h, int niter, int *launches) {
    if (niter == 0) return CFM_OK;
    int st;
    // (the mirror sweep reads the edge cells and writes whole rows: no preset)
    if (h->p.impl != CFM_JACOBI_HOST_LOOP && !h->mirror) {
        st = h->p.precision == CFM_FP64 ? launch_edge_preset<double>(h)
                                        : launch_edge_preset<float>(h);
        if (st) return st;
        ++*launches;
    }
    switch (h->p.impl) {
        case CFM_JACOBI_HOST_LOOP: return host_loop_copy(h, niter, launches);
        case CFM_JACOBI_HOST_LOOP_INKERNEL_HALO: return host_loop_images(h, niter, launches);
        default: return persistent(h, niter, launches);
    }
}

int finish_run(cfm_jacobi *h, int niter, int launches, double extra_h2d, double extra_d2h,
               cfm_stats *st) {
    CFM_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    CFM_CUDA_TRY(cudaEventSynchronize(h->ev1));
    BarrierState s{};
    CFM_CUDA_TRY(cudaMemcpy(&s, h->bar, sizeof(s), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    CFM_CUDA_TRY(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    int status = CFM_OK;
    if (s.error) {
        set_error("grid barrier %d timed out", s.where);
        status = CFM_BARRIER_TIMEOUT;
    }
    if (st) {
        const cfm_jacobi_params &p = h->p;
        std::memset(st, 0, sizeof(*st));
        const double lup = (double)(p.nx - 2) * (p.ny - 2) * (p.dims == 3 ? (p.nz - 2) : 1);
        st->seconds = ms * 1e-3;
        st->iterations = niter;
        st->lups = lup * niter;
        st->glups = st->seconds > 0 ? st->lups / st->seconds * 1e-9 : 0.0;
        st->bytes = st->lups * 2.0 * (double)h->esize;
        st->gbs = st->seconds > 0 ? st->bytes / st->seconds * 1e-9 : 0.0;
        st->h2d_bytes = extra_h2d;
        st->d2h_bytes = extra_d2h;
        st->launches = launches;
        st->status = status;
    }
    return status;
}

}  // namespace

extern "C" {

int cfm_jacobi_problem_host(const cfm_jacobi_params *p, int problem, void *host_grid) {
    int st = check_params(p);
    if (st) return st;
    CFM_ARG_CHECK(host_grid, "host_grid is null");
    CFM_ARG_CHECK(problem == CFM_PROBLEM_REF || problem == CFM_PROBLEM_CONFIG, "problem");
    if (p->precision == CFM_FP64)
        host_problem<double>(p, problem, (double *)host_grid);
    else
        host_problem<float>(p, problem, (float *)host_grid);
    return CFM_OK;
}

int cfm_jacobi_create(const cfm_jacobi_params *p, cfm_jacobi **out) {
    clear_error();
    int st = check_params(p);
    if (st) return st;
    CFM_ARG_CHECK(out, "out is null");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device visible");
        return CFM_NO_DEVICE;
    }
    cfm_jacobi *h = new cfm_jacobi();
    h->p = *p;
    if (h->p.dims == 2) {
        h->p.nz = 1;
        h->p.periodic_y = 1;
    }
    h->elems = grid_elems(&h->p);
    h->esize = p->precision == CFM_FP64 ? 8 : 4;
    auto fail = [&](int s) {
        cfm_jacobi_destroy(h);
        return s;
    };
    cudaError_t e;
    for (int i = 0; i < 2; ++i) {
        if ((e = cudaMalloc(&h->buf[i], h->elems * h->esize)) != cudaSuccess) {
            set_error("cudaMalloc of %zu bytes failed: %s", h->elems * h->esize,
                      cudaGetErrorString(e));
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR);
        }
    }
    if ((e = cudaMalloc(&h->bar, sizeof(BarrierState))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&h->ev1)) != cudaSuccess) {
        set_error("handle setup failed: %s", cudaGetErrorString(e));
        return fail(CFM_CUDA_ERROR);
    }
    h->own_stream = true;
    if ((st = choose_launch(h))) return fail(st);
    if (h->p.impl == CFM_JACOBI_PERSISTENT || h->p.impl == CFM_JACOBI_RESIDENT)
        if ((st = setup_tma(h, default_tma_variant()))) return fail(st);
    if (h->resident) {
        // exchange rows: 2 parities x blocks x 4 rows (the first and last two)
        const size_t xbytes = 2 * (size_t)h->res_blocks * 4 * h->p.nx * h->esize;
        if ((e = cudaMalloc(&h->xbuf, xbytes)) != cudaSuccess ||
            (e = cudaMalloc(&h->flags, sizeof(unsigned int) * h->res_blocks)) != cudaSuccess) {
            set_error("exchange buffers: %s", cudaGetErrorString(e));
            return fail(CFM_CUDA_ERROR);
        }
    }
    // Zero both grids on the handle's own (non-blocking) stream: a legacy-
    // stream memset would not be ordered before later work on that stream.
    for (int i = 0; i < 2; ++i)
        if ((e = cudaMemsetAsync(h->buf[i], 0, h->elems * h->esize, h->stream)) != cudaSuccess) {
            set_error("cudaMemsetAsync failed: %s", cudaGetErrorString(e));
            return fail(CFM_CUDA_ERROR);
        }
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) {
        set_error("grid zeroing failed: %s", cudaGetErrorString(e));
        return fail(CFM_CUDA_ERROR);
    }
    *out = h;
    return CFM_OK;
}

void cfm_jacobi_destroy(cfm_jacobi *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int i = 0; i < 2; ++i)
        if (h->buf[i]) cudaFree(h->buf[i]);
    if (h->bar) cudaFree(h->bar);
    if (h->xbuf) cudaFree(h->xbuf);
    if (h->flags) cudaFree(h->flags);
    if (h->udone) cudaFree(h->udone);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int cfm_jacobi_set_stream(cfm_jacobi *h, void *cuda_stream) {
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

int cfm_jacobi_set_boundary(cfm_jacobi *h, int boundary) {
    CFM_ARG_CHECK(h, "handle is null");
    CFM_ARG_CHECK(boundary == CFM_BOUNDARY_DIRICHLET || boundary == CFM_BOUNDARY_MIRROR,
                  "boundary must be CFM_BOUNDARY_DIRICHLET or CFM_BOUNDARY_MIRROR");
    CFM_ARG_CHECK(boundary == CFM_BOUNDARY_DIRICHLET || h->p.dims == 2,
                  "the mirror boundary is a 2D sweep");
    const bool m = boundary == CFM_BOUNDARY_MIRROR;
    if (m == h->mirror) return CFM_OK;
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->mirror = m;
    // the sweep kernel changes: its occupancy and work units set the grid
    return choose_launch(h);
}

int cfm_jacobi_set_dataflow(cfm_jacobi *h, int on) {
    CFM_ARG_CHECK(h, "handle is null");
    h->dataflow = on != 0;
    return CFM_OK;
}

int cfm_jacobi_load_problem(cfm_jacobi *h, int problem) {
    CFM_ARG_CHECK(h, "handle is null");
    CFM_ARG_CHECK(problem == CFM_PROBLEM_REF || problem == CFM_PROBLEM_CONFIG, "problem");
    const cfm_jacobi_params &p = h->p;
    std::vector<double> sy, sz(1, 0.0);
    if (p.dims == 2) {
        const double pi_t = p.precision == CFM_FP64 ? 2.0 * std::asin(1.0)
                                                    : (double)(float)(2.0 * std::asin(1.0));
        sy.resize(p.ny);
        for (int y = 0; y < p.ny; ++y) sy[y] = std::sin(2.0 * pi_t * (double)y / (double)(p.ny - 1));
    } else {
        sin_factors(p.ny, sy);
        sin_factors(p.nz, sz);
    }
    double *d = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&d, sizeof(double) * (sy.size() + sz.size())));
    cudaError_t e = cudaMemcpy(d, sy.data(), sizeof(double) * sy.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d + sy.size(), sz.data(), sizeof(double) * sz.size(),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int nz = p.dims == 3 ? p.nz : 1;
        for (int i = 0; i < 2; ++i) {
            if (p.precision == CFM_FP64)
                load_problem_kernel<double><<<4 * h->num_sms, 256, 0, h->stream>>>(
                    (double *)h->buf[i], p.dims, p.nx, p.ny, nz, problem, d, d + sy.size());
            else
                load_problem_kernel<float><<<4 * h->num_sms, 256, 0, h->stream>>>(
                    (float *)h->buf[i], p.dims, p.nx, p.ny, nz, problem, d, d + sy.size());
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    }
    cudaFree(d);
    CFM_CUDA_TRY(e);
    h->cur = 0;
    return CFM_OK;
}

int cfm_jacobi_upload(cfm_jacobi *h, const void *host_grid) {
    CFM_ARG_CHECK(h && host_grid, "null argument");
    const size_t bytes = h->elems * h->esize;
    CFM_CUDA_TRY(cudaMemcpyAsync(h->buf[0], host_grid, bytes, cudaMemcpyHostToDevice, h->stream));
    CFM_CUDA_TRY(cudaMemcpyAsync(h->buf[1], h->buf[0], bytes, cudaMemcpyDeviceToDevice, h->stream));
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->cur = 0;
    return CFM_OK;
}

int cfm_jacobi_download(cfm_jacobi *h, void *host_grid) {
    CFM_ARG_CHECK(h && host_grid, "null argument");
    CFM_CUDA_TRY(cudaMemcpyAsync(host_grid, h->buf[h->cur], h->elems * h->esize,
                                 cudaMemcpyDeviceToHost, h->stream));
    CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return CFM_OK;
}

int cfm_jacobi_run(cfm_jacobi *h, int niter, cfm_stats *st) {
    const cfm::NvtxRange nvtx_range("cfm_jacobi_run");
    CFM_ARG_CHECK(h, "handle is null");
    CFM_ARG_CHECK(niter >= 0, "niter must be >= 0");
    clear_error();
    int s = reset_barrier(h);
    if (s) return s;
    int launches = 0;
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    s = enqueue_sweeps(h, niter, &launches);
    if (s) return s;
    return finish_run(h, niter, launches, 0, 0, st);
}

int cfm_jacobi_run_host(cfm_jacobi *h, int niter, const void *host_in, void *host_out,
                        cfm_stats *st) {
    const cfm::NvtxRange nvtx_range("cfm_jacobi_run_host");
    CFM_ARG_CHECK(h && host_in && host_out, "null argument");
    CFM_ARG_CHECK(niter >= 0, "niter must be >= 0");
    clear_error();
    int s = reset_barrier(h);
    if (s) return s;
    const size_t bytes = h->elems * h->esize;
    int launches = 0;
    CFM_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    h->cur = 0;
    CFM_CUDA_TRY(cudaMemcpyAsync(h->buf[0], host_in, bytes, cudaMemcpyHostToDevice, h->stream));
    CFM_CUDA_TRY(cudaMemcpyAsync(h->buf[1], h->buf[0], bytes, cudaMemcpyDeviceToDevice, h->stream));
    s = enqueue_sweeps(h, niter, &launches);
    if (s) return s;
    CFM_CUDA_TRY(cudaMemcpyAsync(host_out, h->buf[h->cur], bytes, cudaMemcpyDeviceToHost,
                                 h->stream));
    return finish_run(h, niter, launches, (double)bytes, (double)bytes, st);
}

void *cfm_jacobi_device_grid(cfm_jacobi *h) { return h ? h->buf[h->cur] : nullptr; }

int cfm_jacobi_variant_info(int index, int *consumer_warps, int *rows_per_warp, int *stages) {
    int n = 0;
    const TmaVariant *v = tma_variants(&n);
    if (index < 0 || index >= n) return CFM_BAD_ARG;
    if (consumer_warps) *consumer_warps = v[index].cw;
    if (rows_per_warp) *rows_per_warp = v[index].rpw;
    if (stages) *stages = v[index].stages;
    return CFM_OK;
}

int cfm_jacobi_zchunk(cfm_jacobi *h) {
    if (!h) return CFM_BAD_ARG;
    return h->tma ? h->tc.zchunk : h->zchunk;
}

int cfm_jacobi_variant_sweeps(int index) {
    int n = 0;
    const TmaVariant *v = tma_variants(&n);
    if (index < 0 || index >= n) return CFM_BAD_ARG;
    return v[index].sweeps;
}

int cfm_jacobi_autotune(cfm_jacobi *h, int sweeps, int *best_variant, double *best_glups) {
    const cfm::NvtxRange nvtx_range("cfm_jacobi_autotune");
    CFM_ARG_CHECK(h, "handle is null");
    CFM_ARG_CHECK(sweeps >= 1, "sweeps must be >= 1");
    if (best_variant) *best_variant = -1;
    if (best_glups) *best_glups = 0.0;
    if (!h->tma) return CFM_OK;  // only the TMA pipeline has shapes to choose from
    const size_t bytes = h->elems * h->esize;
    void *saved = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&saved, bytes));
    auto restore = [&]() -> int {
        for (int i = 0; i < 2; ++i)
            CFM_CUDA_TRY(cudaMemcpyAsync(h->buf[i], saved, bytes, cudaMemcpyDeviceToDevice, h->stream));
        CFM_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->cur = 0;
        return CFM_OK;
    };
    int st = CFM_OK;
    cudaError_t e = cudaMemcpyAsync(saved, h->buf[h->cur], bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    int n = 0, best = -1, best_zc = 0;
    double best_rate = 0.0;
    tma_variants(&n);
    const int zcands[] = {0, 16, 24, 32, 48, 64, 128};  // 0: the cost-model choice
    for (int v = 0; v < n && e == cudaSuccess && st == CFM_OK; ++v) {
        for (int zc : zcands) {
            if ((st = setup_tma(h, v, zc)) || !h->tma) {
                st = CFM_OK;
                break;
            }
            // from the saved grid: a warm-up run, then the better of two timed
            // runs back to back (a run right after the 2-GB restore copy
            // favoured small z-chunks; the steady state is what a solve sees)
            double rate = 0.0;
            if ((st = restore())) break;
            for (int rep = 0; rep < 3 && st == CFM_OK; ++rep) {
                cfm_stats s{};
                if ((st = cfm_jacobi_run(h, sweeps, &s))) break;
                if (rep > 0) rate = std::max(rate, s.glups);
            }
            if (st) break;
            if (rate > best_rate) {
                best_rate = rate;
                best = v;
                best_zc = h->tc.zchunk;
            }
        }
    }
    const int st2 =
        (best >= 0) ? setup_tma(h, best, best_zc) : setup_tma(h, default_tma_variant());
    const int st3 = restore();
    cudaFree(saved);
    CFM_CUDA_TRY(e);
    if (st) return st;
    if (st2) return st2;
    if (st3) return st3;
    if (best_variant) *best_variant = best;
    if (best_glups) *best_glups = best_rate;
    return CFM_OK;
}

int cfm_jacobi_launch_shape(cfm_jacobi *h, int *blocks, int *threads) {
    CFM_ARG_CHECK(h, "handle is null");
    int b = h->blocks, t = h->threads;
    if (h->resident) {
        b = h->res_blocks;
        t = 1024;
    } else if (h->tma) {
        b = h->tc.blocks;
        t = h->tc.threads;
    }
    if (blocks) *blocks = b;
    if (threads) *threads = t;
    return CFM_OK;
}

}  // extern "C"
