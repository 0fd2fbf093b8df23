// Device-wide barrier for persistent kernels, with a bounded wait.
//
// The reference synchronises its persistent kernels with cg::sync(grid)
// (e.g. Stencil/jacobi2D/src/single-stream/multi-threaded-two-block-comm.cu:95)
// and spins without limit on peer flags (Stencil/jacobi2D/src/multi-stream/
// multi-gpu-peer-tiling.cu:47-49).  Here every wait has a time budget: a
// block that waits longer than BarrierState::timeout_ns sets the error word,
// every block leaves its loop at the next barrier, and the host turns the
// word into CFM_BARRIER_TIMEOUT.  A lost arrival therefore ends the kernel
// instead of hanging the GPU.
#pragma once

#include "cfm_internal.h"

namespace cfm {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Arrival: fetch-add with acquire-release order at GPU scope, so the block's
// writes (ordered before it by the block barrier) are released with the
// arrival and the last arriver acquires every earlier block's.
__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(p), "r"(v)
                 : "memory");
    return old;
}

// Generation bump by the last arriver: a release, cumulative over the
// arrivals it acquired.
__device__ __forceinline__ void red_add_release_u32(unsigned int *p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Generation-counting barrier over all `nblocks` blocks of the grid.
// Returns true when every block arrived; false once any wait timed out (the
// caller must then leave its loop).  `site` labels the barrier for the
// error report.  A single block needs only the block barrier, which orders
// the block's global-memory accesses for its own threads.
__device__ __forceinline__ bool grid_barrier(BarrierState *b, unsigned int nblocks, int site) {
    __shared__ int s_ok;
    __syncthreads();
    if (nblocks == 1) return true;
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        int ok = 1;
        // the generation cannot move before this block arrives
        const unsigned int g = ld_acquire_u32(&b->gen);
        const unsigned int arrived = atom_add_acq_rel_u32(&b->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&b->count, 0u);
            red_add_release_u32(&b->gen, 1u);
        } else {
            // the acquire load that sees the new generation synchronises
            // with the last arriver's release
            const unsigned long long t0 = global_ns();
            const unsigned long long budget = b->timeout_ns;
            while (ld_acquire_u32(&b->gen) == g) {
                if (ld_relaxed_i32(&b->error)) {
                    ok = 0;
                    break;
                }
                if (global_ns() - t0 > budget) {
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

}  // namespace cfm
