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

#include <cstddef>

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

// The barrier word: BarrierState::count (low 32 bits) and ::gen (high 32
// bits) read and written as one 64-bit value.
static_assert(offsetof(BarrierState, count) == 0 && offsetof(BarrierState, gen) == 4 &&
                  alignof(BarrierState) >= 8,
              "count and gen form one aligned 64-bit word");
__device__ __forceinline__ unsigned long long *barrier_word(BarrierState *b) {
    return reinterpret_cast<unsigned long long *>(&b->count);
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Arrival: fetch-add on the word with acquire-release order at GPU scope, so
// the block's writes (ordered before it by the block barrier) are released
// with the arrival and the last arriver acquires every earlier block's.
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p,
                                                                  unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;"
                 : "=l"(old)
                 : "l"(p), "l"(v)
                 : "memory");
    return old;
}

// The last arriver's release: one add that sets the count back to 0 and
// bumps the generation, cumulative over the arrivals it acquired.
__device__ __forceinline__ void red_add_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Generation-counting barrier over all `nblocks` blocks of the grid.
// Returns true when every block arrived; false once any wait timed out (the
// caller must then leave its loop).  `site` labels the barrier for the
// error report.  A block arrives with one fetch-add on the 64-bit word
// (count, gen); the block that brings the count to nblocks adds
// 2^32 - nblocks in one operation (count back to 0, next generation), and
// the others wait for the generation they arrived in to pass.  A single
// block needs only the block barrier, which orders the block's
// global-memory accesses for its own threads.
__device__ __forceinline__ bool grid_barrier(BarrierState *b, unsigned int nblocks, int site) {
    __shared__ int s_ok;
    __syncthreads();
    if (nblocks == 1) return true;
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        int ok = 1;
        unsigned long long *w = barrier_word(b);
        const unsigned long long old = atom_add_acq_rel_u64(w, 1ull);
        const unsigned int g = (unsigned int)(old >> 32);
        if ((unsigned int)old == nblocks - 1) {
            red_add_release_u64(w, (1ull << 32) - nblocks);
        } else {
            // the acquire load that sees the next generation synchronises
            // with the last arriver's release
            const unsigned long long t0 = global_ns();
            const unsigned long long budget = b->timeout_ns;
            for (unsigned int n = 1; (unsigned int)(ld_acquire_u64(w) >> 32) == g; ++n) {
                if ((n & 63) == 0) {
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
        }
        if (ld_relaxed_i32(&b->error)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace cfm
