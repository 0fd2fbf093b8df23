// Thin wrappers over the sm_90+/sm_100 PTX used by the TMA-fed stencil
// pipelines: mbarrier init/arrive/wait (bounded) and tiled bulk-tensor loads
// (single CTA, no multicast).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "barrier.cuh"

namespace cfm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of `bar` to complete, for at most `budget_ns`.
// Returns false on timeout (the caller records the error and unwinds).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity,
                                                  unsigned long long budget_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > budget_ns) return false;
    }
    return true;
}

// Orders this thread's earlier generic-proxy accesses to the CTA's shared
// memory before later async-proxy (TMA) accesses to it.  A consumer of a
// TMA-filled ring slot runs it after its last read of the slot and before
// the arrive that lets the producer refill the slot; without it the refill
// was seen, under heavy memory traffic, by reads that precede the arrive in
// program order.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's generic-proxy view of global memory before its later
// async-proxy (TMA) reads.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst_smem, const CUtensorMap *map, int x, int y,
                                            int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst_smem)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace cfm
