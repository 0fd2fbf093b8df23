// Internal declarations shared by the libcfm translation units.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <utility>

#include "cfm.h"
#include "nvtx3/nvToolsExt.h"

namespace cfm {

// Records a one-line error message for cfm_last_error() (thread-local).
void set_error(const char *fmt, ...);
void clear_error();

// Barrier wait budget in nanoseconds (cfm_set_barrier_timeout_ms).
unsigned long long barrier_timeout_ns();

struct DeviceInfo {
    int device = -1;
    int num_sms = 0;
    int cc_major = 0, cc_minor = 0;
    size_t smem_optin = 0;
};
// Queries (and caches per device) the current device's properties.
int current_device_info(DeviceInfo *out);

// Device-side state of one grid barrier; see barrier.cuh.
struct BarrierState {
    // count (low) and gen (high) are updated as one 64-bit word
    unsigned int count;   // arrivals in the current generation
    unsigned int gen;     // generation, bumped by the last arrival
    int error;            // set to 1 by a wait that ran out of budget
    int where;            // barrier index at which the first timeout happened
    unsigned long long timeout_ns;
};

// cuTensorMapEncodeTiled from the driver (nullptr when unavailable).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Kernel launch helper: cooperative launch so that every block is resident
// (the barrier needs co-residency).
cudaError_t launch_cooperative(const void *fn, dim3 grid, dim3 block, void **args, size_t smem,
                               cudaStream_t s);

// Programmatic dependent launch: the kernel may be scheduled while its
// predecessor in the stream is still running, which hides the launch gap
// between the short kernels of a solver iteration.  Every kernel launched
// this way starts with pdl_enter() (griddepcontrol.wait: the predecessor has
// completed and its writes are visible) before it touches global memory.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

#ifdef __CUDACC__
// Waits for the stream predecessor (no-op without a programmatic launch),
// then lets the successor be scheduled.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_enter() {
    pdl_wait();
    pdl_trigger();
}
#endif

// NVTX range over a host phase (the reference's PUSH_RANGE / POP_RANGE
// tracing, Stencil/jacobi2D/include/common.h:81-105): visible in a profiler
// timeline, free when none is attached (NVTX v3 loads its back end lazily).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace cfm

#define CFM_CUDA_TRY(call)                                                                    \
    do {                                                                                      \
        cudaError_t cfm_e_ = (call);                                                          \
        if (cfm_e_ != cudaSuccess) {                                                          \
            cfm::set_error("%s failed: %s (%d) at %s:%d", #call, cudaGetErrorString(cfm_e_), \
                           (int)cfm_e_, __FILE__, __LINE__);                                  \
            return cfm_e_ == cudaErrorMemoryAllocation ? CFM_OUT_OF_MEMORY : CFM_CUDA_ERROR;  \
        }                                                                                     \
    } while (0)

#define CFM_ARG_CHECK(cond, msg)                      \
    do {                                              \
        if (!(cond)) {                                \
            cfm::set_error("bad argument: %s", msg);  \
            return CFM_BAD_ARG;                       \
        }                                             \
    } while (0)
