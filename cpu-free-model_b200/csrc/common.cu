// Library-wide helpers: error strings, device info, cooperative launches and
// the barrier self-test.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "barrier.cuh"
#include "cfm_internal.h"

namespace cfm {

static thread_local char g_last_error[512] = "";
static double g_barrier_timeout_ms = 2000.0;

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

void clear_error() { g_last_error[0] = 0; }

unsigned long long barrier_timeout_ns() {
    return (unsigned long long)(g_barrier_timeout_ms * 1e6);
}

int current_device_info(DeviceInfo *out) {
    static std::mutex mu;
    static DeviceInfo cache[64];
    int dev = 0;
    CFM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("device index %d out of range", dev);
        return CFM_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (cache[dev].device != dev) {
        cudaDeviceProp prop;
        CFM_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
        cache[dev].device = dev;
        cache[dev].num_sms = prop.multiProcessorCount;
        cache[dev].cc_major = prop.major;
        cache[dev].cc_minor = prop.minor;
        cache[dev].smem_optin = prop.sharedMemPerBlockOptin;
    }
    *out = cache[dev];
    return CFM_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

cudaError_t launch_cooperative(const void *fn, dim3 grid, dim3 block, void **args, size_t smem,
                               cudaStream_t s) {
    return cudaLaunchCooperativeKernel(fn, grid, block, args, smem, s);
}

// Self-test kernel: `rounds` barriers; block `drop` skips its first arrival
// (and then leaves), so every other block must come back through the timeout.
__global__ void barrier_selftest_kernel(BarrierState *b, int rounds, int drop, int *visits) {
    if ((int)blockIdx.x == drop) return;  // this block never arrives
    for (int r = 0; r < rounds; ++r) {
        if (threadIdx.x == 0) atomicAdd(visits, 1);
        if (!grid_barrier(b, gridDim.x, r)) return;
    }
}

}  // namespace cfm

extern "C" {

int cfm_api_version(void) { return CFM_API_VERSION; }

const char *cfm_status_string(int status) {
    switch (status) {
        case CFM_OK: return "ok";
        case CFM_BAD_ARG: return "bad argument";
        case CFM_CUDA_ERROR: return "CUDA error";
        case CFM_BARRIER_TIMEOUT: return "grid barrier timeout";
        case CFM_BREAKDOWN: return "CG breakdown";
        case CFM_NOT_CONVERGED: return "not converged";
        case CFM_NO_DEVICE: return "no CUDA device";
        case CFM_UNSUPPORTED: return "unsupported";
        case CFM_OUT_OF_MEMORY: return "out of device memory";
        default: return "unknown status";
    }
}

const char *cfm_last_error(void) { return cfm::g_last_error; }

int cfm_set_barrier_timeout_ms(double ms) {
    CFM_ARG_CHECK(ms > 0 && ms < 3.6e6, "barrier timeout must be in (0, 1 h)");
    cfm::g_barrier_timeout_ms = ms;
    return CFM_OK;
}

int cfm_device_info(int *num_sms, int *cc_major, int *cc_minor) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        cfm::set_error("no CUDA device visible");
        return CFM_NO_DEVICE;
    }
    cfm::DeviceInfo di;
    int st = cfm::current_device_info(&di);
    if (st) return st;
    if (num_sms) *num_sms = di.num_sms;
    if (cc_major) *cc_major = di.cc_major;
    if (cc_minor) *cc_minor = di.cc_minor;
    return CFM_OK;
}

int cfm_barrier_selftest(int blocks, int rounds, int drop_block, double *elapsed_ms) {
    CFM_ARG_CHECK(rounds >= 1 && rounds <= 1000000, "rounds");
    cfm::DeviceInfo di;
    int st = cfm::current_device_info(&di);
    if (st) return st;
    if (blocks <= 0) blocks = di.num_sms;
    CFM_ARG_CHECK(blocks <= di.num_sms, "blocks must not exceed the SM count (co-residency)");
    CFM_ARG_CHECK(drop_block < blocks, "drop_block");
    cfm::BarrierState *b = nullptr;
    int *visits = nullptr;
    CFM_CUDA_TRY(cudaMalloc(&b, sizeof(cfm::BarrierState)));
    cudaError_t e = cudaMalloc(&visits, sizeof(int));
    if (e != cudaSuccess) {
        cudaFree(b);
        CFM_CUDA_TRY(e);
    }
    cfm::BarrierState h{};
    h.timeout_ns = cfm::barrier_timeout_ns();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int result = CFM_OK;
    do {
        if ((e = cudaMemcpy(b, &h, sizeof(h), cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = cudaMemset(visits, 0, sizeof(int))) != cudaSuccess) break;
        void *args[] = {&b, &rounds, &drop_block, &visits};
        cudaEventRecord(e0, 0);
        if ((e = cfm::launch_cooperative((const void *)cfm::barrier_selftest_kernel, dim3(blocks),
                                         dim3(128), args, 0, 0)) != cudaSuccess)
            break;
        cudaEventRecord(e1, 0);
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) break;
        if ((e = cudaMemcpy(&h, b, sizeof(h), cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (elapsed_ms) *elapsed_ms = ms;
        if (h.error) {
            cfm::set_error("grid barrier %d timed out", h.where);
            result = CFM_BARRIER_TIMEOUT;
        }
    } while (0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(b);
    cudaFree(visits);
    if (e != cudaSuccess) {
        cfm::set_error("barrier self-test: %s", cudaGetErrorString(e));
        return CFM_CUDA_ERROR;
    }
    return result;
}

}  // extern "C"
