// Test harness (oracle pinning only): exposes the reference's own single-GPU
// conjugate gradient -- SingleGPUDiscreteStandard::run_single_gpu() of
// CG/src/common.cu:399-538 (b = ones, x0 = 0, exactly iter_max iterations,
// dots summed with atomicAdd(double)) -- and its random tridiagonal generator
// genTridiag() (CG/src/common.cu:46-76), both compiled unmodified from the
// reference tree by oracle/Makefile, through a C ABI.  The NVSHMEM calls of
// that file's multi-GPU kernels resolve to the stand-ins in shim/.
#include <cstdlib>

#include <cuda_runtime.h>

#include "common.h"  // CG/include/common.h of the reference

// Standard CG on a host CSR matrix (copied to the device here, as the
// reference's main() does at CG/src/main.cu:188-197).  Writes x to x_out and
// returns the solve's seconds as run_single_gpu() measures them, or a
// negative value when a CUDA call failed.
extern "C" double ref_cg_standard(int n, int nnz, const int *rowptr, const int *col,
                                  const double *val, int zero_indexed, int iter_max,
                                  double *x_out) {
    int *d_rowptr = nullptr, *d_col = nullptr;
    double *d_val = nullptr;
    if (cudaMalloc((void **)&d_rowptr, sizeof(int) * (n + 1)) != cudaSuccess ||
        cudaMalloc((void **)&d_col, sizeof(int) * nnz) != cudaSuccess ||
        cudaMalloc((void **)&d_val, sizeof(double) * nnz) != cudaSuccess) {
        cudaFree(d_rowptr);
        cudaFree(d_col);
        cudaFree(d_val);
        return -1.0;
    }
    cudaMemcpy(d_rowptr, rowptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(d_col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(d_val, val, sizeof(double) * nnz, cudaMemcpyHostToDevice);
    const double t = SingleGPUDiscreteStandard::run_single_gpu(
        iter_max, d_rowptr, d_col, d_val, x_out, n, nnz, zero_indexed != 0, false);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaFree(d_rowptr);
    cudaFree(d_col);
    cudaFree(d_val);
    return err == cudaSuccess ? t : -1.0;
}

// genTridiag with libc rand() first put in its unseeded start state (glibc
// documents that no seed is the same as srand(1)), as in a fresh reference
// process.  nnz = 3 (n - 2) + 4.
extern "C" int ref_gen_tridiag(int n, int *rowptr, int *col, double *val) {
    if (n < 2) return -1;
    srand(1);
    genTridiag(rowptr, col, val, n, 3 * (n - 2) + 4);
    return 0;
}
