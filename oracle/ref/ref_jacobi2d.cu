// Test harness (oracle pinning only): exposes the reference's own single-GPU
// 2D Jacobi run -- single_gpu() of Stencil/jacobi2D/src/common.cu:154-273,
// compiled unmodified from the reference tree by oracle/Makefile -- through a
// C ABI so tests can compare the CPU oracle against the reference itself.
#include "common.h"  // Stencil/jacobi2D/include/common.h of the reference

extern "C" double ref_jacobi2d_single_gpu(int nx, int ny, int niter, float *out) {
    return single_gpu(nx, ny, niter, out, 1, false);
}

// The PERKS comparator: the same host loop with the mirror-boundary kernel
// (Stencil/jacobi2D/src/common.cu:44-66); nx must be a multiple of 32 there.
extern "C" double ref_jacobi2d_single_gpu_mirror(int nx, int ny, int niter, float *out) {
    return single_gpu(nx, ny, niter, out, 1, false, jacobi_kernel_single_gpu_mirror);
}
