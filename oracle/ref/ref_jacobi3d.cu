// Test harness (oracle pinning only): exposes the reference's own single-GPU
// 3D Jacobi run -- single_gpu() of Stencil/jacobi3D/src/common.cu:110-239,
// compiled unmodified from the reference tree by oracle/Makefile -- through a
// C ABI so tests can compare the CPU oracle against the reference itself.
#include "common.h"  // Stencil/jacobi3D/include/common.h of the reference

extern "C" double ref_jacobi3d_single_gpu(int nx, int ny, int nz, int niter, float *out) {
    return single_gpu(nz, ny, nx, niter, out, 1, false);
}
