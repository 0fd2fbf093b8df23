/* Test harness only (oracle pinning): a stand-in for the two NVSHMEM device
 * calls that the reference's CG/src/common.cu names in its multi-GPU kernels
 * (NVSHMEM::gpuSpMV, CG/src/common.cu:250-280).  The harness in ref_cg.cu
 * only runs the single-GPU discrete solver (CG/src/common.cu:399-538), which
 * never launches those kernels, so these bodies are never executed; they
 * exist so that the reference file compiles unmodified without NVSHMEM. */
#ifndef CFM_REF_SHIM_NVSHMEM_H
#define CFM_REF_SHIM_NVSHMEM_H

__device__ inline int nvshmem_my_pe(void) { return 0; }

/* one-PE reading: the "remote" element is the local one */
__device__ inline double nvshmem_double_g(const double *src, int pe) {
    (void)pe;
    return *src;
}

#endif
