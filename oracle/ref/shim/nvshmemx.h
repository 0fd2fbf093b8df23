/* Test harness only: CG/src/common.cu includes <nvshmemx.h> but calls none of
 * its extensions; everything it names is in the nvshmem.h stand-in. */
#ifndef CFM_REF_SHIM_NVSHMEMX_H
#define CFM_REF_SHIM_NVSHMEMX_H
#include "nvshmem.h"
#endif
