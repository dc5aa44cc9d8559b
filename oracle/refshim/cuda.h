/* Test infrastructure (oracle build only): the reference's host sources
 * include <cuda.h>; the CPU oracle build needs only the runtime shim. */
#ifndef CBM_REFSHIM_CUDA_H
#define CBM_REFSHIM_CUDA_H
#include "cuda_runtime.h"
#endif
