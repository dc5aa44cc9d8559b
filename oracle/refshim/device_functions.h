/* Test infrastructure (oracle build only): empty stand-in for CUDA's
 * device_functions.h, which the reference's host headers include
 * (CBM_CORE_LIB_MGPU_DEV/CBMCoreInclude/cuda/kernels.h:10). */
#ifndef CBM_REFSHIM_DEVICE_FUNCTIONS_H
#define CBM_REFSHIM_DEVICE_FUNCTIONS_H
#endif
