/* Host emulation stand-in: threadIdx/blockIdx/blockDim live in cuda_runtime.h (test infrastructure only). */
#ifndef HCG_SHIM_DEVICE_LAUNCH_PARAMETERS_H
#define HCG_SHIM_DEVICE_LAUNCH_PARAMETERS_H
#include "cuda_runtime.h"
#endif
