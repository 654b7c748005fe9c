/* Host emulation stand-in for <cuda.h> (test infrastructure only; see cuda_runtime.h). */
#ifndef HCG_SHIM_CUDA_H
#define HCG_SHIM_CUDA_H
#include "cuda_runtime.h"
#endif
