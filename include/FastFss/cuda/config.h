/* Launch-configuration knobs kept from include/FastFss/cuda/config.h:18-30 of the reference
 * (defaults 128 and 64, set functions return -2 for dim <= 0, access under a mutex). The
 * values are stored and returned for compatibility only: the sm_100a kernels size their
 * grids from the device's SM count and per-kernel occupancy instead. */
#ifndef FAST_FSS_CUDA_CONFIG
#define FAST_FSS_CUDA_CONFIG

#include <FastFss/api.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_setGridDim(int dim);

FAST_FSS_API int FastFss_cuda_getGridDim();

FAST_FSS_API int FastFss_cuda_getFineGrainParallelGridDimThreshold();

FAST_FSS_API int FastFss_cuda_setFineGrainParallelGridDimThreshold(int dim);

#ifdef __cplusplus
}
#endif

#endif
