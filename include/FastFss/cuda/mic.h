/* DCF-based multiple interval containment on the GPU. Replaces include/FastFss/cuda/mic.h:14-55
 * of the reference with identical prototypes, validation, error codes and layouts. */
#ifndef FAST_FSS_CUDA_MIC_H
#define FAST_FSS_CUDA_MIC_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_dcfMICKeyGen(void *key, size_t keyDataSize, void *z, size_t zDataSize,
                                           const void *alpha, size_t alphaDataSize, const void *seed0,
                                           size_t seedDataSize0, const void *seed1, size_t seedDataSize1,
                                           const void *leftEndpoints, size_t leftEndpointsDataSize,
                                           const void *rightEndpoints, size_t rightEndpointsDataSize,
                                           size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                           size_t elementNum, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_dcfMICEval(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                         size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                         const void *sharedZ, size_t sharedZDataSize, const void *seed,
                                         size_t seedDataSize, int partyId, const void *leftEndpoints,
                                         size_t leftEndpointsDataSize, const void *rightEndpoints,
                                         size_t rightEndpointsDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                         size_t elementSize, size_t elementNum, void *cache, size_t cacheDataSize,
                                         void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
