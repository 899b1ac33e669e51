/* Grotto (Z_2 DPF with 64-bit leaves) on the GPU. Replaces include/FastFss/cuda/grotto.h:13-102
 * of the reference with identical prototypes, validation, error codes and layouts.
 * Conventions as in <FastFss/cuda/dcf.h>. */
#ifndef FAST_FSS_CUDA_GROTTO_H
#define FAST_FSS_CUDA_GROTTO_H

#include <FastFss/api.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_grottoKeyGen(void *key, size_t keyDataSize, const void *alpha, size_t alphaDataSize,
                                           const void *seed0, size_t seedDataSize0, const void *seed1,
                                           size_t seedDataSize1, size_t bitWidthIn, size_t elementSize,
                                           size_t elementNum, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_grottoEqEval(void *sharedBooleanOut, size_t sharedOutDataSize, const void *maskedX,
                                           size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                           const void *seed, size_t seedDataSize, int partyId, size_t bitWidthIn,
                                           size_t elementSize, size_t elementNum, void *cache, size_t cacheDataSize,
                                           void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_grottoEval(void *sharedBooleanOut, size_t sharedOutDataSize, const void *maskedX,
                                         size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                         const void *seed, size_t seedDataSize, bool equalBound, int partyId,
                                         size_t bitWidthIn, size_t elementSize, size_t elementNum, void *cache,
                                         size_t cacheDataSize, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_grottoMICEval(void *sharedBooleanOut, size_t sharedBooleanOutDataSize,
                                            const void *maskedX, size_t maskedXDataSize, const void *key,
                                            size_t keyDataSize, const void *seed, size_t seedDataSize, int partyId,
                                            const void *leftEndpoints, size_t leftEndpointsDataSize,
                                            const void *rightEndpoints, size_t rightEndpointsDataSize,
                                            size_t bitWidthIn, size_t elementSize, size_t elementNum, void *cache,
                                            size_t cacheDataSize, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_grottoIntervalLutEval(void *sharedOutE, size_t sharedOutEDataSize, void *sharedOutT,
                                                    size_t sharedOutTDataSize, const void *maskedX,
                                                    size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                    const void *seed, size_t seedDataSize, int partyId,
                                                    const void *leftEndpoints, size_t leftEndpointsDataSize,
                                                    const void *rightEndpoints, size_t rightEndpointsDataSize,
                                                    const void *lookUpTable, size_t lookUpTableDataSize,
                                                    size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                    size_t elementNum, void *cache, size_t cacheDataSize,
                                                    void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
