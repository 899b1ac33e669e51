/* DCF key generation / evaluation on the GPU. Replaces include/FastFss/cuda/dcf.h:85-183 of
 * the reference with identical prototypes, validation order, error codes and byte layouts.
 *
 * Every data pointer is device memory (key 16-byte aligned); sizes are in bytes; the call
 * is asynchronous on *(cudaStream_t*)cudaStreamPtr, or on cudaStreamPerThread when the
 * pointer is NULL. beta == NULL means beta = 1. The optional cache is accepted for
 * compatibility (its size is validated) but is not needed and not written. */
#ifndef FAST_FSS_CUDA_DCF_H
#define FAST_FSS_CUDA_DCF_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_dcfKeyGen(void *key, size_t keyDataSize, const void *alpha, size_t alphaDataSize,
                                        const void *beta, size_t betaDataSize, const void *seed0,
                                        size_t seedDataSize0, const void *seed1, size_t seedDataSize1,
                                        size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                        size_t elementNum, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_dcfEval(void *sharedOut, size_t sharedOutSize, const void *maskedX,
                                      size_t maskedXDataSize, const void *key, size_t keyDataSize, const void *seed,
                                      size_t seedDataSize, int partyId, size_t bitWidthIn, size_t bitWidthOut,
                                      size_t groupSize, size_t elementSize, size_t elementNum, void *cache,
                                      size_t cacheDataSize, void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
