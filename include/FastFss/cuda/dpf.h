/* DPF key generation / evaluation on the GPU. Replaces include/FastFss/cuda/dpf.h:13-84 of
 * the reference (dpfKeyGen, dpfEval, dpfEvalAll, dpfEvalMulti) with identical prototypes,
 * validation, error codes and layouts. Conventions as in <FastFss/cuda/dcf.h>. */
#ifndef FAST_FSS_CUDA_DPF_H
#define FAST_FSS_CUDA_DPF_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_dpfKeyGen(void *key, size_t keyDataSize, const void *alpha, size_t alphaDataSize,
                                        const void *beta, size_t betaDataSize, const void *seed0,
                                        size_t seedDataSize0, const void *seed1, size_t seedDataSize1,
                                        size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                        size_t elementNum, void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_dpfEval(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                      size_t maskedXDataSize, const void *key, size_t keyDataSize, const void *seed,
                                      size_t seedDataSize, int partyId, size_t bitWidthIn, size_t bitWidthOut,
                                      size_t groupSize, size_t elementSize, size_t elementNum, void *cache,
                                      size_t cacheDataSize, void *cudaStreamPtr);

/* out[i][(maskedX_i - x) mod 2^n][g] = dpfEval(key_i, x) for every x < 2^n. */
FAST_FSS_API int FastFss_cuda_dpfEvalAll(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                         size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                         const void *seed, size_t seedDataSize, int partyId, size_t bitWidthIn,
                                         size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                         size_t elementNum, void *cache, size_t cacheDataSize, void *cudaStreamPtr);

/* out[i][j][g] = dpfEval(key_i, maskedX_i - point_j). */
FAST_FSS_API int FastFss_cuda_dpfEvalMulti(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                           size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                           const void *seed, size_t seedDataSize, int partyId, const void *point,
                                           size_t pointDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                           size_t groupSize, size_t elementSize, size_t elementNum, void *cache,
                                           size_t cacheDataSize, void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
