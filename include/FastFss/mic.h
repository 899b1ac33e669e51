/* Host-side DCF-MIC key/cache sizing. Replaces include/FastFss/mic.h:29-62 of the reference
 * (a DCF key with groupSize 1, src/mic.cpp). */
#ifndef FAST_FSS_MIC_H
#define FAST_FSS_MIC_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_dcfMICKeyZip(void *zippedKey, size_t zippedKeyDataSize, const void *key,
                                      size_t keyDataSize, size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                      size_t elementNum);

FAST_FSS_API int FastFss_dcfMICKeyUnzip(void *key, size_t keyDataSize, const void *zippedKey,
                                        size_t zippedKeyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                        size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dcfMICGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dcfMICGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                              size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dcfMICGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                    size_t elementSize, size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
