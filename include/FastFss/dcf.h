/* Host-side DCF key/cache sizing (no device work). Replaces include/FastFss/dcf.h:62-206 of
 * the reference; values are identical (src/impl/dcf.h:38-67). Zip/Unzip are not
 * implemented by the reference either (src/dcf.cpp:10-34) and return FAST_FSS_RUNTIME_ERROR;
 * the zipped size is 0. */
#ifndef FAST_FSS_DCF_H
#define FAST_FSS_DCF_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_dcfKeyZip(void *zippedKey, size_t zippedKeyDataSize, const void *key, size_t keyDataSize,
                                   size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                   size_t elementNum);

FAST_FSS_API int FastFss_dcfKeyUnzip(void *key, size_t keyDataSize, const void *zippedKey, size_t zippedKeyDataSize,
                                     size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                     size_t elementNum);

/* elementNum * (16 n + es n g + 2 es + es g) */
FAST_FSS_API int FastFss_dcfGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                           size_t groupSize, size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dcfGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                 size_t groupSize, size_t elementSize, size_t elementNum);

/* elementNum * (16 n + es n g) */
FAST_FSS_API int FastFss_dcfGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                             size_t groupSize, size_t elementSize, size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
