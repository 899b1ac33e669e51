/* Host-side DCF-spline key/cache sizing. Replaces include/FastFss/spline.h:29-75 of the
 * reference (argument order degree, intervalNum, bitWidthIn, bitWidthOut, elementSize,
 * elementNum; values from src/impl/spline.h:27-48). */
#ifndef FAST_FSS_SPLINE_H
#define FAST_FSS_SPLINE_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_dcfSplineKeyZip(void *zippedKey, size_t zippedKeyDataSize, const void *key,
                                         size_t keyDataSize, size_t degree, size_t intervalNum, size_t bitWidthIn,
                                         size_t bitWidthOut, size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dcfSplineKeyUnzip(void *key, size_t keyDataSize, const void *zippedKey,
                                           size_t zippedKeyDataSize, size_t degree, size_t intervalNum,
                                           size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                           size_t elementNum);

FAST_FSS_API int FastFss_dcfSplineGetCacheDataSize(size_t *cacheDataSize, size_t degree, size_t intervalNum,
                                                   size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                   size_t elementNum);

FAST_FSS_API int FastFss_dcfSplineGetKeyDataSize(size_t *keyDataSize, size_t degree, size_t intervalNum,
                                                 size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                 size_t elementNum);

FAST_FSS_API int FastFss_dcfSplineGetZippedKeyDataSize(size_t *keyDataSize, size_t degree, size_t intervalNum,
                                                       size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                       size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
