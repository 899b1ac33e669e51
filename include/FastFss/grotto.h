/* Host-side Grotto key/cache sizing. Replaces include/FastFss/grotto.h:27-56 of the
 * reference (src/impl/grotto.h:37-85). The zipped size is SIZE_MAX, as in the reference. */
#ifndef FAST_FSS_GROTTO_H
#define FAST_FSS_GROTTO_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_grottoKeyZip(void *zippedKey, size_t zippedKeyDataSize, const void *key,
                                      size_t keyDataSize, size_t bitWidthIn, size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_grottoKeyUnzip(void *key, size_t keyDataSize, const void *zippedKey,
                                        size_t zippedKeyDataSize, size_t bitWidthIn, size_t elementSize,
                                        size_t elementNum);

/* elementNum * (16 (n - 6) + 8 + 2 es) */
FAST_FSS_API int FastFss_grottoGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementSize,
                                              size_t elementNum);

FAST_FSS_API int FastFss_grottoGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementSize,
                                                    size_t elementNum);

/* elementNum * (16 (n - 6) + (n - 6)) */
FAST_FSS_API int FastFss_grottoGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t elementSize,
                                                size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
