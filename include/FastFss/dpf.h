/* Host-side DPF key/cache sizing. Replaces include/FastFss/dpf.h:27-64 of the reference
 * (values from src/impl/dpf.h:35-61; the cache size takes no bitWidthOut/groupSize). */
#ifndef FAST_FSS_DPF_H
#define FAST_FSS_DPF_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_dpfKeyZip(void *zippedKey, size_t zippedKeyDataSize, const void *key, size_t keyDataSize,
                                   size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                   size_t elementNum);

FAST_FSS_API int FastFss_dpfKeyUnzip(void *key, size_t keyDataSize, const void *zippedKey, size_t zippedKeyDataSize,
                                     size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                     size_t elementNum);

/* elementNum * (16 n + 2 es + es g) */
FAST_FSS_API int FastFss_dpfGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                           size_t groupSize, size_t elementSize, size_t elementNum);

FAST_FSS_API int FastFss_dpfGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                 size_t groupSize, size_t elementSize, size_t elementNum);

/* elementNum * 16 n */
FAST_FSS_API int FastFss_dpfGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t elementSize,
                                             size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
