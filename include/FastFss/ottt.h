/* Host-side one-hot truth-table key sizing. Replaces include/FastFss/ottt.h of the
 * reference: elementNum * 2^n / 8 bytes (src/impl/ottt.h:9-13). */
#ifndef FAST_FSS_OTTT_H
#define FAST_FSS_OTTT_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_otttGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementNum);

#ifdef __cplusplus
}
#endif

#endif
