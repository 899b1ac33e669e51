/* Diagnostics of this library (no counterpart in the reference).
 *
 * FastFss_b200_smemLookupProbe measures the sustained rate of conflict-free, byte-permute
 * addressed 32-bit shared-memory table lookups — the access the AES T-table rounds of every
 * FSS kernel are built from — so a benchmark can report kernel throughput as a fraction of
 * a measured peak. It launches one 512-thread CTA per SM; each thread issues 16 independent
 * lookups per iteration for `iterations` iterations and stores one word per thread into `sink`
 * (sinkBytes >= 4 * 512 * SM count). *lookups receives the total number of lookups issued.
 * Asynchronous on *(cudaStream_t *)cudaStreamPtr (cudaStreamPerThread when NULL). */
#ifndef FAST_FSS_B200_DIAG_H
#define FAST_FSS_B200_DIAG_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_b200_smemLookupProbe(void *sink, size_t sinkBytes, unsigned iterations,
                                              unsigned long long *lookups, void *cudaStreamPtr);

FAST_FSS_API int FastFss_b200_smCount(void);

/* Number of staging failures since the library was loaded on the current device: a kernel's
 * bounded wait for one of its own asynchronous shared-memory staging copies ran out, or a CTA
 * found its shared-memory window unfit for aligned stages (the groupSize-1 DCF evaluation
 * stages its correction words this way). Always 0 in normal operation; a nonzero count means
 * some shares of that launch were not written. Synchronous: waits for the device's earlier
 * work. */
FAST_FSS_API int FastFss_b200_stageTimeouts(unsigned int *count);

#ifdef __cplusplus
}
#endif

#endif
