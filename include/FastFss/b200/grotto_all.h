/* Full-domain Grotto evaluation (extension of this library; the reference evaluates one
 * point per call, src/impl/grotto.h:207-391, and has no full-domain entry point).
 *
 * For every key i and every x in [0, 2^n) these write one bit per x, packed little-endian
 * (bit x of row i is bit x % 8 of byte i * 2^n / 8 + x / 8):
 *   FastFss_cuda_grottoEqEvalAll: the party's share of [x == alpha_i], i.e. exactly
 *       grottoEqEval(key_i, x) of the reference;
 *   FastFss_cuda_grottoLeEvalAll: the party's share of [x <= alpha_i], i.e. exactly
 *       grottoEval(key_i, x, equalBound = true) of the reference (prefix parity rule).
 * outDataSize must be elementNum * 2^n / 8 bytes and out 8-byte aligned; 6 <= n <= 40.
 * Keys, seeds and validation conventions as in <FastFss/cuda/grotto.h>. */
#ifndef FAST_FSS_B200_GROTTO_ALL_H
#define FAST_FSS_B200_GROTTO_ALL_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#define FAST_FSS_GROTTO_ALL_MAX_BITWIDTH 40

#ifdef __cplusplus
extern "C" {
#endif

FAST_FSS_API int FastFss_cuda_grottoEqEvalAll(void *outBits, size_t outBitsDataSize, const void *key,
                                              size_t keyDataSize, const void *seed, size_t seedDataSize, int partyId,
                                              size_t bitWidthIn, size_t elementSize, size_t elementNum,
                                              void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_grottoLeEvalAll(void *outBits, size_t outBitsDataSize, const void *key,
                                              size_t keyDataSize, const void *seed, size_t seedDataSize, int partyId,
                                              size_t bitWidthIn, size_t elementSize, size_t elementNum,
                                              void *cudaStreamPtr);

/* Interval lookup table from full-domain comparison rows (no counterpart in the reference;
 * BASELINE config 3's prefix-parity path). leRows is the output of FastFss_cuda_grottoLeEvalAll
 * for the same keys, seeds and party; the shares written are exactly those of
 * FastFss_cuda_grottoIntervalLutEval on the same inputs: for interval q the endpoint bits
 * sp = row[(x - (L_q - 1)) mod 2^n], sq = row[(x - R_q) mod 2^n] replace the two tree walks.
 * One warp per element; E is a ballot population count per 32 intervals, T_j a shuffle sum. */
FAST_FSS_API int FastFss_cuda_grottoIntervalLutEvalFromRows(
    void *sharedOutE, size_t sharedOutEDataSize, void *sharedOutT, size_t sharedOutTDataSize, const void *maskedX,
    size_t maskedXDataSize, const void *leRows, size_t leRowsDataSize, int partyId, const void *leftEndpoints,
    size_t leftEndpointsDataSize, const void *rightEndpoints, size_t rightEndpointsDataSize, const void *lookUpTable,
    size_t lookUpTableDataSize, size_t bitWidthIn, size_t elementSize, size_t elementNum, void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
