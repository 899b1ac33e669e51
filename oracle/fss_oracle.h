/*
 * fss_oracle.h — CPU restatement of the FastFss evaluation hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA library is compared
 * against; nothing in the product links it. Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg load it.
 *
 * Every function restates one reference routine (cited per function in the .c file) in
 * plain C. Ring elements of elementSize es in {1,2,4,8} are held in uint64_t and reduced
 * modulo 2^(8*es) on every store, which equals the reference's uintN_t arithmetic.
 * Argument order follows the reference's FastFss_cpu_* entry points with the data-size
 * arguments dropped (the oracle validates nothing: callers pass consistent buffers).
 */
#ifndef FSS_ORACLE_H
#define FSS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void oracle_aes128_encrypt(const void *key16, const void *in16, void *out16);

/* AES-128-CTR stream (src/cpu/prng.cpp:20-76); counter16 is advanced in place. */
void oracle_prng_gen(const void *seed16, void *counter16, void *dst, size_t bytesNum);

void oracle_dcfKeyGen(void *key, const void *alpha, const void *beta, const void *seed0, const void *seed1,
                      size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                      size_t elementNum);
void oracle_dcfEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                    size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum);

void oracle_dpfKeyGen(void *key, const void *alpha, const void *beta, const void *seed0, const void *seed1,
                      size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                      size_t elementNum);
void oracle_dpfEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                    size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum);
void oracle_dpfEvalAll(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                       size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                       size_t elementNum);
void oracle_dpfEvalMulti(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                         const void *point, size_t pointNum, size_t bitWidthIn, size_t bitWidthOut,
                         size_t groupSize, size_t elementSize, size_t elementNum);

void oracle_grottoKeyGen(void *key, const void *alpha, const void *seed0, const void *seed1, size_t bitWidthIn,
                         size_t elementSize, size_t elementNum);
void oracle_grottoEqEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                         size_t bitWidthIn, size_t elementSize, size_t elementNum);
void oracle_grottoEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int equalBound,
                       int partyId, size_t bitWidthIn, size_t elementSize, size_t elementNum);
void oracle_grottoMICEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                          const void *leftEndpoints, const void *rightEndpoints, size_t intervalNum,
                          size_t bitWidthIn, size_t elementSize, size_t elementNum);
void oracle_grottoIntervalLutEval(void *sharedOutE, void *sharedOutT, const void *maskedX, const void *key,
                                  const void *seed, int partyId, const void *leftEndpoints,
                                  const void *rightEndpoints, const void *lookUpTable, size_t lutNum,
                                  size_t intervalNum, size_t bitWidthIn, size_t elementSize, size_t elementNum);
/* Full domain: bit x of key i's 2^n-bit row = grottoEqEval(key i, x) (bit-packed, LSB first). */
void oracle_grottoEqEvalAll(void *outBits, const void *key, const void *seed, int partyId, size_t bitWidthIn,
                            size_t elementSize, size_t elementNum);
/* Full domain: bit x of key i's 2^n-bit row = grottoEval(key i, x, equalBound=1). */
void oracle_grottoLeEvalAll(void *outBits, const void *key, const void *seed, int partyId, size_t bitWidthIn,
                            size_t elementSize, size_t elementNum);

void oracle_dcfMICKeyGen(void *key, void *z, const void *alpha, const void *seed0, const void *seed1,
                         const void *leftEndpoints, const void *rightEndpoints, size_t intervalNum,
                         size_t bitWidthIn, size_t bitWidthOut, size_t elementSize, size_t elementNum);
void oracle_dcfMICEval(void *sharedOut, const void *maskedX, const void *key, const void *sharedZ,
                       const void *seed, int partyId, const void *leftEndpoints, const void *rightEndpoints,
                       size_t intervalNum, size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                       size_t elementNum);

void oracle_dcfSplineKeyGen(void *key, void *e, void *beta, const void *alpha, const void *seed0,
                            const void *seed1, const void *coefficients, size_t degree, const void *leftEndpoints,
                            const void *rightEndpoints, size_t intervalNum, size_t bitWidthIn, size_t bitWidthOut,
                            size_t elementSize, size_t elementNum);
void oracle_dcfSplineEval(void *sharedOut, const void *maskedX, const void *key, const void *sharedE,
                          const void *sharedBeta, const void *seed, int partyId, const void *leftEndpoints,
                          const void *rightEndpoints, size_t intervalNum, size_t degree, size_t bitWidthIn,
                          size_t bitWidthOut, size_t elementSize, size_t elementNum);

void oracle_otttKeyGen(void *key, const void *alpha, size_t bitWidthIn, size_t elementSize, size_t elementNum);
void oracle_otttLutEval(void *sharedOutE, void *sharedOutT, const void *maskedX, const void *key, int partyId,
                        const void *lookUpTable, size_t lutNum, size_t bitWidthIn, size_t elementSize,
                        size_t elementNum);

/* Threads used by the element loops (OpenMP); 0 = library default. */
void oracle_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
