// mic_core.cuh — one (element, interval) item of DCF-based MIC evaluation, shared by the MIC
// kernel and the batched persistent kernel (src/impl/mic.h:43-109 of the reference).
#pragma once

#include "dcf_core.cuh"

namespace fss {

// Share of interval q = w % m for element i = w / m:
//   DCF(x - 1 - (R_q + 1)) - DCF(x - 1 - L_q) + z[w] (+ [x > L_q] - [x > R_q + 1] for party 1).
template <typename GE>
__device__ __forceinline__ GE mic_eval_item(const AesLanes &A, const GE *maskedX, const uint8_t *key, const GE *z,
                                            const uint8_t *seed, uint32_t party, const GE *left, const GE *right,
                                            uint32_t m, uint32_t n, uint32_t bo, size_t N, size_t w)
{
    const size_t   i = w / m, q = w % m;
    DcfKeyView<GE> K;
    K.set(key, n, 1, i, N);
    const uint64_t x  = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
    const uint64_t L  = (uint64_t)__ldg(left + q), R = (uint64_t)__ldg(right + q);
    const uint64_t qP = mod_bits<GE>((uint64_t)(GE)(R + 1), n);
    const uint64_t xP = mod_bits<GE>((uint64_t)(GE)(x - 1 - L), n);
    const uint64_t xQ = mod_bits<GE>((uint64_t)(GE)(x - 1 - qP), n);
    const uint64_t p  = mod_bits<GE>(L, n);
    uint64_t       sp, sq;
    dcf_eval_g1_two<GE>(A, K, seed + 16 * i, party, n, bo, xP, xQ, sp, sq);
    uint64_t       o  = sq - sp + (uint64_t)__ldg(z + w);
    if (party == 1) o += (uint64_t)((int64_t)(x > p) - (int64_t)(x > qP));
    return (GE)o;
}

} // namespace fss
