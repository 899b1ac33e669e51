// spline_core.cuh — one element's DCF-spline evaluation by a group of G lanes (G a power of two
// <= 32, all lanes of a warp call it together), shared by the spline kernel and the batched
// persistent kernel. Algorithm: src/impl/spline.h:186-253 of the reference.
#pragma once

#include "dcf_core.cuh"

namespace fss {

constexpr int kSplineMaxC = 4; // coefficients reduced per pass

// Lane lg of element i walks intervals q = lg, lg + G, ...: both DCF paths of interval q,
// reading only slot q's d + 1 values out of each level's convert stream, and accumulates
// w_c += cx beta_qc - s_qc + s'_qc + e_qc. The group sums are reduced with shuffles and
// lane 0 writes sum_c w_c x^c mod 2^bitWidthOut.
template <typename GE>
__device__ __forceinline__ void spline_eval_group(const AesLanes &A, GE *out, const GE *maskedX, const uint8_t *key,
                                                  const GE *sharedE, const GE *sharedBeta, const uint8_t *seed,
                                                  uint32_t party, const GE *left, const GE *right, uint32_t m,
                                                  uint32_t d, uint32_t n, uint32_t bo, size_t N, uint32_t G, size_t i,
                                                  uint32_t lg, bool active)
{
    const uint32_t cn = d + 1, g = m * cn;
    DcfKeyView<GE> K;
    uint64_t       x = 0;
    if (active)
    {
        K.set(key, n, g, i, N);
        x = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
    }
    uint64_t result = 0, xpow = 1;
    for (uint32_t c0 = 0; c0 < cn; c0 += kSplineMaxC)
    {
        const uint32_t cnt = min((uint32_t)kSplineMaxC, cn - c0);
        uint64_t       acc[kSplineMaxC];
#pragma unroll
        for (int k = 0; k < kSplineMaxC; k++) acc[k] = 0;
        if (active)
        {
            for (uint32_t q = lg; q < m; q += G)
            {
                const uint64_t L  = mod_bits<GE>((uint64_t)__ldg(left + q), n);
                const uint64_t R  = mod_bits<GE>((uint64_t)__ldg(right + q), n);
                const uint64_t Rp = mod_bits<GE>((uint64_t)(GE)(R + 1), n);
                uint64_t       sL[kSplineMaxC], sR[kSplineMaxC];
#pragma unroll
                for (int k = 0; k < kSplineMaxC; k++) sL[k] = 0, sR[k] = 0;
                dcf_eval_slice<GE, kSplineMaxC>(A, sL, K, seed + 16 * i, party, n, bo, g,
                                                mod_bits<GE>((uint64_t)(GE)(x - 1 - L), n), q * cn + c0, cnt);
                dcf_eval_slice<GE, kSplineMaxC>(A, sR, K, seed + 16 * i, party, n, bo, g,
                                                mod_bits<GE>((uint64_t)(GE)(x - 1 - Rp), n), q * cn + c0, cnt);
                const uint64_t cx = (uint64_t)((int64_t)(x > L) - (int64_t)(x > Rp));
#pragma unroll
                for (int k = 0; k < kSplineMaxC; k++)
                {
                    if ((uint32_t)k < cnt)
                    {
                        const size_t   o = i * g + q * cn + c0 + k;
                        const uint64_t b = (uint64_t)__ldg(sharedBeta + o);
                        acc[k] += cx * b - sL[k] + sR[k] + (uint64_t)__ldg(sharedE + o);
                    }
                }
            }
        }
        for (uint32_t off = G >> 1; off > 0; off >>= 1)
        {
#pragma unroll
            for (int k = 0; k < kSplineMaxC; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
        }
        // splineEvaluatePolynomial (src/impl/spline.h:119-135): sum of acc_c x^c
#pragma unroll
        for (int k = 0; k < kSplineMaxC; k++)
        {
            if ((uint32_t)k < cnt)
            {
                result += acc[k] * xpow;
                xpow *= x;
            }
        }
    }
    if (active && lg == 0) out[i] = (GE)mod_bits<GE>((uint64_t)(GE)result, bo);
}

} // namespace fss
