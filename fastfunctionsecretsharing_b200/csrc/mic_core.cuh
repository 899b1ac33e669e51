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

// Points of the DCF walks an element needs: intervals that touch (R_q + 1 = L_{q+1} mod 2^n
// for q < m - 1) need the m + 1 points x - 1 - L_0 .. x - 1 - L_{m-1}, x - 1 - (R_{m-1} + 1);
// if the last also touches the first (the intervals tile the ring) the m points alone; 0 if
// the intervals do not touch (two walks per interval then).
template <typename GE>
__device__ uint32_t mic_points(const GE *left, const GE *right, uint32_t m, uint32_t n)
{
    for (uint32_t q = 0; q + 1 < m; q++)
        if (mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(right + q) + 1), n) != mod_bits<GE>((uint64_t)__ldg(left + q + 1), n))
            return 0;
    const bool cyclic =
        mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(right + m - 1) + 1), n) == mod_bits<GE>((uint64_t)__ldg(left), n);
    return cyclic ? m : m + 1;
}

// One batch of touching-interval MIC elements [base, min(base + E, eEnd)), E = blockDim / P,
// by the whole CTA (every thread calls it, it holds two barriers): thread t walks point t % P
// of element base + t / P into shares[t]; then thread t writes interval q = t % m of element
// base + t / m from the points on either side of it (sp = point q, sq = point q + 1, wrapping
// to point 0 when the intervals tile the ring, P = m), for items i m + q in [kFirst, kLast).
template <typename GE>
__device__ __forceinline__ void mic_shared_batch(const AesLanes &A, uint64_t *shares, GE *out, const GE *maskedX,
                                                 const uint8_t *key, const GE *z, const uint8_t *seed, uint32_t party,
                                                 const GE *left, const GE *right, uint32_t m, uint32_t n, uint32_t bo,
                                                 size_t N, uint32_t P, size_t base, size_t eEnd,
                                                 unsigned long long kFirst, unsigned long long kLast)
{
    const uint32_t E = blockDim.x / P, t = threadIdx.x;
    if (t < E * P)
    {
        const size_t i = base + t / P;
        if (i < eEnd)
        {
            const uint32_t p = t % P;
            DcfKeyView<GE> K;
            K.set(key, n, 1, i, N);
            const uint64_t x  = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
            const uint64_t e  = p < m ? (uint64_t)__ldg(left + p) : (uint64_t)(GE)((uint64_t)__ldg(right + m - 1) + 1);
            const uint64_t pt = mod_bits<GE>((uint64_t)(GE)(x - 1 - mod_bits<GE>(e, n)), n);
            shares[t]         = dcf_eval_g1<GE>(A, K, seed + 16 * i, party, n, bo, pt);
        }
    }
    __syncthreads();
    if (t < E * m)
    {
        const size_t             i = base + t / m;
        const uint32_t           q = t % m;
        const unsigned long long k = (unsigned long long)i * m + q;
        if (i < eEnd && k >= kFirst && k < kLast)
        {
            const uint32_t e  = t / m;
            const uint64_t sp = shares[e * P + q], sq = shares[e * P + (q + 1 == P ? 0 : q + 1)];
            const uint64_t x  = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
            const uint64_t qP = mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(right + q) + 1), n);
            const uint64_t lp = mod_bits<GE>((uint64_t)__ldg(left + q), n);
            uint64_t       o  = sq - sp + (uint64_t)__ldg(z + k);
            if (party == 1) o += (uint64_t)((int64_t)(x > lp) - (int64_t)(x > qP));
            out[k] = (GE)o;
        }
    }
    __syncthreads();
}

} // namespace fss
