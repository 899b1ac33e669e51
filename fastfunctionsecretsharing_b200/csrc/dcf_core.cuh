// dcf_core.cuh — per-element DCF routines shared by the DCF, DCF-MIC and spline kernels.
//
// Algorithm: src/impl/dcf.h:187-491 of the reference. Key layout (dcfKeySetPtr,
// src/impl/dcf.h:139-167): region A sCW[N][n][16 B]; region B per element, stride
// es (n g + 2 + g): vCW[n][g], tLCW, tRCW, lastCW[g].
#pragma once

#include "fss_device.cuh"

namespace fss {

template <typename GE>
struct DcfKeyView
{
    const uint8_t *sCW;  // n x 16 B
    const GE      *vCW;  // n x g
    uint64_t       tl, tr;
    const GE      *last; // g

    __device__ __forceinline__ void set(const uint8_t *key, uint32_t n, uint32_t g, size_t i, size_t N)
    {
        const size_t bstr = sizeof(GE) * ((size_t)n * g + 2 + g);
        sCW               = key + i * 16 * n;
        vCW               = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        tl                = (uint64_t)__ldg(vCW + (size_t)n * g);
        tr                = (uint64_t)__ldg(vCW + (size_t)n * g + 1);
        last              = vCW + (size_t)n * g + 2;
    }
};

// One level for groupSize 1 of NK walks under the same key (correction words shared): expands
// the child on direction dir[k] of node (s[k], t[k]) — blocks 2 dir and 2 dir + 1 of G(s) — and
// applies the correction word cw[] (big-endian words, supplied by the caller) where t is set.
// The value child is produced only as far as its first VW words (the bytes a groupSize-1
// convert reads: ceil(bo / 8) <= 4 VW).
template <int NK, int VW>
__device__ __forceinline__ void dcf_step_g1_cw(const AesLanes &A, uint32_t s[NK][4], uint32_t t[NK],
                                               const uint32_t dir[NK], const uint32_t cw[4], uint64_t tl, uint64_t tr,
                                               uint32_t lv, uint32_t v[NK][VW])
{
    uint32_t sn[NK][4];
    aes_prg_pair<NK, VW>(A, s, dir, sn, v);
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
        uint32_t       tn = (sn[k][0] >> 24) & 1u;
        const uint32_t m  = 0u - t[k];
        sn[k][0] &= ~kSeedTBit;
#pragma unroll
        for (int c = 0; c < 4; c++) s[k][c] = sn[k][c] ^ (cw[c] & m);
        tn ^= (uint32_t)(((dir[k] ? tr : tl) >> lv) & 1u) & t[k];
        t[k] = tn;
    }
}

template <int NK, int VW>
__device__ __forceinline__ void dcf_step_g1(const AesLanes &A, uint32_t s[NK][4], uint32_t t[NK],
                                            const uint32_t dir[NK], const uint8_t *cwp, uint64_t tl, uint64_t tr,
                                            uint32_t lv, uint32_t v[NK][VW])
{
    uint32_t cw[4];
    load_block_be(cwp, cw);
    dcf_step_g1_cw<NK, VW>(A, s, t, dir, cw, tl, tr, lv, v);
}

// Little-endian value of the first `nbytes` (1 .. 4 VW) bytes of a block's first VW words.
template <int VW>
__device__ __forceinline__ uint64_t words_le_prefix(const uint32_t w[VW], int nbytes)
{
    const uint64_t v = (uint64_t)bswap32(w[0]) | (VW > 1 ? ((uint64_t)bswap32(w[VW > 1 ? 1 : 0]) << 32) : 0ull);
    return nbytes >= 8 ? v : (v & ((1ull << (8 * nbytes)) - 1ull));
}

// groupSize-1 shares of NK points x[k] under one key (the walks run side by side).
template <typename GE, int NK, int VW>
__device__ __forceinline__ void dcf_eval_g1_vw(const AesLanes &A, const DcfKeyView<GE> &K, const uint8_t *seed,
                                               uint32_t party, uint32_t n, uint32_t bo, const uint64_t x[NK],
                                               uint64_t acc[NK])
{
    const int ges = (int)((bo + 7) / 8);
    uint32_t  s[NK][4], t[NK];
    load_block_be(seed, s[0]);
    s[0][0] &= ~kSeedTBit;
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) s[k][c] = s[0][c];
        t[k]   = party;
        acc[k] = 0;
    }
#pragma unroll 1
    for (uint32_t lv = 0; lv < n; lv++)
    {
        uint32_t dir[NK], tp[NK], v[NK][VW];
#pragma unroll
        for (int k = 0; k < NK; k++) dir[k] = (uint32_t)((x[k] >> (n - 1 - lv)) & 1u), tp[k] = t[k];
        const uint64_t vcw = (uint64_t)__ldg(K.vCW + lv);
        dcf_step_g1<NK, VW>(A, s, t, dir, K.sCW + 16 * lv, K.tl, K.tr, lv, v);
#pragma unroll
        for (int k = 0; k < NK; k++)
        {
            const uint64_t val = words_le_prefix<VW>(v[k], ges) + (tp[k] ? vcw : 0);
            acc[k] += party ? (0 - val) : val;
        }
    }
    const uint64_t last = (uint64_t)__ldg(K.last);
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
        const uint64_t val = block_le_prefix(s[k], ges) + (t[k] ? last : 0);
        acc[k] += party ? (0 - val) : val;
    }
}

// groupSize 1 share (the convert is a plain read of the first ceil(bo/8) bytes).
template <typename GE>
__device__ __forceinline__ uint64_t dcf_eval_g1(const AesLanes &A, const DcfKeyView<GE> &K, const uint8_t *seed,
                                                uint32_t party, uint32_t n, uint32_t bo, uint64_t x)
{
    const uint64_t xs[1] = {x};
    uint64_t       acc[1];
    if (sizeof(GE) <= 4 || bo <= 32)
        dcf_eval_g1_vw<GE, 1, 1>(A, K, seed, party, n, bo, xs, acc);
    else
        dcf_eval_g1_vw<GE, 1, 2>(A, K, seed, party, n, bo, xs, acc);
    return acc[0];
}

// Shares at two points under one key, both walks in the same AES calls.
template <typename GE>
__device__ __forceinline__ void dcf_eval_g1_two(const AesLanes &A, const DcfKeyView<GE> &K, const uint8_t *seed,
                                                uint32_t party, uint32_t n, uint32_t bo, uint64_t xa, uint64_t xb,
                                                uint64_t &sa, uint64_t &sb)
{
    const uint64_t xs[2] = {xa, xb};
    uint64_t       acc[2];
    if (sizeof(GE) <= 4 || bo <= 32)
        dcf_eval_g1_vw<GE, 2, 1>(A, K, seed, party, n, bo, xs, acc);
    else
        dcf_eval_g1_vw<GE, 2, 2>(A, K, seed, party, n, bo, xs, acc);
    sa = acc[0];
    sb = acc[1];
}

// Key generation of one element (src/impl/dcf.h:187-368). beta == nullptr means beta = 1
// (first value; the reference reads only that one for groupSize 1). vAlpha accumulates in
// the element's lastCW slots, as in the reference.
template <typename GE>
__device__ __forceinline__ void dcf_keygen_element(const AesLanes &A, uint8_t *key, size_t N, size_t i,
                                                   uint64_t alpha, const GE *beta, const uint8_t *seed0,
                                                   const uint8_t *seed1, uint32_t n, uint32_t bo, uint32_t g)
{
    const size_t bstr = sizeof(GE) * ((size_t)n * g + 2 + g);
    uint8_t     *sCWp = key + i * 16 * n;
    GE          *vCW  = reinterpret_cast<GE *>(key + N * 16 * n + i * bstr);
    GE          *tLp  = vCW + (size_t)n * g;
    GE          *last = tLp + 2;
    for (uint32_t j = 0; j < g; j++) last[j] = 0;

    uint32_t s0[4], s1[4];
    load_block_be(seed0, s0);
    load_block_be(seed1, s1);
    s0[0] &= ~kSeedTBit;
    s1[0] &= ~kSeedTBit;
    uint32_t t0 = 0, t1 = 1;
    uint64_t tl = 0, tr = 0;
#pragma unroll 1
    for (uint32_t lv = 0; lv < n; lv++)
    {
        uint32_t G0[4][4], G1[4][4];
        // groupSize 1 with values of <= 4 (<= 8) bytes reads 1 (2) words of the value blocks
        const int vw = (g != 1) ? 4 : ((bo + 7) / 8 <= 4 ? 1 : 2);
        if (vw == 1)
        {
            aes_prg_quad<1>(A, s0, G0);
            aes_prg_quad<1>(A, s1, G1);
        }
        else if (vw == 2)
        {
            aes_prg_quad<2>(A, s0, G0);
            aes_prg_quad<2>(A, s1, G1);
        }
        else
        {
            aes_prg_quad<4>(A, s0, G0);
            aes_prg_quad<4>(A, s1, G1);
        }
        const uint32_t tL0 = (G0[0][0] >> 24) & 1u, tR0 = (G0[2][0] >> 24) & 1u;
        const uint32_t tL1 = (G1[0][0] >> 24) & 1u, tR1 = (G1[2][0] >> 24) & 1u;
        G0[0][0] &= ~kSeedTBit, G0[2][0] &= ~kSeedTBit, G1[0][0] &= ~kSeedTBit, G1[2][0] &= ~kSeedTBit;

        const uint32_t keep = (uint32_t)((alpha >> (n - 1 - lv)) & 1u);
        // keep = R (1): lose = L = blocks 0/1, keep = blocks 2/3; keep = L (0): the reverse.
        uint32_t sLose0[4], sLose1[4], vLose0[4], vLose1[4], sKeep0[4], sKeep1[4], vKeep0[4], vKeep1[4];
#pragma unroll
        for (int c = 0; c < 4; c++)
        {
            sLose0[c] = keep ? G0[0][c] : G0[2][c];
            vLose0[c] = keep ? G0[1][c] : G0[3][c];
            sKeep0[c] = keep ? G0[2][c] : G0[0][c];
            vKeep0[c] = keep ? G0[3][c] : G0[1][c];
            sLose1[c] = keep ? G1[0][c] : G1[2][c];
            vLose1[c] = keep ? G1[1][c] : G1[3][c];
            sKeep1[c] = keep ? G1[2][c] : G1[0][c];
            vKeep1[c] = keep ? G1[3][c] : G1[1][c];
        }
        uint32_t sCW[4];
#pragma unroll
        for (int c = 0; c < 4; c++) sCW[c] = sLose0[c] ^ sLose1[c];

        if (g == 1)
        {
            // groupSize 1: the convert is the first ceil(bo/8) bytes of the value block
            const int      ges = (int)((bo + 7) / 8);
            uint64_t       va  = (uint64_t)last[0];
            uint64_t       v   = block_le_prefix(vLose1, ges) - block_le_prefix(vLose0, ges) - va;
            if (t1) v = 0 - v;
            if (keep)
            {
                const uint64_t b = beta ? (uint64_t)beta[0] : 1u;
                v += t1 ? (0 - b) : b;
            }
            vCW[lv] = (GE)v;
            va      = va - block_le_prefix(vKeep1, ges) + block_le_prefix(vKeep0, ges) + (t1 ? (0 - v) : v);
            last[0] = (GE)va;
        }
        else
        {
            ConvertStream cL1, cL0, cK1, cK0;
            cL1.init(vLose1, g, bo);
            cL0.init(vLose0, g, bo);
            cK1.init(vKeep1, g, bo);
            cK0.init(vKeep0, g, bo);
            for (uint32_t j = 0; j < g; j++)
            {
                uint64_t va = (uint64_t)last[j];
                uint64_t v  = cL1.value(A, j) - cL0.value(A, j) - va;
                if (t1) v = 0 - v;
                if (keep)
                {
                    const uint64_t b = beta ? (uint64_t)beta[j] : (uint64_t)(j == 0);
                    v += t1 ? (0 - b) : b;
                }
                vCW[(size_t)lv * g + j] = (GE)v;
                va                      = va - cK1.value(A, j) + cK0.value(A, j) + (t1 ? (0 - v) : v);
                last[j]                 = (GE)va;
            }
        }

        store_block_be(sCWp + 16 * lv, sCW);
        const uint32_t tLCW = tL0 ^ tL1 ^ keep ^ 1u;
        const uint32_t tRCW = tR0 ^ tR1 ^ keep;
        tl |= (uint64_t)tLCW << lv;
        tr |= (uint64_t)tRCW << lv;
        const uint32_t m0 = 0u - t0, m1 = 0u - t1;
#pragma unroll
        for (int c = 0; c < 4; c++)
        {
            s0[c] = sKeep0[c] ^ (sCW[c] & m0);
            s1[c] = sKeep1[c] ^ (sCW[c] & m1);
        }
        const uint32_t tcw = keep ? tRCW : tLCW;
        t0                 = (keep ? tR0 : tL0) ^ (t0 & tcw);
        t1                 = (keep ? tR1 : tL1) ^ (t1 & tcw);
    }
    tLp[0] = (GE)tl;
    tLp[1] = (GE)tr;
    if (g == 1)
    {
        const int ges = (int)((bo + 7) / 8);
        uint64_t  v   = block_le_prefix(s1, ges) - block_le_prefix(s0, ges) - (uint64_t)last[0];
        if (t1) v = 0 - v;
        last[0] = (GE)v;
        return;
    }
    ConvertStream c1, c0;
    c1.init(s1, g, bo);
    c0.init(s0, g, bo);
    for (uint32_t j = 0; j < g; j++)
    {
        uint64_t v = c1.value(A, j) - c0.value(A, j) - (uint64_t)last[j];
        if (t1) v = 0 - v;
        last[j] = (GE)v;
    }
}

} // namespace fss
