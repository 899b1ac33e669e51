// spline_core.cuh — one element's DCF-spline evaluation by a group of G lanes (G a power of two
// <= 32, all lanes of a warp call it together), shared by the spline kernel and the batched
// persistent kernel. Algorithm: src/impl/spline.h:186-253 of the reference.
//
// Lane lg of element i takes intervals q = lg, lg + G, ... . For interval q it walks the two
// DCF paths x - 1 - L_q and x - 1 - (R_q + 1) side by side, and reads only slot q's values out
// of each level's convert stream: the value bytes j0 ges .. (j0 + cnt) ges - 1 lie in at most
// three consecutive 16-byte blocks of the AES-CTR stream, which are encrypted under one key
// schedule and read with register masks (no dynamically indexed arrays). Each AES call carries
// the next level of both walks and the previous level's converts (independent work, so the
// rounds have 4 + 2 NB blocks in flight).
#pragma once

#include "dcf_core.cuh"

namespace fss {

constexpr int kSplineMaxC = 4; // coefficients reduced per pass

// Little-endian 64-bit words of a window of NB blocks held as big-endian words.
template <int NB>
__device__ __forceinline__ void window_words(const uint32_t W[NB][4], uint64_t D[2 * NB])
{
#pragma unroll
    for (int q = 0; q < 2 * NB; q++)
        D[q] = (uint64_t)bswap32(W[q >> 1][2 * (q & 1)]) | ((uint64_t)bswap32(W[q >> 1][2 * (q & 1) + 1]) << 32);
}

// Little-endian value of the `ges` (1..8) bytes at byte offset p of the window; p + ges <= 16 NB.
template <int NB>
__device__ __forceinline__ uint64_t window_value(const uint64_t D[2 * NB], uint32_t p, uint32_t ges)
{
    const uint32_t j = p >> 3, sh = 8u * (p & 7u);
    uint64_t       lo = 0, hi = 0;
    // masks rather than selects: a select chain over D is turned into a local-memory array
#pragma unroll
    for (int q = 0; q < 2 * NB; q++)
    {
        lo ^= D[q] & (0ull - (uint64_t)((uint32_t)q == j));
        hi ^= D[q] & (0ull - (uint64_t)((uint32_t)q == j + 1));
    }
    const uint64_t v = sh ? ((lo >> sh) | (hi << (64u - sh))) : lo;
    return ges >= 8 ? v : (v & ((1ull << (8u * ges)) - 1ull));
}

// Blocks of the convert stream needed for values j0 .. j0 + cnt - 1 of every interval, the
// same for all lanes: the maximum over the intervals' start offsets (period 16 in q).
__device__ __forceinline__ uint32_t spline_window_blocks(uint32_t m, uint32_t cn, uint32_t c0, uint32_t cnt,
                                                         uint32_t ges)
{
    uint32_t nb = 1;
    for (uint32_t q = 0; q < m && q < 16; q++)
    {
        const uint32_t off = ((q * cn + c0) * ges) & 15u;
        nb                 = max(nb, (off + cnt * ges + 15u) >> 4);
    }
    return nb;
}

// Counter blocks of the convert stream for the slot window (blocks ctr[0 .. NB)).
template <int NB>
__device__ __forceinline__ void slot_counters(uint32_t W[2][NB][4], const uint32_t ctr[NB])
{
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
#pragma unroll
        for (int b = 0; b < NB; b++)
        {
            W[k][b][0] = 0;
            W[k][b][1] = 0;
            W[k][b][2] = bswap32(ctr[b]);
            W[k][b][3] = 0;
        }
    }
}

// Adds the shares of values j0 .. j0 + cnt - 1 read out of the windows W[k] (the encrypted
// slot blocks of convert stream k, or for a stream that needs no AES its key block itself in
// W[k][0]) into acc[k][c], with the correction corr[j0 + c] where tc[k] is set.
template <typename GE>
__device__ __forceinline__ void load_corr(uint64_t cv[kSplineMaxC], const GE *corr, uint32_t j0, uint32_t cnt)
{
#pragma unroll
    for (int c = 0; c < kSplineMaxC; c++) cv[c] = ((uint32_t)c < cnt) ? (uint64_t)__ldg(corr + j0 + c) : 0;
}

// cv: the corrections corr[j0 + c], loaded by the caller ahead of the AES work (load_corr)
template <int NB>
__device__ __forceinline__ void slot_accumulate(const uint32_t W[2][NB][4], const uint32_t tc[2],
                                                const uint64_t cv[kSplineMaxC], uint32_t party, uint32_t ges,
                                                uint32_t off, uint32_t cnt, uint64_t acc[2][kSplineMaxC])
{
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
        uint64_t D[2 * NB];
        window_words<NB>(W[k], D);
#pragma unroll
        for (int c = 0; c < kSplineMaxC; c++)
        {
            if ((uint32_t)c < cnt)
            {
                const uint64_t val = window_value<NB>(D, off + (uint32_t)c * ges, ges) + (tc[k] ? cv[c] : 0);
                acc[k][c] += party ? (0 - val) : val;
            }
        }
    }
}

// Seeds and control bits of both walks after the node expansion st (children of s[k] along
// dir[k]); the value children go to v.
__device__ __forceinline__ void walk_advance(uint32_t s[2][4], uint32_t t[2], uint32_t v[2][4],
                                             uint32_t st[2][2][4], const uint32_t dir[2], const uint32_t cw[4],
                                             uint64_t tl, uint64_t tr, uint32_t lv)
{
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
        uint32_t       tn = (st[k][0][0] >> 24) & 1u;
        const uint32_t mk = 0u - t[k];
        st[k][0][0] &= ~kSeedTBit;
#pragma unroll
        for (int c = 0; c < 4; c++)
        {
            s[k][c] = st[k][0][c] ^ (cw[c] & mk);
            v[k][c] = st[k][1][c];
        }
        tn ^= (uint32_t)(((dir[k] ? tr : tl) >> lv) & 1u) & t[k];
        t[k] = tn;
    }
}

// Both DCF walks of one interval (points xa, xb), slot values j0 .. j0 + cnt - 1. The walk is
// software pipelined: one AES call expands level lv + 1 of both walks (2 keys x 2 blocks) and
// encrypts the slot blocks of level lv's value convert (2 keys x NB blocks), which do not
// depend on each other, so every round carries 2 (2 + NB) independent block rounds.
template <typename GE, int NB, bool AES>
__device__ __forceinline__ void spline_walk_pair(const AesLanes &A, const DcfKeyView<GE> &K, const uint8_t *seed,
                                                 uint32_t party, uint32_t n, uint32_t g, uint32_t ges, uint64_t xa,
                                                 uint64_t xb, uint32_t j0, uint32_t cnt, uint64_t acc[2][kSplineMaxC])
{
    const uint32_t start = j0 * ges;
    const uint32_t blo   = AES ? (start >> 4) : 0u;
    const uint32_t off   = start - 16u * blo;
    uint32_t       ctr[NB];
#pragma unroll
    for (int b = 0; b < NB; b++) ctr[b] = (16u * (blo + (uint32_t)b)) / ges;
    uint32_t s[2][4];
    load_block_be(seed, s[0]);
    s[0][0] &= ~kSeedTBit;
#pragma unroll
    for (int c = 0; c < 4; c++) s[1][c] = s[0][c];
    uint32_t t[2] = {party, party};

    // level 0 alone
    uint32_t v[2][4], tp[2] = {party, party};
    {
        uint32_t cw[4];
        load_block_be(K.sCW, cw);
        const uint32_t dir[2] = {(uint32_t)((xa >> (n - 1)) & 1u), (uint32_t)((xb >> (n - 1)) & 1u)};
        uint32_t       st[2][2][4];
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            prg_block(st[k][0], 2 * dir[k]);
            prg_block(st[k][1], 2 * dir[k] + 1);
        }
        aes_encrypt_keys<2, 2>(A, s, st);
        walk_advance(s, t, v, st, dir, cw, K.tl, K.tr, 0);
    }
#pragma unroll 1
    for (uint32_t lv = 0; lv + 1 < n; lv++)
    {
        // holds: v, tp = value child and parent control bit of level lv; s, t at level lv + 1
        const uint32_t l1 = lv + 1;
        uint32_t       cw[4];
        load_block_be(K.sCW + 16 * l1, cw);
        const uint32_t dir[2] = {(uint32_t)((xa >> (n - 1 - l1)) & 1u), (uint32_t)((xb >> (n - 1 - l1)) & 1u)};
        uint32_t       st[2][2][4], W[2][NB][4];
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            prg_block(st[k][0], 2 * dir[k]);
            prg_block(st[k][1], 2 * dir[k] + 1);
        }
        uint64_t cv[kSplineMaxC];
        load_corr<GE>(cv, K.vCW + (size_t)lv * g, j0, cnt); // consumed after the AES work
        if (AES)
        {
            slot_counters<NB>(W, ctr);
            aes_encrypt_groups<2, 2, 2, NB>(A, s, st, v, W);
        }
        else
        {
            aes_encrypt_keys<2, 2>(A, s, st);
#pragma unroll
            for (int k = 0; k < 2; k++)
            {
#pragma unroll
                for (int c = 0; c < 4; c++) W[k][0][c] = v[k][c];
            }
        }
        slot_accumulate<NB>(W, tp, cv, party, ges, off, cnt, acc);
        tp[0] = t[0], tp[1] = t[1];
        walk_advance(s, t, v, st, dir, cw, K.tl, K.tr, l1);
    }
    // level n - 1's convert and the leaf convert (keyed by the final seeds) together
    uint32_t W[2][NB][4], WL[2][NB][4];
    uint64_t cv[kSplineMaxC], cl[kSplineMaxC];
    load_corr<GE>(cv, K.vCW + (size_t)(n - 1) * g, j0, cnt);
    load_corr<GE>(cl, K.last, j0, cnt);
    if (AES)
    {
        slot_counters<NB>(W, ctr);
        slot_counters<NB>(WL, ctr);
        aes_encrypt_groups<2, NB, 2, NB>(A, v, W, s, WL);
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) W[k][0][c] = v[k][c], WL[k][0][c] = s[k][c];
        }
    }
    slot_accumulate<NB>(W, tp, cv, party, ges, off, cnt, acc);
    slot_accumulate<NB>(WL, t, cl, party, ges, off, cnt, acc);
}

// As slot_accumulate for two windows of ONE convert stream: window w is blocks
// [w NB, w NB + NB) of W (a stream that needs no AES: its key block W[0] for both), read at byte
// offset off[w], into acc[w][c], with the corrections cv[w][c] where tc is set.
template <int NB, bool AES>
__device__ __forceinline__ void slot_accumulate2(const uint32_t W[][4], uint32_t tc, const uint64_t cv[2][kSplineMaxC],
                                                 uint32_t party, uint32_t ges, const uint32_t off[2], uint32_t cnt,
                                                 uint64_t acc[2][kSplineMaxC])
{
#pragma unroll
    for (int w = 0; w < 2; w++)
    {
        uint64_t D[2 * NB];
        window_words<NB>(W + (AES ? w * NB : 0), D);
#pragma unroll
        for (int c = 0; c < kSplineMaxC; c++)
        {
            if ((uint32_t)c < cnt)
            {
                const uint64_t val = window_value<NB>(D, off[w] + (uint32_t)c * ges, ges) + (tc ? cv[w][c] : 0);
                acc[w][c] += party ? (0 - val) : val;
            }
        }
    }
}

// When the intervals tile the ring (R_{q-1} + 1 = L_q for every q, cyclically), the left
// endpoint point x - 1 - L_q of interval q is also the right endpoint point of interval q - 1,
// so one DCF walk serves both: it reads slot q (window 0, into acc[0]) and slot q - 1
// (window 1, into acc[1]) of every level's convert stream, both under the one key schedule of
// that stream. Software pipelined like spline_walk_pair: each AES call carries the next level
// (1 key x 2 blocks) and the previous level's convert (1 key x 2 NB blocks).
template <typename GE, int NB, bool AES>
__device__ __forceinline__ void spline_walk_shared(const AesLanes &A, const DcfKeyView<GE> &K, const uint8_t *seed,
                                                   uint32_t party, uint32_t n, uint32_t g, uint32_t ges, uint64_t xp,
                                                   uint32_t j0a, uint32_t j0b, uint32_t cnt,
                                                   uint64_t acc[2][kSplineMaxC])
{
    const uint32_t j0[2] = {j0a, j0b};
    uint32_t       off[2], ctr[2][NB];
#pragma unroll
    for (int w = 0; w < 2; w++)
    {
        const uint32_t start = j0[w] * ges;
        const uint32_t blo   = AES ? (start >> 4) : 0u;
        off[w]               = start - 16u * blo;
#pragma unroll
        for (int b = 0; b < NB; b++) ctr[w][b] = (16u * (blo + (uint32_t)b)) / ges;
    }
    constexpr int WB = AES ? 2 * NB : 1; // blocks per convert
    uint32_t      s[1][4];
    load_block_be(seed, s[0]);
    s[0][0] &= ~kSeedTBit;
    uint32_t t = party, tp = party, v[1][4];
    auto advance = [&](uint32_t st[1][2][4], uint32_t dir, const uint32_t cw[4], uint32_t lv) {
        uint32_t       tn = (st[0][0][0] >> 24) & 1u;
        const uint32_t mk = 0u - t;
        st[0][0][0] &= ~kSeedTBit;
#pragma unroll
        for (int c = 0; c < 4; c++)
        {
            s[0][c] = st[0][0][c] ^ (cw[c] & mk);
            v[0][c] = st[0][1][c];
        }
        tn ^= (uint32_t)(((dir ? K.tr : K.tl) >> lv) & 1u) & t;
        t = tn;
    };
    auto counters = [&](uint32_t W[WB][4]) {
#pragma unroll
        for (int w = 0; w < 2; w++)
        {
#pragma unroll
            for (int b = 0; b < NB; b++)
            {
                W[w * NB + b][0] = 0;
                W[w * NB + b][1] = 0;
                W[w * NB + b][2] = bswap32(ctr[w][b]);
                W[w * NB + b][3] = 0;
            }
        }
    };
    {
        uint32_t cw[4];
        load_block_be(K.sCW, cw);
        const uint32_t dir = (uint32_t)((xp >> (n - 1)) & 1u);
        uint32_t       st[1][2][4];
        prg_block(st[0][0], 2 * dir);
        prg_block(st[0][1], 2 * dir + 1);
        aes_encrypt_keys<1, 2>(A, s, st);
        advance(st, dir, cw, 0);
    }
#pragma unroll 1
    for (uint32_t lv = 0; lv + 1 < n; lv++)
    {
        const uint32_t l1 = lv + 1;
        uint32_t       cw[4];
        load_block_be(K.sCW + 16 * l1, cw);
        const uint32_t dir = (uint32_t)((xp >> (n - 1 - l1)) & 1u);
        uint32_t       st[1][2][4], W[1][WB][4];
        prg_block(st[0][0], 2 * dir);
        prg_block(st[0][1], 2 * dir + 1);
        uint64_t cv[2][kSplineMaxC];
        load_corr<GE>(cv[0], K.vCW + (size_t)lv * g, j0a, cnt); // consumed after the AES work
        load_corr<GE>(cv[1], K.vCW + (size_t)lv * g, j0b, cnt);
        if (AES)
        {
            counters(W[0]);
            aes_encrypt_groups<1, 2, 1, WB>(A, s, st, v, W);
        }
        else
        {
            aes_encrypt_keys<1, 2>(A, s, st);
#pragma unroll
            for (int c = 0; c < 4; c++) W[0][0][c] = v[0][c];
        }
        slot_accumulate2<NB, AES>(W[0], tp, cv, party, ges, off, cnt, acc);
        tp = t;
        advance(st, dir, cw, l1);
    }
    // level n - 1's convert and the leaf convert (keyed by the final seed) together
    uint32_t W[2][WB][4];
    uint64_t cv[2][kSplineMaxC], cl[2][kSplineMaxC];
    load_corr<GE>(cv[0], K.vCW + (size_t)(n - 1) * g, j0a, cnt);
    load_corr<GE>(cv[1], K.vCW + (size_t)(n - 1) * g, j0b, cnt);
    load_corr<GE>(cl[0], K.last, j0a, cnt);
    load_corr<GE>(cl[1], K.last, j0b, cnt);
    if (AES)
    {
        counters(W[0]);
        counters(W[1]);
        const uint32_t keys[2][4] = {{v[0][0], v[0][1], v[0][2], v[0][3]}, {s[0][0], s[0][1], s[0][2], s[0][3]}};
        aes_encrypt_keys<2, WB>(A, keys, W);
    }
    else
    {
#pragma unroll
        for (int c = 0; c < 4; c++) W[0][0][c] = v[0][c], W[1][0][c] = s[0][c];
    }
    slot_accumulate2<NB, AES>(W[0], tp, cv, party, ges, off, cnt, acc);
    slot_accumulate2<NB, AES>(W[1], t, cl, party, ges, off, cnt, acc);
}

// The group sums w_c += cx beta_qc - s_qc + s'_qc + e_qc are reduced with shuffles and lane 0
// writes sum_c w_c x^c mod 2^bitWidthOut.
template <typename GE>
__device__ __forceinline__ void spline_eval_group(const AesLanes &A, GE *out, const GE *maskedX, const uint8_t *key,
                                                  const GE *sharedE, const GE *sharedBeta, const uint8_t *seed,
                                                  uint32_t party, const GE *left, const GE *right, uint32_t m,
                                                  uint32_t d, uint32_t n, uint32_t bo, size_t N, uint32_t G, size_t i,
                                                  uint32_t lg, bool active)
{
    const uint32_t cn = d + 1, g = m * cn;
    const uint32_t ges = (bo + 7) / 8;
    const bool     aes = (uint64_t)ges * g > 16; // convert keyed stream (src/impl/dcf.h:69-137)
    DcfKeyView<GE> K;
    uint64_t       x = 0;
    if (active)
    {
        K.set(key, n, g, i, N);
        x = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
    }
    // intervals that tile the ring cyclically share endpoint walks (spline_walk_shared);
    // the same answer for every lane of the group
    bool contig = true;
    for (uint32_t q = 0; q < m && contig; q++)
    {
        const uint64_t Lq    = mod_bits<GE>((uint64_t)__ldg(left + q), n);
        const uint64_t Rprev = mod_bits<GE>((uint64_t)__ldg(right + (q == 0 ? m - 1 : q - 1)), n);
        contig               = mod_bits<GE>((uint64_t)(GE)(Rprev + 1), n) == Lq;
    }
    uint64_t result = 0, xpow = 1;
    for (uint32_t c0 = 0; c0 < cn; c0 += kSplineMaxC)
    {
        const uint32_t cnt = min((uint32_t)kSplineMaxC, cn - c0);
        const uint32_t nb  = aes ? spline_window_blocks(m, cn, c0, cnt, ges) : 1u;
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
                const uint64_t xa = mod_bits<GE>((uint64_t)(GE)(x - 1 - L), n);
                const uint64_t xb = mod_bits<GE>((uint64_t)(GE)(x - 1 - Rp), n);
                const uint32_t j0 = q * cn + c0;
                uint64_t       w[2][kSplineMaxC];
#pragma unroll
                for (int k = 0; k < kSplineMaxC; k++) w[0][k] = 0, w[1][k] = 0;
                const uint8_t *sd = seed + 16 * i;
                if (contig)
                {
                    // w[0] = slot q at x - 1 - L_q (this interval's left endpoint); w[1] = slot
                    // q - 1 at the same point, the right endpoint of interval q - 1. Their sum
                    // over all q equals the per-interval sum of the pair walks.
                    const uint32_t jb = (q == 0 ? m - 1 : q - 1) * cn + c0;
                    if (!aes)
                        spline_walk_shared<GE, 1, false>(A, K, sd, party, n, g, ges, xa, j0, jb, cnt, w);
                    else if (nb == 1)
                        spline_walk_shared<GE, 1, true>(A, K, sd, party, n, g, ges, xa, j0, jb, cnt, w);
                    else if (nb == 2)
                        spline_walk_shared<GE, 2, true>(A, K, sd, party, n, g, ges, xa, j0, jb, cnt, w);
                    else
                        spline_walk_shared<GE, 3, true>(A, K, sd, party, n, g, ges, xa, j0, jb, cnt, w);
                }
                else if (!aes)
                    spline_walk_pair<GE, 1, false>(A, K, sd, party, n, g, ges, xa, xb, j0, cnt, w);
                else if (nb == 1)
                    spline_walk_pair<GE, 1, true>(A, K, sd, party, n, g, ges, xa, xb, j0, cnt, w);
                else if (nb == 2)
                    spline_walk_pair<GE, 2, true>(A, K, sd, party, n, g, ges, xa, xb, j0, cnt, w);
                else
                    spline_walk_pair<GE, 3, true>(A, K, sd, party, n, g, ges, xa, xb, j0, cnt, w);
                const uint64_t cx = (uint64_t)((int64_t)(x > L) - (int64_t)(x > Rp));
#pragma unroll
                for (int k = 0; k < kSplineMaxC; k++)
                {
                    if ((uint32_t)k < cnt)
                    {
                        const size_t   o = i * g + q * cn + c0 + k;
                        const uint64_t b = (uint64_t)__ldg(sharedBeta + o);
                        acc[k] += cx * b - w[0][k] + w[1][k] + (uint64_t)__ldg(sharedE + o);
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
