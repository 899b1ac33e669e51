// grotto_core.cuh — per-element Grotto routines shared by the Grotto kernels and the batched
// persistent kernel. Algorithm: src/impl/grotto.h:207-391,414-423 of the reference; key layout
// grottoKeySetPtr (src/impl/grotto.h:53-79).
#pragma once

#include "fss_device.cuh"

namespace fss {

template <typename GE>
struct GrottoKeyView
{
    const uint8_t *sCW;
    uint64_t       last, tl, tr;

    __device__ __forceinline__ void set(const uint8_t *key, uint32_t n, size_t i, size_t N)
    {
        const size_t a = N * 16 * (n - 6);
        sCW            = key + i * 16 * (n - 6);
        last           = __ldg(reinterpret_cast<const unsigned long long *>(key + a) + i);
        const GE *t    = reinterpret_cast<const GE *>(key + a + N * 8) + 2 * i;
        tl             = (uint64_t)__ldg(t);
        tr             = (uint64_t)__ldg(t + 1);
    }
};

// Bytes 8..15 of a block (big-endian words 2, 3) as the little-endian uint64 seed[1].
__device__ __forceinline__ uint64_t hi_u64(const uint32_t w[4])
{
    return (uint64_t)bswap32(w[2]) | ((uint64_t)bswap32(w[3]) << 32);
}

// Expands child `dir` of (s, t) at level lv; returns the child's control bit.
__device__ __forceinline__ uint32_t grotto_step(const AesLanes &A, uint32_t s[4], uint32_t t, uint32_t dir,
                                                const uint8_t *cwp, uint64_t tl, uint64_t tr, uint32_t lv)
{
    uint32_t cw[4];
    load_block_be(cwp, cw);
    uint32_t st[1][4];
    prg_block(st[0], dir);
    aes_encrypt<1>(A, s, st);
    uint32_t       tn = (st[0][0] >> 24) & 1u;
    const uint32_t m  = 0u - t;
    st[0][0] &= ~kSeedTBit;
#pragma unroll
    for (int c = 0; c < 4; c++) s[c] = st[0][c] ^ (cw[c] & m);
    tn ^= (uint32_t)(((dir ? tr : tl) >> lv) & 1u) & t;
    return tn;
}

// Root-to-leaf walk along x (x < 2^n). Returns the leaf word u; *parity gets the right-turn
// parity. With equalBound the walk stops as soon as the remaining bits of x are zero
// (*early = 1, u undefined).
template <typename GE>
__device__ __forceinline__ uint64_t grotto_walk(const AesLanes &A, const GrottoKeyView<GE> &K, const uint8_t *seed,
                                                uint32_t party, uint32_t n, uint64_t x, bool equalBound,
                                                uint32_t *parity, bool *early)
{
    uint32_t s[4];
    load_block_be(seed, s);
    s[0] &= ~kSeedTBit;
    uint32_t t = party, par = 0;
    *early     = false;
#pragma unroll 1
    for (uint32_t lv = 0; lv + 6 < n; lv++)
    {
        if (equalBound && mod_bits<GE>(x, n - lv) == 0)
        {
            *early  = true;
            *parity = par;
            return 0;
        }
        const uint32_t dir = (uint32_t)((x >> (n - 1 - lv)) & 1u);
        const uint32_t tn  = grotto_step(A, s, t, dir, K.sCW + 16 * lv, K.tl, K.tr, lv);
        par ^= dir & (t ^ tn);
        t = tn;
    }
    *parity = par;
    const uint64_t u = hi_u64(s);
    return t ? (u ^ K.last) : u;
}

// grottoEval share (src/impl/grotto.h:284-391).
template <typename GE>
__device__ __forceinline__ uint32_t grotto_cmp(const AesLanes &A, const GrottoKeyView<GE> &K, const uint8_t *seed,
                                               uint32_t party, uint32_t n, uint64_t x, bool equalBound)
{
    uint32_t       par;
    bool           early;
    const uint64_t u = grotto_walk<GE>(A, K, seed, party, n, x, equalBound, &par, &early);
    if (early) return par ^ party;
    const uint32_t pre = (uint32_t)(x & 63u);
    uint64_t       mask;
    if (equalBound)
        mask = pre ? (~0ull >> (64 - pre)) : 0ull;
    else
        mask = ~0ull >> (63 - pre);
    return par ^ (uint32_t)(__popcll(u & mask) & 1) ^ party;
}

// grotto_cmp at two points x[0], x[1] under one key, both walks in the same AES calls (a walk
// that stops early keeps its state while the other goes on).
template <typename GE>
__device__ __forceinline__ void grotto_cmp2(const AesLanes &A, const GrottoKeyView<GE> &K, const uint8_t *seed,
                                            uint32_t party, uint32_t n, const uint64_t x[2], bool equalBound,
                                            uint32_t share[2])
{
    uint32_t s[2][4];
    load_block_be(seed, s[0]);
    s[0][0] &= ~kSeedTBit;
#pragma unroll
    for (int c = 0; c < 4; c++) s[1][c] = s[0][c];
    uint32_t t[2] = {party, party}, par[2] = {0, 0};
    bool     early[2] = {false, false};
#pragma unroll 1
    for (uint32_t lv = 0; lv + 6 < n; lv++)
    {
#pragma unroll
        for (int k = 0; k < 2; k++)
            if (equalBound && !early[k] && mod_bits<GE>(x[k], n - lv) == 0) early[k] = true;
        if (early[0] && early[1]) break;
        uint32_t cw[4];
        load_block_be(K.sCW + 16 * lv, cw);
        uint32_t dir[2], st[2][1][4];
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            dir[k] = (uint32_t)((x[k] >> (n - 1 - lv)) & 1u);
            prg_block(st[k][0], dir[k]);
        }
        aes_encrypt_keys<2, 1>(A, s, st);
#pragma unroll
        for (int k = 0; k < 2; k++)
        {
            if (early[k]) continue;
            uint32_t       tn = (st[k][0][0] >> 24) & 1u;
            const uint32_t m  = 0u - t[k];
            st[k][0][0] &= ~kSeedTBit;
#pragma unroll
            for (int c = 0; c < 4; c++) s[k][c] = st[k][0][c] ^ (cw[c] & m);
            tn ^= (uint32_t)(((dir[k] ? K.tr : K.tl) >> lv) & 1u) & t[k];
            par[k] ^= dir[k] & (t[k] ^ tn);
            t[k] = tn;
        }
    }
#pragma unroll
    for (int k = 0; k < 2; k++)
    {
        if (early[k])
        {
            share[k] = par[k] ^ party;
            continue;
        }
        const uint64_t u0   = hi_u64(s[k]);
        const uint64_t u    = t[k] ? (u0 ^ K.last) : u0;
        const uint32_t pre  = (uint32_t)(x[k] & 63u);
        const uint64_t mask = equalBound ? (pre ? (~0ull >> (64 - pre)) : 0ull) : (~0ull >> (63 - pre));
        share[k]            = par[k] ^ (uint32_t)(__popcll(u & mask) & 1) ^ party;
    }
}

// Interval endpoints shared by MIC and the LUT (src/impl/grotto.h:414-423,499-517):
// sp = share of [x - (L - 1) <= alpha'], sq = share of [x - R <= alpha'], bit = sp ^ sq ^
// party [xQ >= xP] (the reference reuses sq of interval i-1 as sp of interval i when the
// intervals touch; that point is the same, so every interval is evaluated on its own here).
template <typename GE>
__device__ __forceinline__ uint32_t grotto_interval_bit(const AesLanes &A, const GrottoKeyView<GE> &K,
                                                        const uint8_t *seed, uint32_t party, uint32_t n, uint64_t mx,
                                                        uint64_t L, uint64_t R)
{
    const uint64_t xP = mod_bits<GE>((uint64_t)(GE)(mx - (uint64_t)(GE)(L - 1)), n);
    const uint64_t xQ = mod_bits<GE>((uint64_t)(GE)(mx - R), n);
    const uint64_t xs[2] = {xP, xQ};
    uint32_t       sh[2];
    grotto_cmp2<GE>(A, K, seed, party, n, xs, true, sh);
    return (sh[0] ^ sh[1] ^ ((xQ >= xP) ? party : 0u)) & 1u;
}

} // namespace fss
