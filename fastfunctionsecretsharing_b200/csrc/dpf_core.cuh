// dpf_core.cuh — per-element DPF evaluation shared by the DPF kernels and the batched
// persistent kernel. Algorithm: src/impl/dpf.h:290-380 of the reference; key layout
// dpfKeySetPtr (src/impl/dpf.h:130-156): region A sCW[N][n][16 B], region B per element
// tLCW, tRCW, lastCW[g]. The leaf convert is init(seed, bitWidthOut, groupSize), as the
// reference calls it (src/impl/dpf.h:375).
#pragma once

#include "fss_device.cuh"

namespace fss {

// One level along direction `dir`: the child block AES_s(LE64(2 dir) || LE64(2 dir + 1)),
// corrected by cw[] (big-endian words) when t is set; returns the child's control bit.
__device__ __forceinline__ uint32_t dpf_step(const AesLanes &A, uint32_t s[4], uint32_t t, uint32_t dir,
                                             const uint32_t cw[4], uint64_t tl, uint64_t tr, uint32_t lv)
{
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

// The g outputs of the leaf (seed s, control bit t): convert(s) + t lastCW, negated for party 1.
template <typename GE>
__device__ __forceinline__ void dpf_leaf(const AesLanes &A, GE *o, const uint32_t s[4], uint32_t t, const GE *kb,
                                         uint32_t party, uint32_t bo, uint32_t g)
{
    ConvertStream cv;
    cv.init(s, bo, g);
    for (uint32_t j = 0; j < g; j++)
    {
        const uint64_t v = cv.value(A, j) + (t ? (uint64_t)__ldg(kb + 2 + j) : 0);
        o[j]             = (GE)(party ? (0 - v) : v);
    }
}

// Walks one element's tree along x (already reduced mod 2^n) and writes the g outputs.
template <typename GE>
__device__ __forceinline__ void dpf_eval_point(const AesLanes &A, GE *o, const uint8_t *sCWp, const GE *kb,
                                               const uint8_t *seed, uint32_t party, uint32_t n, uint32_t bo,
                                               uint32_t g, uint64_t x, uint64_t tl, uint64_t tr)
{
    uint32_t s[4];
    load_block_be(seed, s);
    s[0] &= ~kSeedTBit;
    uint32_t t = party;
#pragma unroll 1
    for (uint32_t lv = 0; lv < n; lv++)
    {
        uint32_t cw[4];
        load_block_be(sCWp + 16 * lv, cw);
        t = dpf_step(A, s, t, (uint32_t)((x >> (n - 1 - lv)) & 1u), cw, tl, tr, lv);
    }
    dpf_leaf<GE>(A, o, s, t, kb, party, bo, g);
}

} // namespace fss
