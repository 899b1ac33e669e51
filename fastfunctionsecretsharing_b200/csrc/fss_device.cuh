// fss_device.cuh — device building blocks shared by every FSS kernel (sm_100a).
//
// AES-128 here is the PRG of the GGM trees: every tree node re-keys AES with its own
// 16-byte seed (src/impl/dcf.h:230-233 of the reference), so nothing about a round key is
// shared between threads and the key schedule runs next to the block rounds, in registers.
//
// Shared-memory T-tables. The four encryption tables Te0..Te3 (Te_k = ror(Te0, 8k)) live
// in dynamic shared memory, replicated 32 times so that lane l only ever touches bank l:
//
//     byte offset(k, x, lane) = (k >> 1) << 16  |  x << 8  |  (k & 1) << 7  |  lane << 2
//
// i.e. two 64 KiB regions (Te0|Te1 and Te2|Te3), 256 rows of 256 bytes, each row holding
// 32 lane copies of Te_{2h} followed by 32 lane copies of Te_{2h+1}. Every lookup is
// conflict-free, and the address is one byte-permute (PRMT) of the state word with a
// per-lane constant: the state byte lands in bits 8..15, the lane/table constant fills the
// rest. The S-box needed by the last round and the key schedule is read out of these same
// tables (Te0 = (2s, s, s, 3s) and its rotations carry s in every byte position).
//
// All state words are big-endian views of the 16 state bytes, as in FIPS-197 and the
// reference (src/impl/aes.h:10-18): byte 0 of the block is the MSB of word 0.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fss {

constexpr int      kAesSmemBytes   = 2 * 65536;         // replicated Te0..Te3
constexpr int      kSboxScratchOff = kAesSmemBytes;     // 256-byte S-box scratch during set-up
constexpr int      kAesSmemTotal   = kAesSmemBytes + 256;
constexpr uint32_t kSeedTBit       = 1u << 24;          // bit 0 of byte 0 = t bit / MASK_MSB63

extern __shared__ __align__(16) unsigned char fss_smem[];

// ---------------------------------------------------------------------------------------
// Table construction (S-box from its definition: inverse in GF(2^8), then the affine map).
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t gf_xtime(uint32_t a)
{
    return ((a << 1) ^ ((a & 0x80u) ? 0x1bu : 0u)) & 0xffu;
}

__device__ __forceinline__ uint32_t gf_mul(uint32_t a, uint32_t b)
{
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
    {
        if (b & 1u) r ^= a;
        a = gf_xtime(a);
        b >>= 1;
    }
    return r;
}

__device__ __forceinline__ uint32_t sbox_of(uint32_t x)
{
    uint32_t inv = 0;
    if (x != 0)
    {
        // x^254 = x^-1 ; 254 = 0b11111110
        uint32_t r = 1, b = x;
#pragma unroll
        for (int i = 0; i < 8; i++)
        {
            if ((254u >> i) & 1u) r = gf_mul(r, b);
            b = gf_mul(b, b);
        }
        inv = r;
    }
    uint32_t s = inv;
#pragma unroll
    for (int i = 1; i <= 4; i++) s ^= ((inv << i) | (inv >> (8 - i))) & 0xffu;
    return (s ^ 0x63u) & 0xffu;
}

// Fills the replicated tables. Every thread of the block must call it (it syncs).
__device__ __forceinline__ void aes_tables_build()
{
    uint8_t* sb = fss_smem + kSboxScratchOff;
    for (int x = threadIdx.x; x < 256; x += blockDim.x) sb[x] = (uint8_t)sbox_of((uint32_t)x);
    __syncthreads();
    uint32_t* tab = reinterpret_cast<uint32_t*>(fss_smem);
    // 32768 words; word w: region h = w >> 14, row x = (w >> 6) & 255, column c = w & 63.
    for (int w = threadIdx.x; w < kAesSmemBytes / 4; w += blockDim.x)
    {
        const uint32_t h  = (uint32_t)w >> 14;
        const uint32_t x  = ((uint32_t)w >> 6) & 255u;
        const uint32_t k  = 2u * h + (((uint32_t)w >> 5) & 1u);
        const uint32_t s  = sb[x];
        const uint32_t s2 = gf_xtime(s);
        const uint32_t t0 = (s2 << 24) | (s << 16) | (s << 8) | (s2 ^ s);
        tab[w]            = (k == 0) ? t0 : __funnelshift_r(t0, t0, 8 * k);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------
// Lookups
// ---------------------------------------------------------------------------------------

struct AesLanes
{
    uint32_t L[4]; // per-table lane constants: (k>>1)<<16 | (k&1)<<7 | lane<<2

    __device__ __forceinline__ void init()
    {
        const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
        for (int k = 0; k < 4; k++) L[k] = ((uint32_t)(k >> 1) << 16) | ((uint32_t)(k & 1) << 7) | (lane << 2);
    }
};

// Te_k[byte B of w] for this lane. B = 3 is the most significant byte.
template <int K, int B>
__device__ __forceinline__ uint32_t te(const AesLanes& A, uint32_t w)
{
    const uint32_t addr = __byte_perm(w, A.L[K], 0x7604u | ((uint32_t)B << 4));
    return *reinterpret_cast<const uint32_t*>(fss_smem + addr);
}

// Assembles (va.b3, vb.b2, vc.b1, vd.b0): the S-box bytes read out of four rotated-table
// lookups (Te2 carries s in byte 3, Te3 in byte 2, Te0 in byte 1, Te1 in byte 0).
__device__ __forceinline__ uint32_t merge_sbytes(uint32_t va, uint32_t vb, uint32_t vc, uint32_t vd)
{
    const uint32_t lo = __byte_perm(vc, vd, 0x0014u);
    const uint32_t hi = __byte_perm(va, vb, 0x3600u);
    return __byte_perm(lo, hi, 0x7610u);
}

// (S[a.b3] << 24 | S[b.b2] << 16 | S[c.b1] << 8 | S[d.b0]): SubBytes+ShiftRows of a column.
__device__ __forceinline__ uint32_t sub_col(const AesLanes& A, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    return merge_sbytes(te<2, 3>(A, a), te<3, 2>(A, b), te<0, 1>(A, c), te<1, 0>(A, d));
}

// One key-schedule step in place: w <- next round key (FIPS-197 5.2).
__device__ __forceinline__ void key_step(const AesLanes& A, uint32_t w[4], uint32_t rcon)
{
    // SubWord(RotWord(w3)) = (S[w3.b2], S[w3.b1], S[w3.b0], S[w3.b3]).
    const uint32_t t =
        merge_sbytes(te<2, 2>(A, w[3]), te<3, 1>(A, w[3]), te<0, 0>(A, w[3]), te<1, 3>(A, w[3])) ^ (rcon << 24);
    w[0] ^= t;
    w[1] ^= w[0];
    w[2] ^= w[1];
    w[3] ^= w[2];
}

__device__ __forceinline__ void enc_round(const AesLanes& A, uint32_t s[4], const uint32_t k[4])
{
    const uint32_t t0 = te<0, 3>(A, s[0]) ^ te<1, 2>(A, s[1]) ^ te<2, 1>(A, s[2]) ^ te<3, 0>(A, s[3]) ^ k[0];
    const uint32_t t1 = te<0, 3>(A, s[1]) ^ te<1, 2>(A, s[2]) ^ te<2, 1>(A, s[3]) ^ te<3, 0>(A, s[0]) ^ k[1];
    const uint32_t t2 = te<0, 3>(A, s[2]) ^ te<1, 2>(A, s[3]) ^ te<2, 1>(A, s[0]) ^ te<3, 0>(A, s[1]) ^ k[2];
    const uint32_t t3 = te<0, 3>(A, s[3]) ^ te<1, 2>(A, s[0]) ^ te<2, 1>(A, s[1]) ^ te<3, 0>(A, s[2]) ^ k[3];
    s[0] = t0, s[1] = t1, s[2] = t2, s[3] = t3;
}

__device__ __forceinline__ void enc_last(const AesLanes& A, uint32_t s[4], const uint32_t k[4])
{
    const uint32_t t0 = sub_col(A, s[0], s[1], s[2], s[3]) ^ k[0];
    const uint32_t t1 = sub_col(A, s[1], s[2], s[3], s[0]) ^ k[1];
    const uint32_t t2 = sub_col(A, s[2], s[3], s[0], s[1]) ^ k[2];
    const uint32_t t3 = sub_col(A, s[3], s[0], s[1], s[2]) ^ k[3];
    s[0] = t0, s[1] = t1, s[2] = t2, s[3] = t3;
}

// Encrypts NB blocks (in place, big-endian words) under one 16-byte key given as
// big-endian words; the key schedule runs alongside the rounds.
template <int NB>
__device__ __forceinline__ void aes_encrypt(const AesLanes& A, const uint32_t key[4], uint32_t st[NB][4])
{
    uint32_t w[4] = {key[0], key[1], key[2], key[3]};
#pragma unroll
    for (int b = 0; b < NB; b++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) st[b][c] ^= w[c];
    }
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 0; r < 9; r++)
    {
        key_step(A, w, RCON[r]);
#pragma unroll
        for (int b = 0; b < NB; b++) enc_round(A, st[b], w);
    }
    key_step(A, w, RCON[9]);
#pragma unroll
    for (int b = 0; b < NB; b++) enc_last(A, st[b], w);
}

// Word 0 of AES_key(0^128). The state after the initial AddRoundKey of the all-zero block is
// the key itself; the last round computes only the first column: 40 + 144 + 4 = 188 lookups.
__device__ __forceinline__ uint32_t aes_zero_block_word0(const AesLanes& A, const uint32_t key[4])
{
    uint32_t           w[4]  = {key[0], key[1], key[2], key[3]};
    uint32_t           st[4] = {key[0], key[1], key[2], key[3]};
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 0; r < 9; r++)
    {
        key_step(A, w, RCON[r]);
        enc_round(A, st, w);
    }
    key_step(A, w, RCON[9]);
    return sub_col(A, st[0], st[1], st[2], st[3]) ^ w[0];
}

// Blocks 2 dir and 2 dir + 1 of the GGM expansion under `key`: the seed child (all four words,
// into sOut) and the value child (its first VW words, into vOut). Their plaintexts differ only
// in bytes 0 and 8, which feed one lookup each of first-round columns 0 and 2, so the other 14
// first-round lookups are shared; the value child's last round computes only the VW columns
// that are read. Lookups: 40 (schedule) + 160 (seed child) + 160 - 14 - 4 (4 - VW) (value).
// NK independent nodes (keys and directions) are expanded side by side, round by round.
template <int NK, int VW>
__device__ __forceinline__ void aes_prg_pair(const AesLanes& A, const uint32_t key[NK][4], const uint32_t dir[NK],
                                             uint32_t sOut[NK][4], uint32_t vOut[NK][VW])
{
    uint32_t w[NK][4], sa[NK][4], sb[NK][4];
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) w[k][c] = key[k][c];
        const uint32_t a0 = w[k][0] ^ ((4u * dir[k]) << 24), b0 = w[k][0] ^ ((4u * dir[k] + 2u) << 24);
        const uint32_t a2 = w[k][2] ^ ((4u * dir[k] + 1u) << 24), b2 = w[k][2] ^ ((4u * dir[k] + 3u) << 24);
        const uint32_t s1 = w[k][1], s3 = w[k][3];
        key_step(A, w[k], 0x01u);
        // round 1: bytes other than the MSBs of words 0 and 2 are the same in both states
        const uint32_t x0 = te<1, 2>(A, s1) ^ te<2, 1>(A, a2) ^ te<3, 0>(A, s3) ^ w[k][0];
        const uint32_t t1 = te<0, 3>(A, s1) ^ te<1, 2>(A, a2) ^ te<2, 1>(A, s3) ^ te<3, 0>(A, a0) ^ w[k][1];
        const uint32_t x2 = te<1, 2>(A, s3) ^ te<2, 1>(A, a0) ^ te<3, 0>(A, s1) ^ w[k][2];
        const uint32_t t3 = te<0, 3>(A, s3) ^ te<1, 2>(A, a0) ^ te<2, 1>(A, s1) ^ te<3, 0>(A, a2) ^ w[k][3];
        sa[k][0] = te<0, 3>(A, a0) ^ x0, sa[k][1] = t1, sa[k][2] = te<0, 3>(A, a2) ^ x2, sa[k][3] = t3;
        sb[k][0] = te<0, 3>(A, b0) ^ x0, sb[k][1] = t1, sb[k][2] = te<0, 3>(A, b2) ^ x2, sb[k][3] = t3;
    }
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 1; r < 9; r++)
    {
#pragma unroll
        for (int k = 0; k < NK; k++)
        {
            key_step(A, w[k], RCON[r]);
            enc_round(A, sa[k], w[k]);
            enc_round(A, sb[k], w[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
        key_step(A, w[k], RCON[9]);
        enc_last(A, sa[k], w[k]);
#pragma unroll
        for (int c = 0; c < 4; c++) sOut[k][c] = sa[k][c];
#pragma unroll
        for (int c = 0; c < VW; c++)
            vOut[k][c] = sub_col(A, sb[k][c], sb[k][(c + 1) & 3], sb[k][(c + 2) & 3], sb[k][(c + 3) & 3]) ^ w[k][c];
    }
}

// Both children of the GGM node keyed by `key` (blocks 0 and 1: LE64(0) || LE64(1) and
// LE64(2) || LE64(3)), sharing the 14 first-round lookups their plaintexts have in common. The
// last round computes only the columns set in MASK (bit c: word c); the others are left 0.
template <int MASK>
__device__ __forceinline__ void aes_prg_children(const AesLanes& A, const uint32_t key[4], uint32_t L[4], uint32_t R[4])
{
    uint32_t       w[4] = {key[0], key[1], key[2], key[3]};
    const uint32_t a0 = w[0], b0 = w[0] ^ (2u << 24);
    const uint32_t a2 = w[2] ^ (1u << 24), b2 = w[2] ^ (3u << 24);
    const uint32_t s1 = w[1], s3 = w[3];
    key_step(A, w, 0x01u);
    const uint32_t x0 = te<1, 2>(A, s1) ^ te<2, 1>(A, a2) ^ te<3, 0>(A, s3) ^ w[0];
    const uint32_t t1 = te<0, 3>(A, s1) ^ te<1, 2>(A, a2) ^ te<2, 1>(A, s3) ^ te<3, 0>(A, a0) ^ w[1];
    const uint32_t x2 = te<1, 2>(A, s3) ^ te<2, 1>(A, a0) ^ te<3, 0>(A, s1) ^ w[2];
    const uint32_t t3 = te<0, 3>(A, s3) ^ te<1, 2>(A, a0) ^ te<2, 1>(A, s1) ^ te<3, 0>(A, a2) ^ w[3];
    uint32_t       sa[4] = {te<0, 3>(A, a0) ^ x0, t1, te<0, 3>(A, a2) ^ x2, t3};
    uint32_t       sb[4] = {te<0, 3>(A, b0) ^ x0, t1, te<0, 3>(A, b2) ^ x2, t3};
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 1; r < 9; r++)
    {
        key_step(A, w, RCON[r]);
        enc_round(A, sa, w);
        enc_round(A, sb, w);
    }
    key_step(A, w, RCON[9]);
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        if (MASK & (1 << c))
        {
            L[c] = sub_col(A, sa[c], sa[(c + 1) & 3], sa[(c + 2) & 3], sa[(c + 3) & 3]) ^ w[c];
            R[c] = sub_col(A, sb[c], sb[(c + 1) & 3], sb[(c + 2) & 3], sb[(c + 3) & 3]) ^ w[c];
        }
        else
        {
            L[c] = 0;
            R[c] = 0;
        }
    }
}

// Both children of the tree node (s, t) at level lv, as evaluation derives them: the control
// bit of a child is bit 0 of its byte 0 xor (its tCW bit at lv, i.e. bit lv of tl / tr) when
// t is set; the seed is the child block with that bit cleared, xor cw when t is set.
__device__ __forceinline__ void ggm_children(const AesLanes& A, const uint32_t s[4], uint32_t t, const uint32_t cw[4],
                                             uint64_t tl, uint64_t tr, uint32_t lv, uint32_t L[4], uint32_t& tL,
                                             uint32_t R[4], uint32_t& tR)
{
    aes_prg_children<0xF>(A, s, L, R);
    const uint32_t m = 0u - t;
    tL               = ((L[0] >> 24) & 1u) ^ ((uint32_t)((tl >> lv) & 1u) & t);
    tR               = ((R[0] >> 24) & 1u) ^ ((uint32_t)((tr >> lv) & 1u) & t);
    L[0] &= ~kSeedTBit;
    R[0] &= ~kSeedTBit;
#pragma unroll
    for (int c = 0; c < 4; c++)
    {
        L[c] ^= cw[c] & m;
        R[c] ^= cw[c] & m;
    }
}

// Blocks 0..3 of the GGM expansion under `key` (block j: LE64(2j) || LE64(2j + 1)), as key
// generation needs them: the seed children 0 and 2 in full, the value children 1 and 3 only as
// far as their first VW words (VW = 4: in full). The four plaintexts differ only in bytes 0 and
// 8, so first-round columns 1 and 3 are shared by all four blocks and columns 0 and 2 share
// three of their four lookups: 22 first-round lookups instead of 64.
template <int VW>
__device__ __forceinline__ void aes_prg_quad(const AesLanes& A, const uint32_t key[4], uint32_t G[4][4])
{
    uint32_t       w[4] = {key[0], key[1], key[2], key[3]};
    const uint32_t s0 = w[0], s1 = w[1], s2 = w[2], s3 = w[3];
    key_step(A, w, 0x01u);
    const uint32_t x0 = te<1, 2>(A, s1) ^ te<2, 1>(A, s2) ^ te<3, 0>(A, s3) ^ w[0];
    const uint32_t t1 = te<0, 3>(A, s1) ^ te<1, 2>(A, s2) ^ te<2, 1>(A, s3) ^ te<3, 0>(A, s0) ^ w[1];
    const uint32_t x2 = te<1, 2>(A, s3) ^ te<2, 1>(A, s0) ^ te<3, 0>(A, s1) ^ w[2];
    const uint32_t t3 = te<0, 3>(A, s3) ^ te<1, 2>(A, s0) ^ te<2, 1>(A, s1) ^ te<3, 0>(A, s2) ^ w[3];
    uint32_t       st[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
    {
        // bytes 0 and 8 of block j are 2j and 2j + 1; the other bytes of the plaintext are 0
        st[j][0] = te<0, 3>(A, s0 ^ ((2u * j) << 24)) ^ x0;
        st[j][1] = t1;
        st[j][2] = te<0, 3>(A, s2 ^ ((2u * j + 1u) << 24)) ^ x2;
        st[j][3] = t3;
    }
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 1; r < 9; r++)
    {
        key_step(A, w, RCON[r]);
#pragma unroll
        for (int j = 0; j < 4; j++) enc_round(A, st[j], w);
    }
    key_step(A, w, RCON[9]);
#pragma unroll
    for (int j = 0; j < 4; j++)
    {
        const int cols = (j & 1) ? VW : 4;
#pragma unroll
        for (int c = 0; c < 4; c++)
            G[j][c] = (c < cols) ? (sub_col(A, st[j][c], st[j][(c + 1) & 3], st[j][(c + 2) & 3], st[j][(c + 3) & 3]) ^
                                    w[c])
                                 : 0u;
    }
}

// NK independent keys, NB blocks under each. The round loop is not unrolled (small code for
// the kernels that instantiate several of these); inside an iteration the block rounds under
// round key r and the schedule step to round key r + 1 are independent, so they overlap.
template <int NK, int NB>
__device__ __forceinline__ void aes_encrypt_keys(const AesLanes& A, const uint32_t key[NK][4],
                                                 uint32_t st[NK][NB][4])
{
    uint32_t w[NK][4];
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) w[k][c] = key[k][c];
#pragma unroll
        for (int b = 0; b < NB; b++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) st[k][b][c] ^= w[k][c];
        }
        key_step(A, w[k], 0x01u);
    }
    uint32_t rcon = 0x01u;
#pragma unroll 1
    for (int r = 1; r < 10; r++)
    {
        rcon = gf_xtime(rcon);
        uint32_t nw[NK][4];
#pragma unroll
        for (int k = 0; k < NK; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) nw[k][c] = w[k][c];
            key_step(A, nw[k], rcon);
#pragma unroll
            for (int b = 0; b < NB; b++) enc_round(A, st[k][b], w[k]);
        }
#pragma unroll
        for (int k = 0; k < NK; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) w[k][c] = nw[k][c];
        }
    }
#pragma unroll
    for (int k = 0; k < NK; k++)
    {
#pragma unroll
        for (int b = 0; b < NB; b++) enc_last(A, st[k][b], w[k]);
    }
}

// Two independent groups in the same rounds: N1 keys with B1 blocks each and N2 keys with B2
// blocks each (e.g. the next tree level of a walk together with the value convert of the level
// before it, which do not depend on each other). Rolled rounds, as aes_encrypt_keys.
template <int N1, int B1, int N2, int B2>
__device__ __forceinline__ void aes_encrypt_groups(const AesLanes& A, const uint32_t k1[N1][4], uint32_t st1[N1][B1][4],
                                                   const uint32_t k2[N2][4], uint32_t st2[N2][B2][4])
{
    uint32_t w1[N1][4], w2[N2][4];
#pragma unroll
    for (int k = 0; k < N1; k++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) w1[k][c] = k1[k][c];
#pragma unroll
        for (int b = 0; b < B1; b++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) st1[k][b][c] ^= w1[k][c];
        }
        key_step(A, w1[k], 0x01u);
    }
#pragma unroll
    for (int k = 0; k < N2; k++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) w2[k][c] = k2[k][c];
#pragma unroll
        for (int b = 0; b < B2; b++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) st2[k][b][c] ^= w2[k][c];
        }
        key_step(A, w2[k], 0x01u);
    }
    uint32_t rcon = 0x01u;
#pragma unroll 1
    for (int r = 1; r < 10; r++)
    {
        rcon = gf_xtime(rcon);
        uint32_t n1[N1][4], n2[N2][4];
#pragma unroll
        for (int k = 0; k < N1; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) n1[k][c] = w1[k][c];
            key_step(A, n1[k], rcon);
#pragma unroll
            for (int b = 0; b < B1; b++) enc_round(A, st1[k][b], w1[k]);
        }
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) n2[k][c] = w2[k][c];
            key_step(A, n2[k], rcon);
#pragma unroll
            for (int b = 0; b < B2; b++) enc_round(A, st2[k][b], w2[k]);
        }
#pragma unroll
        for (int k = 0; k < N1; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) w1[k][c] = n1[k][c];
        }
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
#pragma unroll
            for (int c = 0; c < 4; c++) w2[k][c] = n2[k][c];
        }
    }
#pragma unroll
    for (int k = 0; k < N1; k++)
    {
#pragma unroll
        for (int b = 0; b < B1; b++) enc_last(A, st1[k][b], w1[k]);
    }
#pragma unroll
    for (int k = 0; k < N2; k++)
    {
#pragma unroll
        for (int b = 0; b < B2; b++) enc_last(A, st2[k][b], w2[k]);
    }
}

// PRG block j of the GGM expansion: plaintext = LE64(2j) || LE64(2j+1) as BE words.
__device__ __forceinline__ void prg_block(uint32_t st[4], uint32_t j)
{
    st[0] = (2u * j) << 24;
    st[1] = 0;
    st[2] = (2u * j + 1u) << 24;
    st[3] = 0;
}

// ---------------------------------------------------------------------------------------
// Byte-order helpers
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t bswap32(uint32_t x)
{
    return __byte_perm(x, 0, 0x0123u);
}

// 16 bytes from global memory (16-byte aligned) as big-endian words.
__device__ __forceinline__ void load_block_be(const void* p, uint32_t w[4])
{
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    w[0]          = bswap32(v.x);
    w[1]          = bswap32(v.y);
    w[2]          = bswap32(v.z);
    w[3]          = bswap32(v.w);
}

__device__ __forceinline__ void store_block_be(void* p, const uint32_t w[4])
{
    uint4 v;
    v.x                            = bswap32(w[0]);
    v.y                            = bswap32(w[1]);
    v.z                            = bswap32(w[2]);
    v.w                            = bswap32(w[3]);
    *reinterpret_cast<uint4*>(p) = v;
}

// Byte b (0..15) of a block held as big-endian words.
__device__ __forceinline__ uint32_t block_byte(const uint32_t w[4], int b)
{
    return (w[b >> 2] >> (24 - 8 * (b & 3))) & 0xffu;
}

// Little-endian value of the first `nbytes` (1..8) bytes of a block.
__device__ __forceinline__ uint64_t block_le_prefix(const uint32_t w[4], int nbytes)
{
    const uint64_t v = (uint64_t)bswap32(w[0]) | ((uint64_t)bswap32(w[1]) << 32);
    return nbytes >= 8 ? v : (v & ((1ull << (8 * nbytes)) - 1ull));
}

// ---------------------------------------------------------------------------------------
// Ring element access
// ---------------------------------------------------------------------------------------

template <typename GE>
__device__ __forceinline__ uint64_t ld_ge(const void* p, size_t i)
{
    return (uint64_t)__ldg(reinterpret_cast<const GE*>(p) + i);
}

template <typename GE>
__device__ __forceinline__ void st_ge(void* p, size_t i, uint64_t v)
{
    reinterpret_cast<GE*>(p)[i] = (GE)v;
}

template <typename GE>
__device__ __forceinline__ uint64_t mod_bits(uint64_t x, uint32_t w)
{
    return w >= 64 ? x : (x & ((1ull << w) - 1ull));
}

// ---------------------------------------------------------------------------------------
// Value convert (reference DcfConvertCtx / DpfConvertCtx, src/impl/dcf.h:69-137).
// The group vector of `groupSize` values of `ges` bytes each is read out of one 16-byte
// seed when ges*groupSize <= 16, else out of an AES-CTR stream keyed by the seed whose
// 16-byte block b is AES_seed(LE64(0) || LE64(floor(16 b / ges))).
// ---------------------------------------------------------------------------------------

struct ConvertStream
{
    uint32_t key[4];
    uint32_t blk[4];
    int      cur; // index of the block held in blk (-1: none)
    int      ges;
    bool     aes;

    __device__ __forceinline__ void init(const uint32_t seed[4], uint32_t groupSize, uint32_t bitWidth)
    {
        ges = (int)((bitWidth + 7) / 8);
        aes = (uint64_t)ges * groupSize > 16;
#pragma unroll
        for (int c = 0; c < 4; c++) key[c] = seed[c], blk[c] = seed[c];
        cur = aes ? -1 : 0;
    }

    __device__ __forceinline__ void fetch(const AesLanes& A, int b)
    {
        const uint32_t ctr = (uint32_t)((16 * b) / ges);
        uint32_t       st[1][4];
        st[0][0] = 0;
        st[0][1] = 0;
        st[0][2] = bswap32(ctr);
        st[0][3] = 0;
        aes_encrypt<1>(A, key, st);
#pragma unroll
        for (int c = 0; c < 4; c++) blk[c] = st[0][c];
        cur = b;
    }

    // Value j of the group (bytes at or beyond position 8 of a value are dropped).
    __device__ __forceinline__ uint64_t value(const AesLanes& A, uint32_t j)
    {
        uint64_t r   = 0;
        int      off = (int)j * ges;
        for (int i = 0; i < ges; i++)
        {
            const int p = off + i;
            int       b = aes ? (p >> 4) : 0;
            if (aes && b != cur) fetch(A, b);
            if (i < 8) r |= (uint64_t)block_byte(blk, p & 15) << (8 * i);
        }
        return r;
    }
};

} // namespace fss
