// grotto.cu — Grotto (a Z_2 DPF with 64-bit leaves): key generation, equality and prefix-
// parity comparison shares, multiple-interval containment, interval lookup tables, and a
// full-domain expansion (sm_100a).
//
// Reference behaviour: src/impl/grotto.h:111-545 (algorithm), src/kernel/grotto.h
// (validation), include/FastFss/cuda/grotto.h (ABI). Key layout (grottoKeySetPtr,
// src/impl/grotto.h:53-79): region A sCW[N][n-6][16 B]; region B lastCW[N] (uint64);
// region C per element tLCW, tRCW (ring elements).
//
// Per-party comparison share (grottoEval, src/impl/grotto.h:284-391): parity of the
// control-bit changes (t_parent ^ t_child) on the right turns of the path, xor the parity of
// the leaf word below the input's offset, xor the party id. With equalBound the reference
// returns early once the remaining input bits are zero; every later turn is a left turn and
// the leaf offset is 0, so the early value equals the full walk's — the full-domain kernel
// below relies on that to read every x out of one leaf word and one path parity.
#include <FastFss/b200/grotto_all.h>
#include <FastFss/cuda/grotto.h>
#include <FastFss/grotto.h>

#include "fss_device.cuh"
#include "fss_host.h"
#include "grotto_core.cuh"

namespace fss {

constexpr int kGrottoThreads = 512;

// ---------------------------------------------------------------------------------------
// Key generation (src/impl/grotto.h:111-205)
// ---------------------------------------------------------------------------------------
template <typename GE>
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_keygen_kernel(uint8_t *__restrict__ key, const GE *__restrict__ alpha, const uint8_t *__restrict__ seed0,
                         const uint8_t *__restrict__ seed1, uint32_t n, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t a = N * 16 * (n - 6);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        uint8_t       *sCWp = key + i * 16 * (n - 6);
        const uint64_t al   = (uint64_t)alpha[i];
        uint32_t       s0[4], s1[4];
        load_block_be(seed0 + 16 * i, s0);
        load_block_be(seed1 + 16 * i, s1);
        s0[0] &= ~kSeedTBit;
        s1[0] &= ~kSeedTBit;
        uint32_t t0 = 0, t1 = 1;
        uint64_t tl = 0, tr = 0;
#pragma unroll 1
        for (uint32_t lv = 0; lv + 6 < n; lv++)
        {
            uint32_t G0[2][4], G1[2][4];
            aes_prg_children<0xF>(A, s0, G0[0], G0[1]);
            aes_prg_children<0xF>(A, s1, G1[0], G1[1]);
            const uint32_t tL0 = (G0[0][0] >> 24) & 1u, tR0 = (G0[1][0] >> 24) & 1u;
            const uint32_t tL1 = (G1[0][0] >> 24) & 1u, tR1 = (G1[1][0] >> 24) & 1u;
            G0[0][0] &= ~kSeedTBit, G0[1][0] &= ~kSeedTBit, G1[0][0] &= ~kSeedTBit, G1[1][0] &= ~kSeedTBit;
            const uint32_t keep = (uint32_t)((al >> (n - 1 - lv)) & 1u), lose = 1u - keep;
            uint32_t       cw[4], k0[4], k1[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
            {
                cw[c] = lose == 0 ? (G0[0][c] ^ G1[0][c]) : (G0[1][c] ^ G1[1][c]);
                k0[c] = keep == 0 ? G0[0][c] : G0[1][c];
                k1[c] = keep == 0 ? G1[0][c] : G1[1][c];
            }
            store_block_be(sCWp + 16 * lv, cw);
            const uint32_t tLCW = tL0 ^ tL1 ^ lose, tRCW = tR0 ^ tR1 ^ keep;
            tl |= (uint64_t)tLCW << lv;
            tr |= (uint64_t)tRCW << lv;
            const uint32_t m0 = 0u - t0, m1 = 0u - t1;
#pragma unroll
            for (int c = 0; c < 4; c++)
            {
                s0[c] = k0[c] ^ (cw[c] & m0);
                s1[c] = k1[c] ^ (cw[c] & m1);
            }
            const uint32_t tcw = keep ? tRCW : tLCW;
            t0                 = (keep ? tR0 : tL0) ^ (t0 & tcw);
            t1                 = (keep ? tR1 : tL1) ^ (t1 & tcw);
        }
        reinterpret_cast<unsigned long long *>(key + a)[i] = hi_u64(s0) ^ hi_u64(s1) ^ (1ull << (al & 63u));
        GE *t                                               = reinterpret_cast<GE *>(key + a + N * 8) + 2 * i;
        t[0]                                                = (GE)tl;
        t[1]                                                = (GE)tr;
    }
}

// ---------------------------------------------------------------------------------------
// Point evaluations: mode 0 = equality share, 1 = comparison share (equalBound flag)
// ---------------------------------------------------------------------------------------
template <typename GE, int MODE>
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_eval_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                       const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, bool equalBound, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        GrottoKeyView<GE> K;
        K.set(key, n, i, N);
        const uint64_t x = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
        if (MODE == 0)
        {
            uint32_t       par;
            bool           early;
            const uint64_t u = grotto_walk<GE>(A, K, seed + 16 * i, party, n, x, false, &par, &early);
            out[i]           = (GE)((u >> (x & 63u)) & 1u);
        }
        else
        {
            out[i] = (GE)grotto_cmp<GE>(A, K, seed + 16 * i, party, n, x, equalBound);
        }
    }
}

// MIC: one thread per (element, interval).
template <typename GE>
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_mic_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                      const uint8_t *__restrict__ seed, uint32_t party, const GE *__restrict__ left,
                      const GE *__restrict__ right, uint32_t m, uint32_t n, size_t N)
{
    aes_tables_build();
    AesLanes     A;
    const size_t work = N * m;
    A.init();
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t   i = w / m, q = w % m;
        GrottoKeyView<GE> K;
        K.set(key, n, i, N);
        out[w] = (GE)grotto_interval_bit<GE>(A, K, seed + 16 * i, party, n, (uint64_t)__ldg(maskedX + i),
                                             (uint64_t)__ldg(left + q), (uint64_t)__ldg(right + q));
    }
}

// MIC and interval LUT by endpoint points walked once each. Interval q needs the comparison
// shares at xP_q = x - (L_q - 1) and xQ_q = x - R_q. When the intervals touch (R_q + 1 =
// L_{q+1}), xQ_q is xP_{q+1} (the reference reuses it the same way, src/impl/grotto.h:414-423):
// the m + 1 points xP_0 .. xP_{m-1}, xQ_{m-1} serve all m intervals, or m points when the last
// interval also touches the first; otherwise each interval has its own 2 points. A CTA takes E
// elements at a time: their points are walked two per thread (both walks in the same AES
// calls, grotto_cmp2) into shared-memory bytes, and after a barrier each output (MIC: one interval's bit; LUT: E or one T_j, summed over the
// intervals) is formed from the bytes. Shares equal grotto_interval_bit's.
constexpr uint32_t kPointBytes = 32768; // shared-memory bytes for point shares per CTA pass

template <typename GE>
__device__ __forceinline__ uint32_t grotto_points_layout(const GE *left, const GE *right, uint32_t m, uint32_t n)
{
    // 0: independent intervals (2 m points); 1: touching chain (m + 1); 2: touching cycle (m)
    for (uint32_t q = 0; q + 1 < m; q++)
        if (mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(left + q + 1) - 1), n) != mod_bits<GE>((uint64_t)__ldg(right + q), n))
            return 0;
    return mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(left) - 1), n) == mod_bits<GE>((uint64_t)__ldg(right + m - 1), n)
               ? 2
               : 1;
}

// Point p of an element with masked input mx under the given layout.
template <typename GE>
__device__ __forceinline__ uint64_t grotto_point(const GE *left, const GE *right, uint32_t m, uint32_t n,
                                                 uint32_t layout, uint64_t mx, uint32_t p)
{
    uint32_t q;
    bool     isQ;
    if (layout == 0)
        q = p >> 1, isQ = (p & 1u) != 0;
    else
        q = p < m ? p : m - 1, isQ = p == m;
    const uint64_t e = isQ ? (uint64_t)__ldg(right + q) : (uint64_t)(GE)((uint64_t)__ldg(left + q) - 1);
    return mod_bits<GE>((uint64_t)(GE)(mx - e), n);
}

template <typename GE, bool LUT>
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_intervals_kernel(GE *__restrict__ out, GE *__restrict__ outT, const GE *__restrict__ maskedX,
                            const uint8_t *__restrict__ key, const uint8_t *__restrict__ seed, uint32_t party,
                            const GE *__restrict__ left, const GE *__restrict__ right, const GE *__restrict__ lut,
                            uint32_t lutNum, uint32_t m, uint32_t n, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    uint32_t *layoutSlot = reinterpret_cast<uint32_t *>(fss_smem + kAesSmemTotal);
    uint8_t  *bits       = fss_smem + kAesSmemTotal + 16;
    if (threadIdx.x == 0) *layoutSlot = grotto_points_layout<GE>(left, right, m, n);
    __syncthreads();
    const uint32_t layout = *layoutSlot;
    const uint32_t P      = layout == 0 ? 2 * m : (layout == 1 ? m + 1 : m);
    const uint32_t H      = (P + 1) / 2; // point pairs per element: one thread walks two points
    uint32_t       E      = blockDim.x / H;
    E                     = E < 1 ? 1 : E;
    if (E * P > kPointBytes) E = kPointBytes / P; // the host keeps 2 m <= kPointBytes
    if (E == 0) return;
    const uint32_t outs = LUT ? 1 + lutNum : m;     // outputs per element
    for (size_t base = (size_t)blockIdx.x * E; base < N; base += (size_t)gridDim.x * E)
    {
        for (uint32_t idx = threadIdx.x; idx < E * H; idx += blockDim.x)
        {
            const size_t i = base + idx / H;
            if (i >= N) continue;
            GrottoKeyView<GE> K;
            K.set(key, n, i, N);
            const uint32_t e = idx / H, p0 = 2 * (idx % H), p1 = p0 + 1 < P ? p0 + 1 : p0;
            const uint64_t mx    = (uint64_t)__ldg(maskedX + i);
            const uint64_t pt[2] = {grotto_point<GE>(left, right, m, n, layout, mx, p0),
                                    grotto_point<GE>(left, right, m, n, layout, mx, p1)};
            uint32_t       sh[2];
            grotto_cmp2<GE>(A, K, seed + 16 * i, party, n, pt, true, sh);
            bits[e * P + p0] = (uint8_t)sh[0];
            bits[e * P + p1] = (uint8_t)sh[1];
        }
        __syncthreads();
        for (uint32_t idx = threadIdx.x; idx < E * outs; idx += blockDim.x)
        {
            const size_t i = base + idx / outs;
            if (i >= N) continue;
            const uint32_t e = idx / outs, o = idx % outs;
            const uint64_t mx = (uint64_t)__ldg(maskedX + i);
            // interval q's bit from its two points (layout as grotto_point)
            auto bit = [&](uint32_t q) -> uint32_t {
                const uint32_t a = layout == 0 ? 2 * q : q;
                const uint32_t b = layout == 0 ? 2 * q + 1 : (q + 1 == P ? 0 : q + 1);
                // point b is xQ_q itself, or (touching) xP_{q+1} = xQ_q
                const uint64_t xP = grotto_point<GE>(left, right, m, n, layout, mx, a);
                const uint64_t xQ = grotto_point<GE>(left, right, m, n, layout, mx, b);
                return (bits[e * P + a] ^ bits[e * P + b] ^ ((xQ >= xP) ? party : 0u)) & 1u;
            };
            if (!LUT)
            {
                out[i * m + o] = (GE)bit(o);
                continue;
            }
            uint64_t acc = 0;
            for (uint32_t q = 0; q < m; q++)
            {
                const uint64_t b = bit(q);
                acc += (o == 0) ? b : b * (uint64_t)__ldg(lut + q + (size_t)(o - 1) * m);
            }
            if (party) acc = 0 - acc;
            if (o == 0)
                out[i] = (GE)acc;
            else
                outT[i * lutNum + (o - 1)] = (GE)acc;
        }
        __syncthreads();
    }
}

// Interval LUT (src/impl/grotto.h:449-545): G lanes per element stride over the intervals;
// E and T[j0 .. j0 + LMAX) are summed in the ring and reduced with warp shuffles.
template <typename GE, int LMAX>
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_lut_kernel(GE *__restrict__ outE, GE *__restrict__ outT, const GE *__restrict__ maskedX,
                      const uint8_t *__restrict__ key, const uint8_t *__restrict__ seed, uint32_t party,
                      const GE *__restrict__ left, const GE *__restrict__ right, const GE *__restrict__ lut,
                      uint32_t lutNum, uint32_t m, uint32_t n, size_t N, uint32_t G, uint32_t j0)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t   work  = ((N * G + 31) / 32) * 32; // whole warps stay in the loop (shuffles)
    const uint32_t lg    = threadIdx.x % G;
    const uint32_t jcnt  = lutNum > j0 ? min((uint32_t)LMAX, lutNum - j0) : 0u;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t i      = w / G;
        const bool   active = i < N;
        uint64_t     E = 0, T[LMAX];
#pragma unroll
        for (int k = 0; k < LMAX; k++) T[k] = 0;
        if (active)
        {
            GrottoKeyView<GE> K;
            K.set(key, n, i, N);
            const uint64_t mx = (uint64_t)__ldg(maskedX + i);
            for (uint32_t q = lg; q < m; q += G)
            {
                const uint64_t bit = grotto_interval_bit<GE>(A, K, seed + 16 * i, party, n, mx,
                                                             (uint64_t)__ldg(left + q), (uint64_t)__ldg(right + q));
                E += bit;
#pragma unroll
                for (int k = 0; k < LMAX; k++)
                    if ((uint32_t)k < jcnt) T[k] += bit * (uint64_t)__ldg(lut + q + (size_t)(j0 + k) * m);
            }
        }
        for (uint32_t off = G >> 1; off > 0; off >>= 1)
        {
            E += __shfl_xor_sync(0xffffffffu, E, off);
#pragma unroll
            for (int k = 0; k < LMAX; k++) T[k] += __shfl_xor_sync(0xffffffffu, T[k], off);
        }
        if (active && lg == 0)
        {
            if (party)
            {
                E = 0 - E;
#pragma unroll
                for (int k = 0; k < LMAX; k++) T[k] = 0 - T[k];
            }
            if (j0 == 0) outE[i] = (GE)E;
#pragma unroll
            for (int k = 0; k < LMAX; k++)
                if ((uint32_t)k < jcnt) outT[i * lutNum + j0 + k] = (GE)T[k];
        }
    }
}

// ---------------------------------------------------------------------------------------
// Full domain. One thread expands a subtree of depth d (2^d leaves) below a node reached by
// walking the top D - d levels, expanding both children of every internal node once
// (key schedule + 2 blocks sharing 14 first-round lookups; for the parents of leaves the last
// round skips word 1, which no leaf reads) and keeping right siblings on a small stack. Each
// leaf j yields the 64-bit word u_j (equality shares of x = 64 j .. 64 j + 63) and the right-turn parity
// P_j; the comparison row is excl_prefix_xor(u_j) ^ (P_j ^ party ? ~0 : 0).
// ---------------------------------------------------------------------------------------
constexpr int kAllMaxSub = 7; // 128 leaves per thread (measured best of 5..8 at n = 16)

__device__ __forceinline__ uint64_t excl_prefix_xor(uint64_t u)
{
    uint64_t p = u;
    p ^= p << 1;
    p ^= p << 2;
    p ^= p << 4;
    p ^= p << 8;
    p ^= p << 16;
    p ^= p << 32;
    return p << 1;
}

// A thread owns a subtree of 2^d leaf words of one key: the n - 6 - d levels above it are
// walked along the subtree index, then the subtree is expanded depth first. Every node
// expansion (walk, interior and leaf parents) goes through the one ggm_children call site of
// the loop, which keeps the kernel's code small; leaf parents emit both leaf words, and the
// corrected right children wait on a stack of 16-byte entries whose control and parity bits
// live in two registers.
template <typename GE, int MODE> // MODE 0: equality rows, 1: comparison (equalBound) rows
__global__ void __launch_bounds__(kGrottoThreads, 1)
    grotto_all_kernel(unsigned long long *__restrict__ out, const uint8_t *__restrict__ key,
                      const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, size_t N, uint32_t d)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t D     = n - 6;
    const uint32_t top   = D - d;
    const size_t   S     = (size_t)1 << top;
    const size_t   work  = N * S;
    const size_t   words = (size_t)1 << D; // leaf words per key
    const size_t   nleaf = (size_t)1 << d;
    const bool     vec   = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t      i = w >> top, sub = w & (S - 1);
        GrottoKeyView<GE> K;
        K.set(key, n, i, N);
        uint32_t s[4];
        load_block_be(seed + 16 * i, s);
        s[0] &= ~kSeedTBit;
        uint32_t            t = party, par = 0;
        unsigned long long *row = out + i * words + sub * nleaf;
        // leaf word of seed x with control bit tx and right-turn parity px
        auto leaf = [&](const uint32_t x[4], uint32_t tx, uint32_t px) -> unsigned long long {
            const uint64_t u0 = hi_u64(x);
            const uint64_t u  = tx ? (u0 ^ K.last) : u0;
            return (MODE == 0) ? u : (excl_prefix_xor(u) ^ ((px ^ party) ? ~0ull : 0ull));
        };
        if (d == 0)
        {
            row[0] = leaf(s, t, par); // n = 6: the root is the only leaf
            continue;
        }
        uint4    stk[kAllMaxSub - 1]; // right children below the subtree root (index: parent depth)
        uint32_t tstk = 0, pstk = 0;
        uint32_t lv = 0;               // level of the node (s, t)
        size_t   q  = 0;               // leaf parents done
#pragma unroll 1
        for (;;)
        {
            uint32_t cw[4], L[4], R[4], tL, tR;
            load_block_be(K.sCW + 16 * lv, cw);
            ggm_children(A, s, t, cw, K.tl, K.tr, lv, L, tL, R, tR);
            if (lv < top)
            {
                const uint32_t dir = (uint32_t)((sub >> (top - 1 - lv)) & 1u);
                const uint32_t tn  = dir ? tR : tL;
#pragma unroll
                for (int c = 0; c < 4; c++) s[c] = dir ? R[c] : L[c];
                par ^= dir & (t ^ tn);
                t = tn;
                lv++;
                continue;
            }
            const uint32_t depth = lv - top;
            if (depth + 1 < d)
            {
                stk[depth] = make_uint4(R[0], R[1], R[2], R[3]);
                tstk       = (tstk & ~(1u << depth)) | (tR << depth);
                pstk       = (pstk & ~(1u << depth)) | ((par ^ t ^ tR) << depth);
#pragma unroll
                for (int c = 0; c < 4; c++) s[c] = L[c];
                t = tL;
                lv++;
                continue;
            }
            // the two leaf words are adjacent: one 16-byte store when the rows are 16-byte aligned
            const unsigned long long wl = leaf(L, tL, par), wr = leaf(R, tR, par ^ t ^ tR);
            if (vec)
                reinterpret_cast<ulonglong2 *>(row)[q] = make_ulonglong2(wl, wr);
            else
                row[2 * q] = wl, row[2 * q + 1] = wr;
            if (++q == (nleaf >> 1)) break;
            // next leaf parent: the right child stacked at depth d - 2 - ctz(q)
            const uint32_t dp = d - 2 - ((uint32_t)__ffsll((long long)q) - 1);
            const uint4    e  = stk[dp];
            s[0] = e.x, s[1] = e.y, s[2] = e.z, s[3] = e.w;
            t   = (tstk >> dp) & 1u;
            par = (pstk >> dp) & 1u;
            lv  = top + dp + 1;
        }
    }
}

// Interval LUT from comparison rows: one warp per element, lanes stride over the intervals.
template <typename GE, int LMAX>
__global__ void __launch_bounds__(256)
    grotto_lut_rows_kernel(GE *__restrict__ outE, GE *__restrict__ outT, const GE *__restrict__ maskedX,
                           const uint8_t *__restrict__ rows, uint32_t party, const GE *__restrict__ left,
                           const GE *__restrict__ right, const GE *__restrict__ lut, uint32_t lutNum, uint32_t m,
                           uint32_t n, size_t N, uint32_t j0)
{
    const uint32_t lane  = threadIdx.x & 31u;
    const size_t   warps = ((size_t)gridDim.x * blockDim.x) >> 5;
    const size_t   rowBytes = ((size_t)1 << n) >> 3;
    const uint32_t jcnt  = lutNum > j0 ? min((uint32_t)LMAX, lutNum - j0) : 0u;
    for (size_t i = (((size_t)blockIdx.x * blockDim.x) + threadIdx.x) >> 5; i < N; i += warps)
    {
        const uint8_t *row = rows + i * rowBytes;
        const uint64_t x   = (uint64_t)__ldg(maskedX + i);
        uint32_t       E   = 0;
        uint64_t       T[LMAX];
#pragma unroll
        for (int k = 0; k < LMAX; k++) T[k] = 0;
        for (uint32_t q0 = 0; q0 < m; q0 += 32)
        {
            const uint32_t q   = q0 + lane;
            uint32_t       bit = 0;
            if (q < m)
            {
                const uint64_t L  = (uint64_t)__ldg(left + q), R = (uint64_t)__ldg(right + q);
                const uint64_t xP = mod_bits<GE>((uint64_t)(GE)(x - (uint64_t)(GE)(L - 1)), n);
                const uint64_t xQ = mod_bits<GE>((uint64_t)(GE)(x - R), n);
                const uint32_t sp = (__ldg(row + (xP >> 3)) >> (xP & 7)) & 1u;
                const uint32_t sq = (__ldg(row + (xQ >> 3)) >> (xQ & 7)) & 1u;
                bit               = (sp ^ sq ^ ((xQ >= xP) ? party : 0u)) & 1u;
#pragma unroll
                for (int k = 0; k < LMAX; k++)
                    if ((uint32_t)k < jcnt) T[k] += bit * (uint64_t)__ldg(lut + q + (size_t)(j0 + k) * m);
            }
            E += __popc(__ballot_sync(0xffffffffu, bit));
        }
#pragma unroll
        for (int k = 0; k < LMAX; k++)
            for (uint32_t off = 16; off > 0; off >>= 1) T[k] += __shfl_xor_sync(0xffffffffu, T[k], off);
        if (lane == 0)
        {
            uint64_t e = E;
            if (party)
            {
                e = 0 - e;
#pragma unroll
                for (int k = 0; k < LMAX; k++) T[k] = 0 - T[k];
            }
            if (j0 == 0) outE[i] = (GE)e;
#pragma unroll
            for (int k = 0; k < LMAX; k++)
                if ((uint32_t)k < jcnt) outT[i * lutNum + j0 + k] = (GE)T[k];
        }
    }
}

static inline size_t grotto_key_bytes(size_t n, size_t es, size_t N)
{
    return N * (16 * (n - 6) + 8 + 2 * es);
}

static inline size_t grotto_cache_bytes(size_t n, size_t N)
{
    return N * (16 * (n - 6) + (n - 6));
}

template <typename K, typename... Args>
static int launch(K kern, size_t work, cudaStream_t stream, Args... args)
{
    if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
    const int threads = aes_threads(work, kGrottoThreads);
    kern<<<grid_for(work, threads, 1), threads, kAesSmemTotal, stream>>>(args...);
    return launch_status();
}

template <typename GE, bool LUT, typename... Args>
static int launch_intervals(size_t N, size_t m, cudaStream_t stream, Args... args)
{
    auto          kern = grotto_intervals_kernel<GE, LUT>;
    constexpr int smem = kAesSmemTotal + 16 + (int)kPointBytes;
    if (!ensure_smem(reinterpret_cast<const void *>(kern), smem)) return FAST_FSS_RUNTIME_ERROR;
    const int threads = aes_threads(N * m, kGrottoThreads);
    kern<<<grid_for(N * m, threads, 1), threads, smem, stream>>>(args...);
    return launch_status();
}

} // namespace fss

using namespace fss;

// Validation order: GrottoKeyGenTask::check (src/kernel/grotto.h:26-47).
extern "C" FAST_FSS_API int FastFss_cuda_grottoKeyGen(void *key, size_t keyDataSize, const void *alpha,
                                                      size_t alphaDataSize, const void *seed0, size_t seedDataSize0,
                                                      const void *seed1, size_t seedDataSize1, size_t bitWidthIn,
                                                      size_t elementSize, size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum;
        if (!(6 <= bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (seedDataSize0 != N * 16 || seedDataSize1 != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (keyDataSize != grotto_key_bytes(bitWidthIn, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {alpha}, {key, seed0, seed1}); rc != FAST_FSS_SUCCESS) return rc;
        return launch(grotto_keygen_kernel<GE>, N, resolve_stream(cudaStreamPtr), (uint8_t *)key, (const GE *)alpha,
                      (const uint8_t *)seed0, (const uint8_t *)seed1, (uint32_t)bitWidthIn, N);
    });
}

// Shared checks of GrottoEqEvalTask / GrottoEvalTask (src/kernel/grotto.h:77-114,155-192).
template <typename GE>
static int grotto_point_checks(size_t sharedOutDataSize, size_t maskedXDataSize, size_t keyDataSize,
                               size_t seedDataSize, int partyId, size_t n, size_t N, size_t cacheDataSize)
{
    const size_t es = sizeof(GE);
    if (!(6 <= n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (sharedOutDataSize != N * es) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
    if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
    if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
    if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
    if (keyDataSize != grotto_key_bytes(n, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
    if (cacheDataSize != 0 && cacheDataSize != grotto_cache_bytes(n, N)) return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
    return FAST_FSS_SUCCESS;
}

extern "C" FAST_FSS_API int FastFss_cuda_grottoEqEval(void *sharedBooleanOut, size_t sharedOutDataSize,
                                                      const void *maskedX, size_t maskedXDataSize, const void *key,
                                                      size_t keyDataSize, const void *seed, size_t seedDataSize,
                                                      int partyId, size_t bitWidthIn, size_t elementSize,
                                                      size_t elementNum, void *cache, size_t cacheDataSize,
                                                      void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE = decltype(tag);
        int rc   = grotto_point_checks<GE>(sharedOutDataSize, maskedXDataSize, keyDataSize, seedDataSize, partyId,
                                         bitWidthIn, elementNum, cacheDataSize);
        if (rc != FAST_FSS_SUCCESS || elementNum == 0) return rc;
        if (int ra = check_alignment(sizeof(GE), {sharedBooleanOut, maskedX}, {key, seed}); ra != FAST_FSS_SUCCESS)
            return ra;
        return launch(grotto_eval_kernel<GE, 0>, elementNum, resolve_stream(cudaStreamPtr), (GE *)sharedBooleanOut,
                      (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                      (uint32_t)bitWidthIn, false, elementNum);
    });
}

extern "C" FAST_FSS_API int FastFss_cuda_grottoEval(void *sharedBooleanOut, size_t sharedOutDataSize,
                                                    const void *maskedX, size_t maskedXDataSize, const void *key,
                                                    size_t keyDataSize, const void *seed, size_t seedDataSize,
                                                    bool equalBound, int partyId, size_t bitWidthIn,
                                                    size_t elementSize, size_t elementNum, void *cache,
                                                    size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE = decltype(tag);
        int rc   = grotto_point_checks<GE>(sharedOutDataSize, maskedXDataSize, keyDataSize, seedDataSize, partyId,
                                         bitWidthIn, elementNum, cacheDataSize);
        if (rc != FAST_FSS_SUCCESS || elementNum == 0) return rc;
        if (int ra = check_alignment(sizeof(GE), {sharedBooleanOut, maskedX}, {key, seed}); ra != FAST_FSS_SUCCESS)
            return ra;
        return launch(grotto_eval_kernel<GE, 1>, elementNum, resolve_stream(cudaStreamPtr), (GE *)sharedBooleanOut,
                      (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                      (uint32_t)bitWidthIn, equalBound, elementNum);
    });
}

// Validation order: GrottoMICEvalTask::check (src/kernel/grotto.h:236-278).
extern "C" FAST_FSS_API int FastFss_cuda_grottoMICEval(void *sharedBooleanOut, size_t sharedBooleanOutDataSize,
                                                       const void *maskedX, size_t maskedXDataSize, const void *key,
                                                       size_t keyDataSize, const void *seed, size_t seedDataSize,
                                                       int partyId, const void *leftEndpoints,
                                                       size_t leftEndpointsDataSize, const void *rightEndpoints,
                                                       size_t rightEndpointsDataSize, size_t bitWidthIn,
                                                       size_t elementSize, size_t elementNum, void *cache,
                                                       size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(6 <= n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        const size_t m = leftEndpointsDataSize / es;
        if (m * es != leftEndpointsDataSize || m * es != rightEndpointsDataSize)
            return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (sharedBooleanOutDataSize != N * es * m) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != grotto_key_bytes(n, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != grotto_cache_bytes(n, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        if (N == 0 || m == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedBooleanOut, maskedX, leftEndpoints, rightEndpoints}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        if (2 * m <= kPointBytes)
            return launch_intervals<GE, false>(N, m, resolve_stream(cudaStreamPtr), (GE *)sharedBooleanOut, nullptr,
                                               (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed,
                                               (uint32_t)partyId, (const GE *)leftEndpoints,
                                               (const GE *)rightEndpoints, nullptr, 0u, (uint32_t)m, (uint32_t)n, N);
        return launch(grotto_mic_kernel<GE>, N * m, resolve_stream(cudaStreamPtr), (GE *)sharedBooleanOut,
                      (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                      (const GE *)leftEndpoints, (const GE *)rightEndpoints, (uint32_t)m, (uint32_t)n, N);
    });
}

// Validation order: GrottoIntervalLutEvalTask::check (src/kernel/grotto.h:330-381). With no
// intervals the reference's modulo by (elementSize * intervalNum) is undefined; this
// library reports an invalid lookup table instead.
extern "C" FAST_FSS_API int FastFss_cuda_grottoIntervalLutEval(
    void *sharedOutE, size_t sharedOutEDataSize, void *sharedOutT, size_t sharedOutTDataSize, const void *maskedX,
    size_t maskedXDataSize, const void *key, size_t keyDataSize, const void *seed, size_t seedDataSize, int partyId,
    const void *leftEndpoints, size_t leftEndpointsDataSize, const void *rightEndpoints, size_t rightEndpointsDataSize,
    const void *lookUpTable, size_t lookUpTableDataSize, size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
    size_t elementNum, void *cache, size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache, (void)bitWidthOut;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(6 <= n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(leftEndpointsDataSize == rightEndpointsDataSize && leftEndpointsDataSize % es == 0))
            return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        const size_t m = leftEndpointsDataSize / es;
        if (m == 0 || lookUpTableDataSize % (es * m) != 0) return FAST_FSS_INVALID_LOOKUP_TABLE_DATA_SIZE_ERROR;
        const size_t lutNum = lookUpTableDataSize / (es * m);
        if (sharedOutEDataSize != N * es) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (sharedOutTDataSize != N * es * lutNum) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != grotto_key_bytes(n, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != grotto_cache_bytes(n, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOutE, sharedOutT, maskedX, leftEndpoints, rightEndpoints, lookUpTable}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        if (2 * m <= kPointBytes)
            return launch_intervals<GE, true>(N, m, stream, (GE *)sharedOutE, (GE *)sharedOutT, (const GE *)maskedX,
                                              (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                                              (const GE *)leftEndpoints, (const GE *)rightEndpoints,
                                              (const GE *)lookUpTable, (uint32_t)lutNum, (uint32_t)m, (uint32_t)n, N);
        uint32_t G = 1;
        while (G < 32 && G < m) G <<= 1;
        constexpr int LMAX = 4;
        for (size_t j0 = 0; j0 < (lutNum ? lutNum : 1); j0 += LMAX)
        {
            const int rc = launch(grotto_lut_kernel<GE, LMAX>, N * G, stream, (GE *)sharedOutE, (GE *)sharedOutT,
                                  (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                                  (const GE *)leftEndpoints, (const GE *)rightEndpoints, (const GE *)lookUpTable,
                                  (uint32_t)lutNum, (uint32_t)m, (uint32_t)n, N, G, (uint32_t)j0);
            if (rc != FAST_FSS_SUCCESS) return rc;
        }
        return FAST_FSS_SUCCESS;
    });
}

template <int MODE>
static int grotto_all_entry(void *out, size_t outDataSize, const void *key, size_t keyDataSize, const void *seed,
                            size_t seedDataSize, int partyId, size_t bitWidthIn, size_t elementSize,
                            size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(6 <= n && n <= es * 8 && n <= FAST_FSS_GROTTO_ALL_MAX_BITWIDTH)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != grotto_key_bytes(n, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (outDataSize != N * (((size_t)1 << n) / 8)) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (((uintptr_t)out & 7u) != 0) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        const uint32_t D = (uint32_t)n - 6;
        const uint32_t d = D < (uint32_t)kAllMaxSub ? D : (uint32_t)kAllMaxSub;
        return launch(grotto_all_kernel<GE, MODE>, N << (D - d), resolve_stream(cudaStreamPtr),
                      (unsigned long long *)out, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                      (uint32_t)n, N, d);
    });
}

extern "C" FAST_FSS_API int FastFss_cuda_grottoEqEvalAll(void *outBits, size_t outBitsDataSize, const void *key,
                                                         size_t keyDataSize, const void *seed, size_t seedDataSize,
                                                         int partyId, size_t bitWidthIn, size_t elementSize,
                                                         size_t elementNum, void *cudaStreamPtr)
{
    return grotto_all_entry<0>(outBits, outBitsDataSize, key, keyDataSize, seed, seedDataSize, partyId, bitWidthIn,
                               elementSize, elementNum, cudaStreamPtr);
}

extern "C" FAST_FSS_API int FastFss_cuda_grottoLeEvalAll(void *outBits, size_t outBitsDataSize, const void *key,
                                                         size_t keyDataSize, const void *seed, size_t seedDataSize,
                                                         int partyId, size_t bitWidthIn, size_t elementSize,
                                                         size_t elementNum, void *cudaStreamPtr)
{
    return grotto_all_entry<1>(outBits, outBitsDataSize, key, keyDataSize, seed, seedDataSize, partyId, bitWidthIn,
                               elementSize, elementNum, cudaStreamPtr);
}

// Validation follows FastFss_cuda_grottoIntervalLutEval, with the rows in place of the key.
extern "C" FAST_FSS_API int FastFss_cuda_grottoIntervalLutEvalFromRows(
    void *sharedOutE, size_t sharedOutEDataSize, void *sharedOutT, size_t sharedOutTDataSize, const void *maskedX,
    size_t maskedXDataSize, const void *leRows, size_t leRowsDataSize, int partyId, const void *leftEndpoints,
    size_t leftEndpointsDataSize, const void *rightEndpoints, size_t rightEndpointsDataSize, const void *lookUpTable,
    size_t lookUpTableDataSize, size_t bitWidthIn, size_t elementSize, size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(6 <= n && n <= es * 8 && n <= FAST_FSS_GROTTO_ALL_MAX_BITWIDTH)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(leftEndpointsDataSize == rightEndpointsDataSize && leftEndpointsDataSize % es == 0))
            return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        const size_t m = leftEndpointsDataSize / es;
        if (m == 0 || lookUpTableDataSize % (es * m) != 0) return FAST_FSS_INVALID_LOOKUP_TABLE_DATA_SIZE_ERROR;
        const size_t lutNum = lookUpTableDataSize / (es * m);
        if (sharedOutEDataSize != N * es) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (sharedOutTDataSize != N * es * lutNum) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (leRowsDataSize != N * (((size_t)1 << n) / 8)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOutE, sharedOutT, maskedX, leftEndpoints, rightEndpoints, lookUpTable}, {}); rc != FAST_FSS_SUCCESS) return rc;
        cudaStream_t  stream = resolve_stream(cudaStreamPtr);
        constexpr int LMAX   = 4;
        for (size_t j0 = 0; j0 < (lutNum ? lutNum : 1); j0 += LMAX)
        {
            grotto_lut_rows_kernel<GE, LMAX><<<grid_for(N * 32, 256, 8), 256, 0, stream>>>(
                (GE *)sharedOutE, (GE *)sharedOutT, (const GE *)maskedX, (const uint8_t *)leRows, (uint32_t)partyId,
                (const GE *)leftEndpoints, (const GE *)rightEndpoints, (const GE *)lookUpTable, (uint32_t)lutNum,
                (uint32_t)m, (uint32_t)n, N, (uint32_t)j0);
            if (launch_status() != FAST_FSS_SUCCESS) return FAST_FSS_RUNTIME_ERROR;
        }
        return FAST_FSS_SUCCESS;
    });
}
