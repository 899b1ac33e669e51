// dpf.cu — distributed point function: key generation, evaluation, full-domain evaluation
// and multi-point evaluation (sm_100a).
//
// Reference behaviour: src/impl/dpf.h:172-380 (algorithm), src/kernel/dpf.h (validation and
// the evalAll / evalMulti index maps), include/FastFss/cuda/dpf.h (ABI). Key layout:
//   region A  sCW[N][n][16 B]; region B per element: tLCW, tRCW, lastCW[g].
//
// The leaf value convert is initialised the way the reference calls it,
// init(seed, bitWidthOut, groupSize) (src/impl/dpf.h:278,283,375): the per-value byte width
// is ceil(groupSize / 8) and the AES-CTR threshold is ceil(groupSize / 8) * bitWidthOut > 16.
// Keys and shares therefore match the reference bit for bit.
#include <FastFss/cuda/dpf.h>
#include <FastFss/dpf.h>

#include "dpf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "region_a_map.h"
#include "region_a_stage.cuh"

namespace fss {

constexpr int kDpfThreads = 512;

template <typename GE>
__global__ void __launch_bounds__(kDpfThreads, 1)
    dpf_keygen_kernel(uint8_t *__restrict__ key, const GE *__restrict__ alpha, const GE *__restrict__ beta,
                      const uint8_t *__restrict__ seed0, const uint8_t *__restrict__ seed1, uint32_t n, uint32_t bo,
                      uint32_t g, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t bstr = sizeof(GE) * (2 + (size_t)g);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        uint8_t *sCWp = key + i * 16 * n;
        GE      *kb   = reinterpret_cast<GE *>(key + N * 16 * n + i * bstr);
        uint32_t s0[4], s1[4];
        load_block_be(seed0 + 16 * i, s0);
        load_block_be(seed1 + 16 * i, s1);
        s0[0] &= ~kSeedTBit;
        s1[0] &= ~kSeedTBit;
        uint32_t       t0 = 0, t1 = 1;
        const uint64_t a  = (uint64_t)alpha[i];
        uint64_t       tl = 0, tr = 0;
        for (uint32_t lv = 0; lv < n; lv++)
        {
            uint32_t G0[2][4], G1[2][4];
            aes_prg_children<0xF>(A, s0, G0[0], G0[1]);
            aes_prg_children<0xF>(A, s1, G1[0], G1[1]);
            const uint32_t tL0 = (G0[0][0] >> 24) & 1u, tR0 = (G0[1][0] >> 24) & 1u;
            const uint32_t tL1 = (G1[0][0] >> 24) & 1u, tR1 = (G1[1][0] >> 24) & 1u;
            G0[0][0] &= ~kSeedTBit, G0[1][0] &= ~kSeedTBit, G1[0][0] &= ~kSeedTBit, G1[1][0] &= ~kSeedTBit;
            const uint32_t keep = (uint32_t)((a >> (n - 1 - lv)) & 1u);
            uint32_t       sCW[4], k0[4], k1[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
            {
                sCW[c] = keep ? (G0[0][c] ^ G1[0][c]) : (G0[1][c] ^ G1[1][c]);
                k0[c]  = keep ? G0[1][c] : G0[0][c];
                k1[c]  = keep ? G1[1][c] : G1[0][c];
            }
            store_block_be(sCWp + 16 * lv, sCW);
            const uint32_t tLCW = tL0 ^ tL1 ^ keep ^ 1u, tRCW = tR0 ^ tR1 ^ keep;
            tl |= (uint64_t)tLCW << lv;
            tr |= (uint64_t)tRCW << lv;
            const uint32_t m0 = 0u - t0, m1 = 0u - t1;
#pragma unroll
            for (int c = 0; c < 4; c++)
            {
                s0[c] = k0[c] ^ (sCW[c] & m0);
                s1[c] = k1[c] ^ (sCW[c] & m1);
            }
            const uint32_t tcw = keep ? tRCW : tLCW;
            t0                 = (keep ? tR0 : tL0) ^ (t0 & tcw);
            t1                 = (keep ? tR1 : tL1) ^ (t1 & tcw);
        }
        kb[0] = (GE)tl;
        kb[1] = (GE)tr;
        ConvertStream c0, c1;
        c0.init(s0, bo, g);
        c1.init(s1, bo, g);
        for (uint32_t j = 0; j < g; j++)
        {
            const uint64_t b = beta ? (uint64_t)beta[i * g + j] : 1u;
            uint64_t       v = b - c0.value(A, j) + c1.value(A, j);
            if (t1) v = 0 - v;
            kb[2 + j] = (GE)v;
        }
    }
}

// One leaf's g outputs. With groupSize 1 (G1) the convert (init(seed, bitWidthOut, 1), values
// of one byte) yields byte 0 of its stream: byte 0 of the seed when bitWidthOut <= 16, else
// byte 0 of AES_seed(0^128).
template <typename GE, bool G1>
__device__ __forceinline__ void dpf_all_leaf(const AesLanes &A, GE *o, const uint32_t s[4], uint32_t t, const GE *kb,
                                             uint64_t last, uint32_t party, uint32_t bo, uint32_t g)
{
    if constexpr (G1)
    {
        const uint32_t b = (bo <= 16) ? (s[0] >> 24) : (aes_zero_block_word0(A, s) >> 24);
        const uint64_t v = (uint64_t)b + (t ? last : 0);
        o[0]             = (GE)(party ? (0 - v) : v);
    }
    else
    {
        dpf_leaf<GE>(A, o, s, t, kb, party, bo, g);
    }
}

// Multi-point evaluation (work = N P): point j of element i evaluates at maskedX - point[j]
// (src/kernel/dpf.h:490-495), one tree walk per (element, point).
template <typename GE>
__global__ void __launch_bounds__(kDpfThreads, 1)
    dpf_eval_multi_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                          const uint8_t *__restrict__ seed, const GE *__restrict__ point, uint32_t party, uint32_t n,
                          uint32_t bo, uint32_t g, size_t N, size_t per, size_t work)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t bstr = sizeof(GE) * (2 + (size_t)g);
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t   i  = w / per, j = w % per;
        const GE      *kb = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        const uint64_t x  = mod_bits<GE>((uint64_t)(GE)((uint64_t)__ldg(maskedX + i) - (uint64_t)__ldg(point + j)), n);
        dpf_eval_point<GE>(A, out + (i * per + j) * g, key + i * 16 * n, kb, seed + 16 * i, party, n, bo, g, x,
                           (uint64_t)__ldg(kb), (uint64_t)__ldg(kb + 1));
    }
}

// Full-domain evaluation: out[i][(maskedX - x) mod 2^n] = dpfEval(x) for every x < 2^n
// (src/kernel/dpf.h:268-275). A thread owns one subtree of 2^d leaves of one element: it
// walks the n - d levels above the subtree root along the subtree index, then expands the
// subtree depth first, computing both children of a node under one key schedule
// (aes_prg_children). Leaf parents emit both leaves at once; above them the corrected right
// children wait on a stack (16-byte entries, control bits in a register). An element costs
// 2^n - 1 node expansions plus 2^n leaf converts instead of n 2^n single-child steps.
constexpr uint32_t kDpfAllMaxSub = 8;

// The loop has a single call site for the node expansion and one for the leaf convert, so
// the kernel's code stays small; the n - d levels above the subtree also expand both
// children and keep the one on the path.
template <typename GE, bool G1>
__global__ void __launch_bounds__(kDpfThreads, 1)
    dpf_eval_all_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                        const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, uint32_t g,
                        size_t N, uint32_t d)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t top   = n - d;
    const size_t   S     = (size_t)1 << top;
    const size_t   work  = N * S;
    const size_t   per   = (size_t)1 << n;
    const size_t   npair = (size_t)1 << (d - 1); // leaf parents per subtree (d >= 1)
    const size_t   bstr  = sizeof(GE) * (2 + (size_t)g);
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t   i    = w >> top, sub = w & (S - 1);
        const uint8_t *sCWp = key + i * 16 * n;
        const GE      *kb   = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        const uint64_t tl = (uint64_t)__ldg(kb), tr = (uint64_t)__ldg(kb + 1), last = (uint64_t)__ldg(kb + 2);
        const size_t   mx = (size_t)__ldg(maskedX + i);
        GE            *row = out + i * per * g;
        uint32_t       s[4];
        load_block_be(seed + 16 * i, s);
        s[0] &= ~kSeedTBit;
        uint32_t     t = party;
        uint4        stk[kDpfAllMaxSub - 1]; // right children below the subtree root (index: parent depth)
        uint32_t     tstk = 0;
        uint32_t     lv   = 0; // level of the node (s, t)
        size_t       q    = 0; // leaf parents done
        const size_t x0   = sub << d;
#pragma unroll 1
        for (;;)
        {
            uint32_t cw[4], L[4], R[4], tL, tR;
            load_block_be(sCWp + 16 * lv, cw);
            ggm_children(A, s, t, cw, tl, tr, lv, L, tL, R, tR);
            if (lv < top)
            {
                const bool right = (sub >> (top - 1 - lv)) & 1u;
#pragma unroll
                for (int c = 0; c < 4; c++) s[c] = right ? R[c] : L[c];
                t = right ? tR : tL;
                lv++;
                continue;
            }
            const uint32_t depth = lv - top;
            if (depth + 1 < d)
            {
                stk[depth] = make_uint4(R[0], R[1], R[2], R[3]);
                tstk       = (tstk & ~(1u << depth)) | (tR << depth);
#pragma unroll
                for (int c = 0; c < 4; c++) s[c] = L[c];
                t = tL;
                lv++;
                continue;
            }
            const size_t x = x0 + 2 * q;
#pragma unroll 1
            for (uint32_t k = 0; k < 2; k++)
            {
                uint32_t ls[4];
#pragma unroll
                for (int c = 0; c < 4; c++) ls[c] = k ? R[c] : L[c];
                dpf_all_leaf<GE, G1>(A, row + ((mx - x - k) & (per - 1)) * g, ls, k ? tR : tL, kb, last, party, bo,
                                     g);
            }
            if (++q == npair) break;
            // next leaf parent: the right child stacked at depth d - 2 - ctz(q)
            const uint32_t dp = d - 2 - ((uint32_t)__ffsll((long long)q) - 1);
            const uint4    e  = stk[dp];
            s[0] = e.x, s[1] = e.y, s[2] = e.z, s[3] = e.w;
            t  = (tstk >> dp) & 1u;
            lv = top + dp + 1;
        }
    }
}

// Plain evaluation (mode 0) with region A staged per warp through shared memory
// (region_a_stage.cuh; keys are 16-byte aligned, checked by the entry points). A warp whose
// copy does not arrive in time counts the failure in g_dpf_stage_failures, drains and stops.
__device__ unsigned int g_dpf_stage_failures;

template <typename GE, bool G1>
__global__ void __launch_bounds__(kDpfThreads, 1)
    dpf_eval_staged_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                           const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, uint32_t g,
                           size_t N, const __grid_constant__ CUtensorMap sCWmap)
{
    if (!stage_window_ok())
    {
        if (threadIdx.x == 0) atomicAdd(&g_dpf_stage_failures, 1u);
        return;
    }
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t lane = threadIdx.x & 31u, W = blockDim.x >> 5;
    const size_t   tile0 = (size_t)blockIdx.x * W + (threadIdx.x >> 5), tstride = (size_t)gridDim.x * W;
    const size_t   tiles = (N + 31) / 32;
    const size_t   bstr  = sizeof(GE) * (2 + (size_t)g);
    RegionAStage   S;
    S.init(&sCWmap, n, N, tile0, tstride);
    bool failed = false;
    for (size_t T = tile0; T < tiles && !failed; T += tstride)
    {
        const size_t i      = T * 32 + lane;
        const bool   active = i < N;
        const GE    *kb     = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        uint64_t     x = 0, tl = 0, tr = 0;
        uint32_t     s[4], t = party;
        if (active)
        {
            x  = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
            tl = (uint64_t)__ldg(kb);
            tr = (uint64_t)__ldg(kb + 1);
            load_block_be(seed + 16 * i, s);
            s[0] &= ~kSeedTBit;
        }
        for (uint32_t lv0 = 0; lv0 < n; lv0 += kStageLevels)
        {
            if (!S.wait())
            {
                failed = true;
                break;
            }
            if (active)
            {
                const uint32_t lc = min((uint32_t)kStageLevels, n - lv0);
#pragma unroll 1
                for (uint32_t j = 0; j < lc; j++)
                {
                    const uint32_t lv = lv0 + j;
                    uint32_t       cw[4];
                    S.level(j, cw);
                    t = dpf_step(A, s, t, (uint32_t)((x >> (n - 1 - lv)) & 1u), cw, tl, tr, lv);
                }
            }
            S.next();
        }
        if (failed) break;
        if (active) dpf_all_leaf<GE, G1>(A, out + i * g, s, t, kb, (uint64_t)__ldg(kb + 2), party, bo, g);
    }
    if (failed)
    {
        if (lane == 0) atomicAdd(&g_dpf_stage_failures, 1u);
        S.drain();
    }
}

unsigned int dpf_stage_failures()
{
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_dpf_stage_failures, sizeof(v)) != cudaSuccess)
    {
        cudaGetLastError();
        return 0xffffffffu;
    }
    return v;
}

static inline size_t dpf_key_bytes(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n + es + es + es * g);
}

static inline size_t dpf_cache_bytes(size_t n, size_t N)
{
    return N * 16 * n;
}

template <typename GE, int MODE>
static int dpf_launch(void *out, const void *maskedX, const void *key, const void *seed, const void *point,
                      int partyId, size_t n, size_t bo, size_t g, size_t N, size_t per, void *cudaStreamPtr)
{
    const size_t work = (MODE == 0) ? N : N * per;
    if (work == 0) return FAST_FSS_SUCCESS;
    if (int rc = check_alignment(sizeof(GE), {out, maskedX, point}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
    cudaStream_t stream = resolve_stream(cudaStreamPtr);
    if constexpr (MODE == 0)
    {
        CUtensorMap map;
        if (!encode_region_a_map(&map, key, n, N)) return FAST_FSS_RUNTIME_ERROR;
        auto           kern    = (g == 1) ? dpf_eval_staged_kernel<GE, true> : dpf_eval_staged_kernel<GE, false>;
        const int      threads = aes_threads(N, kDpfThreads);
        if (!ensure_smem(reinterpret_cast<const void *>(kern), stage_smem_bytes(kDpfThreads / 32)))
            return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, threads, 1), threads, stage_smem_bytes(threads / 32), stream>>>(
            (GE *)out, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
            (uint32_t)n, (uint32_t)bo, (uint32_t)g, N, map);
        return launch_status();
    }
    else if constexpr (MODE == 1)
    {
        const uint32_t d       = n < kDpfAllMaxSub ? (uint32_t)n : kDpfAllMaxSub;
        const size_t   units   = N << (n - d);
        auto           kern    = (g == 1) ? dpf_eval_all_kernel<GE, true> : dpf_eval_all_kernel<GE, false>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        const int threads = aes_threads(units, kDpfThreads);
        kern<<<grid_for(units, threads, 1), threads, kAesSmemTotal, stream>>>(
            (GE *)out, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
            (uint32_t)n, (uint32_t)bo, (uint32_t)g, N, d);
        return launch_status();
    }
    else
    {
        auto kern = dpf_eval_multi_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        const int threads = aes_threads(work, kDpfThreads);
        kern<<<grid_for(work, threads, 1), threads, kAesSmemTotal, stream>>>(
            (GE *)out, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (const GE *)point,
            (uint32_t)partyId, (uint32_t)n, (uint32_t)bo, (uint32_t)g, N, per, work);
        return launch_status();
    }
}

} // namespace fss

using namespace fss;

// Validation order follows DpfKeyGenTask::check (src/kernel/dpf.h:32-74).
extern "C" FAST_FSS_API int FastFss_cuda_dpfKeyGen(void *key, size_t keyDataSize, const void *alpha,
                                                   size_t alphaDataSize, const void *beta, size_t betaDataSize,
                                                   const void *seed0, size_t seedDataSize0, const void *seed1,
                                                   size_t seedDataSize1, size_t bitWidthIn, size_t bitWidthOut,
                                                   size_t groupSize, size_t elementSize, size_t elementNum,
                                                   void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum;
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (keyDataSize != dpf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (betaDataSize != 0)
        {
            if (betaDataSize != N * es * groupSize) return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        }
        else if (groupSize != 1)
        {
            return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        }
        if (seedDataSize0 != N * 16 || seedDataSize1 != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {alpha, beta}, {key, seed0, seed1}); rc != FAST_FSS_SUCCESS) return rc;
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        auto         kern   = dpf_keygen_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, aes_threads(N, kDpfThreads), 1), aes_threads(N, kDpfThreads), kAesSmemTotal, stream>>>(
            (uint8_t *)key, (const GE *)alpha, (const GE *)beta, (const uint8_t *)seed0, (const uint8_t *)seed1,
            (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, (uint32_t)groupSize, N);
        return launch_status();
    });
}

// Validation order follows DpfEvalTask::check (src/kernel/dpf.h:115-160).
extern "C" FAST_FSS_API int FastFss_cuda_dpfEval(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                                 size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                 const void *seed, size_t seedDataSize, int partyId,
                                                 size_t bitWidthIn, size_t bitWidthOut, size_t groupSize,
                                                 size_t elementSize, size_t elementNum, void *cache,
                                                 size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum;
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != dpf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (sharedOutDataSize != N * es * groupSize) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != dpf_cache_bytes(bitWidthIn, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        return dpf_launch<GE, 0>(sharedOut, maskedX, key, seed, nullptr, partyId, bitWidthIn, bitWidthOut, groupSize,
                                 N, 1, cudaStreamPtr);
    });
}

// Validation order follows DpfEvalAllTask::check (src/kernel/dpf.h:203-251).
extern "C" FAST_FSS_API int FastFss_cuda_dpfEvalAll(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                                    size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                    const void *seed, size_t seedDataSize, int partyId,
                                                    size_t bitWidthIn, size_t bitWidthOut, size_t groupSize,
                                                    size_t elementSize, size_t elementNum, void *cache,
                                                    size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum;
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != dpf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        // The full domain must be addressable: the reference computes 1ULL << n here.
        if (bitWidthIn >= 64) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        const size_t dom = (size_t)1 << bitWidthIn;
        if (sharedOutDataSize != N * es * dom * groupSize) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != dpf_cache_bytes(bitWidthIn, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        return dpf_launch<GE, 1>(sharedOut, maskedX, key, seed, nullptr, partyId, bitWidthIn, bitWidthOut, groupSize,
                                 N, dom, cudaStreamPtr);
    });
}

// Validation order follows DpfEvalMultiTask::check (src/kernel/dpf.h:406-458).
extern "C" FAST_FSS_API int FastFss_cuda_dpfEvalMulti(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                                      size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                      const void *seed, size_t seedDataSize, int partyId,
                                                      const void *point, size_t pointDataSize, size_t bitWidthIn,
                                                      size_t bitWidthOut, size_t groupSize, size_t elementSize,
                                                      size_t elementNum, void *cache, size_t cacheDataSize,
                                                      void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum;
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (pointDataSize % es != 0) return FAST_FSS_INVALID_POINT_DATA_SIZE_ERROR;
        if (keyDataSize != dpf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        const size_t P = pointDataSize / es;
        if (sharedOutDataSize != N * es * P * groupSize) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != dpf_cache_bytes(bitWidthIn, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        return dpf_launch<GE, 2>(sharedOut, maskedX, key, seed, point, partyId, bitWidthIn, bitWidthOut, groupSize,
                                 N, P, cudaStreamPtr);
    });
}
