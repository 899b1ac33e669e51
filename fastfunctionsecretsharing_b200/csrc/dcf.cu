// dcf.cu — distributed comparison function: key generation and evaluation (sm_100a).
//
// Reference behaviour: src/impl/dcf.h:187-491 (algorithm), src/kernel/dcf.h:30-71,115-163
// (validation), include/FastFss/cuda/dcf.h (ABI). Keys use the reference byte layout:
//   region A  sCW[N][n][16 B]                       (element-major, 16-byte aligned)
//   region B  per element: vCW[n][g], tLCW, tRCW, lastCW[g]   (ring elements)
//
// One thread walks one element's tree; the AES PRG runs out of the replicated shared-memory
// T-tables (fss_device.cuh). Evaluation only expands the child on the input's path: the
// seed/value blocks (2 dir, 2 dir + 1) of G(s) (2 blocks + 1 key schedule per level instead
// of the reference's 4 blocks), which yields the same shares bit for bit because the other
// direction's blocks never reach the output.
#include <FastFss/cuda/dcf.h>
#include <FastFss/dcf.h>

#include <FastFss/b200/diag.h>

#include "dcf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "region_a_map.h"
#include "region_a_stage.cuh"

namespace fss {

constexpr int kDcfThreads       = 512;
constexpr int kDcfKeygenThreads = 512; // 256 threads without a register cap measured 5 % slower

// Staging failures (FastFss_b200_stageTimeouts): a wait for a copy that ran out, or a launch
// whose shared window could not hold aligned stages. Zero in normal operation.
__device__ unsigned int g_stage_timeouts;

// ---------------------------------------------------------------------------------------
// Key generation (src/impl/dcf.h:187-368): one element per thread.
// ---------------------------------------------------------------------------------------
template <typename GE>
__global__ void __launch_bounds__(kDcfKeygenThreads, 1)
    dcf_keygen_kernel(uint8_t *__restrict__ key, const GE *__restrict__ alpha, const GE *__restrict__ beta,
                      const uint8_t *__restrict__ seed0, const uint8_t *__restrict__ seed1, uint32_t n, uint32_t bo,
                      uint32_t g, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
        dcf_keygen_element<GE>(A, key, N, i, (uint64_t)alpha[i], beta ? beta + i * g : nullptr, seed0 + 16 * i,
                               seed1 + 16 * i, n, bo, g);
}

// ---------------------------------------------------------------------------------------
// Evaluation, groupSize == 1 (the hot path): seed, control bit and accumulator in registers.
// ---------------------------------------------------------------------------------------
// The walk of dcf_eval_g1 (dcf_core.cuh) with region A (correction words) staged per warp
// through shared memory (region_a_stage.cuh; the entry point refuses keys that are not
// 16-byte aligned). A warp whose copy does not arrive in time counts the failure in
// g_stage_timeouts, drains its copies in flight and stops; its remaining shares are not written.
template <typename GE>
__global__ void __launch_bounds__(kDcfThreads, 1)
    dcf_eval_g1_staged_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                              const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, size_t N,
                              const __grid_constant__ CUtensorMap sCWmap)
{
    if (!stage_window_ok())
    {
        if (threadIdx.x == 0) atomicAdd(&g_stage_timeouts, 1u);
        return;
    }
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t lane = threadIdx.x & 31u, W = blockDim.x >> 5;
    const size_t   tile0 = (size_t)blockIdx.x * W + (threadIdx.x >> 5), tstride = (size_t)gridDim.x * W;
    const size_t   tiles = (N + 31) / 32;
    const int      ges   = (int)((bo + 7) / 8);
    RegionAStage   S;
    S.init(&sCWmap, n, N, tile0, tstride);
    bool failed = false;
    for (size_t T = tile0; T < tiles && !failed; T += tstride)
    {
        const size_t   i      = T * 32 + lane;
        const bool     active = i < N;
        DcfKeyView<GE> K;
        uint64_t       x = 0, acc = 0;
        uint32_t       s[1][4], t[1] = {party};
        if (active)
        {
            K.set(key, n, 1, i, N);
            x = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
            load_block_be(seed + 16 * i, s[0]);
            s[0][0] &= ~kSeedTBit;
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
                    const uint32_t dir[1] = {(uint32_t)((x >> (n - 1 - lv)) & 1u)};
                    const uint64_t vcw    = (uint64_t)__ldg(K.vCW + lv);
                    const uint32_t tp     = t[0];
                    uint64_t       val;
                    if (sizeof(GE) <= 4 || bo <= 32)
                    {
                        uint32_t v[1][1];
                        dcf_step_g1_cw<1, 1>(A, s, t, dir, cw, K.tl, K.tr, lv, v);
                        val = words_le_prefix<1>(v[0], ges);
                    }
                    else
                    {
                        uint32_t v[1][2];
                        dcf_step_g1_cw<1, 2>(A, s, t, dir, cw, K.tl, K.tr, lv, v);
                        val = words_le_prefix<2>(v[0], ges);
                    }
                    val += tp ? vcw : 0;
                    acc += party ? (0 - val) : val;
                }
            }
            S.next();
        }
        if (failed) break;
        if (active)
        {
            const uint64_t val = block_le_prefix(s[0], ges) + (t[0] ? (uint64_t)__ldg(K.last) : 0);
            acc += party ? (0 - val) : val;
            out[i] = (GE)acc;
        }
    }
    if (failed)
    {
        if (lane == 0) atomicAdd(&g_stage_timeouts, 1u);
        S.drain();
    }
}

// ---------------------------------------------------------------------------------------
// Evaluation, any groupSize: the group vector accumulates in the caller's output.
// ---------------------------------------------------------------------------------------
template <typename GE>
__global__ void __launch_bounds__(kDcfThreads, 1)
    dcf_eval_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                    const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, uint32_t g, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t bstr = sizeof(GE) * ((size_t)n * g + 2 + g);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint8_t *sCWp = key + i * 16 * n;
        const GE      *vCW  = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        const GE      *last = vCW + (size_t)n * g + 2;
        const uint64_t tl = (uint64_t)vCW[(size_t)n * g], tr = (uint64_t)vCW[(size_t)n * g + 1];
        const uint64_t x  = mod_bits<GE>((uint64_t)maskedX[i], n);
        GE            *o  = out + i * g;
        for (uint32_t j = 0; j < g; j++) o[j] = 0;

        uint32_t s[4];
        load_block_be(seed + 16 * i, s);
        s[0] &= ~kSeedTBit;
        uint32_t t = party;
#pragma unroll 1
        for (uint32_t lv = 0; lv < n; lv++)
        {
            uint32_t cw[4];
            load_block_be(sCWp + 16 * lv, cw);
            const uint32_t dir = (uint32_t)((x >> (n - 1 - lv)) & 1u);
            uint32_t       st[2][4];
            {
                const uint32_t sk[1][4] = {{s[0], s[1], s[2], s[3]}}, d1[1] = {dir};
                uint32_t       sn[1][4], vv[1][4];
                aes_prg_pair<1, 4>(A, sk, d1, sn, vv);
#pragma unroll
                for (int c = 0; c < 4; c++) st[0][c] = sn[0][c], st[1][c] = vv[0][c];
            }
            uint32_t       tn = (st[0][0] >> 24) & 1u;
            const uint32_t m  = 0u - t;
            st[0][0] &= ~kSeedTBit;
#pragma unroll
            for (int c = 0; c < 4; c++) s[c] = st[0][c] ^ (cw[c] & m);
            tn ^= (uint32_t)(((dir ? tr : tl) >> lv) & 1u) & t;
            ConvertStream cv;
            cv.init(st[1], g, bo);
            for (uint32_t j = 0; j < g; j++)
            {
                const uint64_t v = cv.value(A, j) + (t ? (uint64_t)vCW[(size_t)lv * g + j] : 0);
                o[j]             = (GE)((uint64_t)o[j] + (party ? (0 - v) : v));
            }
            t = tn;
        }
        ConvertStream cv;
        cv.init(s, g, bo);
        for (uint32_t j = 0; j < g; j++)
        {
            const uint64_t v = cv.value(A, j) + (t ? (uint64_t)last[j] : 0);
            o[j]             = (GE)((uint64_t)o[j] + (party ? (0 - v) : v));
        }
    }
}

static inline size_t dcf_key_bytes(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n + es * n * g + es + es + es * g);
}

static inline size_t dcf_cache_bytes(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n) + N * es * n * g;
}

} // namespace fss

using namespace fss;

// Validation order follows DcfKeyGenTask::check (src/kernel/dcf.h:30-71).
extern "C" FAST_FSS_API int FastFss_cuda_dcfKeyGen(void *key, size_t keyDataSize, const void *alpha,
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
        if (keyDataSize != dcf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (betaDataSize != 0 && betaDataSize != N * es * groupSize) return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        if (seedDataSize0 != N * 16 || seedDataSize1 != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {alpha, beta}, {key, seed0, seed1}); rc != FAST_FSS_SUCCESS) return rc;
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        auto         kern   = dcf_keygen_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, aes_threads(N, kDcfKeygenThreads), 1), aes_threads(N, kDcfKeygenThreads), kAesSmemTotal,
               stream>>>(
            (uint8_t *)key, (const GE *)alpha, (const GE *)beta, (const uint8_t *)seed0, (const uint8_t *)seed1,
            (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, (uint32_t)groupSize, N);
        return launch_status();
    });
}

// Validation order follows DcfEvalTask::check (src/kernel/dcf.h:115-163).
extern "C" FAST_FSS_API int FastFss_cuda_dcfEval(void *sharedOut, size_t sharedOutSize, const void *maskedX,
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
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (groupSize == 0) return FAST_FSS_INVALID_GROUP_SIZE_ERROR;
        if (keyDataSize != dcf_key_bytes(bitWidthIn, groupSize, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (sharedOutSize != N * es * groupSize) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != dcf_cache_bytes(bitWidthIn, groupSize, es, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOut, maskedX}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        if (groupSize == 1)
        {
            CUtensorMap map;
            if (!encode_region_a_map(&map, key, bitWidthIn, N)) return FAST_FSS_RUNTIME_ERROR;
            auto           kern    = dcf_eval_g1_staged_kernel<GE>;
            const int      threads = aes_threads(N, kDcfThreads);
            const unsigned grid    = grid_for(N, threads, 1);
            if (!ensure_smem(reinterpret_cast<const void *>(kern), stage_smem_bytes(kDcfThreads / 32)))
                return FAST_FSS_RUNTIME_ERROR;
            kern<<<grid, threads, stage_smem_bytes(threads / 32), stream>>>(
                (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, N, map);
        }
        else
        {
            auto kern = dcf_eval_kernel<GE>;
            if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
            kern<<<grid_for(N, aes_threads(N, kDcfThreads), 1), aes_threads(N, kDcfThreads), kAesSmemTotal, stream>>>(
                (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, (uint32_t)groupSize, N);
        }
        return launch_status();
    });
}

namespace fss {
unsigned int dpf_stage_failures(); // dpf.cu
}

extern "C" FAST_FSS_API int FastFss_b200_stageTimeouts(unsigned int *count)
{
    if (count == nullptr) return FAST_FSS_RUNTIME_ERROR;
    unsigned int dcf = 0;
    if (cudaMemcpyFromSymbol(&dcf, fss::g_stage_timeouts, sizeof(dcf)) != cudaSuccess) return FAST_FSS_RUNTIME_ERROR;
    const unsigned int dpf = fss::dpf_stage_failures();
    if (dpf == 0xffffffffu) return FAST_FSS_RUNTIME_ERROR;
    *count = dcf + dpf;
    return FAST_FSS_SUCCESS;
}
