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
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "dcf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "stage.cuh"

namespace fss {

constexpr int kDcfThreads = 512;

// Key staging of the groupSize-1 evaluation: a warp evaluates 32 consecutive elements at a
// time and brings their per-level correction words (region A: one 16n-byte row of 16-byte
// words per element) into its own shared-memory stage, kStageLevels levels at a time, with one
// TMA copy of a 64-byte x 32-row box of a 2-D tensor map over region A; double buffered, so the
// next levels arrive while these are evaluated, and the walk reads them with conflict-free
// 16-byte shared loads instead of 32 scattered global loads per warp and level. The copy uses
// the 64-byte swizzle (16-byte chunk k of row r lands in chunk k ^ ((r >> 1) & 3)), which makes
// the 8 rows of a load phase hit 8 different bank groups.
constexpr int kStageLevels    = 4;
constexpr int kStageRowBytes  = 16 * kStageLevels;        // 64: the swizzle span
constexpr int kStageBytes     = 32 * kStageRowBytes;      // 2048 per stage
constexpr int kStageBase      = (kAesSmemTotal + 1023) / 1024 * 1024; // stages 1024-byte aligned
constexpr int kWarpStageBytes = 2 * kStageBytes;
// dynamic shared memory of a CTA of `warps` warps: tables, stages, then 2 mbarriers per warp
constexpr int stage_smem_bytes(int warps)
{
    return kStageBase + warps * kWarpStageBytes + warps * 16;
}

// Staging failures (FastFss_b200_stageTimeouts): a wait for a copy that ran out, or a launch
// whose shared window could not hold aligned stages. Zero in normal operation.
__device__ unsigned int g_stage_timeouts;

// ---------------------------------------------------------------------------------------
// Key generation (src/impl/dcf.h:187-368): one element per thread.
// ---------------------------------------------------------------------------------------
template <typename GE>
__global__ void __launch_bounds__(kDcfThreads, 1)
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
// through shared memory by bulk copies (the entry point refuses keys that are not 16-byte
// aligned). Every mbarrier wait is bounded:
// a warp whose copy does not complete in time counts the event in g_stage_timeouts, drains its
// other copies (bounded) and stops; its remaining shares are not written.
template <typename GE>
__global__ void __launch_bounds__(kDcfThreads, 1)
    dcf_eval_g1_staged_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                              const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, size_t N,
                              const __grid_constant__ CUtensorMap sCWmap)
{
    // The swizzled copies need 1024-byte aligned stages; should the dynamic shared window ever
    // start elsewhere, record it and write nothing rather than issue a misaligned copy.
    if ((smem_u32(fss_smem + kStageBase) & 1023u) != 0)
    {
        if (threadIdx.x == 0) atomicAdd(&g_stage_timeouts, 1u);
        return;
    }
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
    uint8_t       *ws    = fss_smem + kStageBase + (size_t)warp * kWarpStageBytes;
    const uint32_t st0   = smem_u32(ws);
    const uint32_t bar0  = smem_u32(fss_smem + kStageBase + (size_t)W * kWarpStageBytes + 16 * warp);
    const uint32_t swz   = 16u * ((lane >> 1) & 3u); // xor of this lane's row within a stage
    if (lane == 0)
    {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncwarp();

    const size_t   tiles = (N + 31) / 32;
    const size_t   tile0 = (size_t)blockIdx.x * W + warp, tstride = (size_t)gridDim.x * W;
    const uint32_t C     = (n + kStageLevels - 1) / kStageLevels; // chunks per tile
    // Copies are issued in the order they are consumed: chunk c (levels c * L ...) of tile T,
    // then the next chunk, moving to tile T + tstride after the last chunk of a tile. The issue
    // position (iT, ic) runs two chunks ahead of the evaluation; stage b alternates per chunk.
    size_t   iT = tile0;
    uint32_t ic = 0, ib = 0;
    auto     issue = [&]() {
        if (iT >= tiles) return; // warp-uniform
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
        {
            // the whole box counts, rows past N and levels past n included (zero filled)
            mbar_arrive_expect_tx(bar0 + 8 * ib, kStageBytes);
            tensor_copy_2d_g2s(st0 + ib * kStageBytes, &sCWmap, (int32_t)(ic * kStageRowBytes), (int32_t)(iT * 32),
                               bar0 + 8 * ib);
        }
        ib ^= 1u;
        if (++ic == C)
        {
            ic = 0;
            iT += tstride;
        }
    };

    uint32_t parity = 0; // bit b: parity of stage b's next phase
    bool     failed    = false;
    uint32_t b = 0; // stage of the chunk being evaluated
    issue();
    issue();
    for (size_t T = tile0; T < tiles && !failed; T += tstride)
    {
        const size_t   i      = T * 32 + lane;
        const bool     active = i < N;
        DcfKeyView<GE> K;
        uint64_t       x = 0;
        if (active)
        {
            K.set(key, n, 1, i, N);
            x = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);
        }
        const int ges = (int)((bo + 7) / 8);
        uint32_t  s[1][4], t[1] = {party};
        if (active)
        {
            load_block_be(seed + 16 * i, s[0]);
            s[0][0] &= ~kSeedTBit;
        }
        uint64_t acc = 0;
        for (uint32_t c = 0; c < C; c++, b ^= 1u)
        {
            if (!mbar_wait_bounded(bar0 + 8 * b, (parity >> b) & 1u))
            {
                failed = true;
                break;
            }
            parity ^= 1u << b;
            if (active)
            {
                const uint8_t *cwp = ws + b * kStageBytes + lane * kStageRowBytes;
                const uint32_t lv0 = c * kStageLevels, lc = min((uint32_t)kStageLevels, n - lv0);
#pragma unroll 1
                for (uint32_t j = 0; j < lc; j++)
                {
                    const uint32_t lv  = lv0 + j;
                    const uint4    raw = *reinterpret_cast<const uint4 *>(cwp + ((16 * j) ^ swz));
                    const uint32_t cw[4] = {bswap32(raw.x), bswap32(raw.y), bswap32(raw.z), bswap32(raw.w)};
                    const uint32_t dir[1] = {(uint32_t)((x >> (n - 1 - lv)) & 1u)};
                    const uint64_t vcw    = (uint64_t)__ldg(K.vCW + lv);
                    const uint32_t tp     = t[0];
                    uint32_t       v[1][1];
                    if (sizeof(GE) <= 4 || bo <= 32)
                    {
                        dcf_step_g1_cw<1, 1>(A, s, t, dir, cw, K.tl, K.tr, lv, v);
                        const uint64_t val = words_le_prefix<1>(v[0], ges) + (tp ? vcw : 0);
                        acc += party ? (0 - val) : val;
                    }
                    else
                    {
                        uint32_t v2[1][2];
                        dcf_step_g1_cw<1, 2>(A, s, t, dir, cw, K.tl, K.tr, lv, v2);
                        const uint64_t val = words_le_prefix<2>(v2[0], ges) + (tp ? vcw : 0);
                        acc += party ? (0 - val) : val;
                    }
                }
            }
            issue(); // the stage just read is refilled two chunks ahead
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
        // copies of this warp still in flight land in its own stages: wait for them (bounded)
        mbar_wait_bounded(bar0, parity & 1u);
        mbar_wait_bounded(bar0 + 8, (parity >> 1) & 1u);
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
            prg_block(st[0], 2 * dir);
            prg_block(st[1], 2 * dir + 1);
            aes_encrypt<2>(A, s, st);
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

// Tensor map over region A of a DCF key: rows = elements (16 n bytes each), x in bytes; boxes of
// kStageRowBytes x 32 rows, 64-byte swizzle. The driver's encoder is looked up once.
static bool encode_scw_map(CUtensorMap *map, const void *key, size_t n, size_t N)
{
    static std::once_flag                    once;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    std::call_once(once, [] {
        void                            *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        else
            cudaGetLastError();
    });
    if (encode == nullptr || N >= (1ull << 32)) return false;
    const cuuint64_t dims[2]    = {(cuuint64_t)(16 * n), (cuuint64_t)N};
    const cuuint64_t strides[1] = {(cuuint64_t)(16 * n)};
    const cuuint32_t box[2]     = {(cuuint32_t)kStageRowBytes, 32u};
    const cuuint32_t estr[2]    = {1u, 1u};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(key), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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
        kern<<<grid_for(N, aes_threads(N, kDcfThreads), 1), aes_threads(N, kDcfThreads), kAesSmemTotal, stream>>>(
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
            if (!encode_scw_map(&map, key, bitWidthIn, N)) return FAST_FSS_RUNTIME_ERROR;
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

extern "C" FAST_FSS_API int FastFss_b200_stageTimeouts(unsigned int *count)
{
    if (count == nullptr) return FAST_FSS_RUNTIME_ERROR;
    return cudaMemcpyFromSymbol(count, fss::g_stage_timeouts, sizeof(unsigned int)) == cudaSuccess
               ? FAST_FSS_SUCCESS
               : FAST_FSS_RUNTIME_ERROR;
}
