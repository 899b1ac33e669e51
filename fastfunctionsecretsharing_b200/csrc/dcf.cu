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

#include "fss_device.cuh"
#include "fss_host.h"

namespace fss {

constexpr int kDcfThreads = 512;

// ---------------------------------------------------------------------------------------
// Key generation (src/impl/dcf.h:187-368). vAlpha is accumulated in the lastCW slots, as
// the reference does.
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
    const size_t bstr = sizeof(GE) * ((size_t)n * g + 2 + g);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        uint8_t *sCWp = key + i * 16 * n;
        GE      *vCW  = reinterpret_cast<GE *>(key + N * 16 * n + i * bstr);
        GE      *tLp  = vCW + (size_t)n * g;
        GE      *last = tLp + 2;
        for (uint32_t j = 0; j < g; j++) last[j] = 0;

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
            uint32_t G0[4][4], G1[4][4];
#pragma unroll
            for (int b = 0; b < 4; b++) prg_block(G0[b], b), prg_block(G1[b], b);
            aes_encrypt<4>(A, s0, G0);
            aes_encrypt<4>(A, s1, G1);
            const uint32_t tL0 = (G0[0][0] >> 24) & 1u, tR0 = (G0[2][0] >> 24) & 1u;
            const uint32_t tL1 = (G1[0][0] >> 24) & 1u, tR1 = (G1[2][0] >> 24) & 1u;
            G0[0][0] &= ~kSeedTBit, G0[2][0] &= ~kSeedTBit, G1[0][0] &= ~kSeedTBit, G1[2][0] &= ~kSeedTBit;

            const uint32_t keep = (uint32_t)((a >> (n - 1 - lv)) & 1u);
            // keep = R (1): lose = L = blocks 0/1, keep blocks 2/3; keep = L (0): the reverse.
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
                    const uint64_t b = beta ? (uint64_t)beta[i * g + j] : (uint64_t)(j == 0);
                    v += t1 ? (0 - b) : b;
                }
                vCW[(size_t)lv * g + j] = (GE)v;
                va                      = va - cK1.value(A, j) + cK0.value(A, j) + (t1 ? (0 - v) : v);
                last[j]                 = (GE)va;
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
}

// ---------------------------------------------------------------------------------------
// Evaluation, groupSize == 1 (the hot path): accumulator, seed and control bit in registers.
// ---------------------------------------------------------------------------------------
template <typename GE>
__global__ void __launch_bounds__(kDcfThreads, 1)
    dcf_eval_g1_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                       const uint8_t *__restrict__ seed, uint32_t party, uint32_t n, uint32_t bo, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const int    ges  = (int)((bo + 7) / 8);
    const size_t bstr = sizeof(GE) * ((size_t)n + 3);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint8_t *sCWp = key + i * 16 * n;
        const GE      *kb   = reinterpret_cast<const GE *>(key + N * 16 * n + i * bstr);
        const uint64_t tl = (uint64_t)__ldg(kb + n), tr = (uint64_t)__ldg(kb + n + 1);
        const uint64_t x  = mod_bits<GE>((uint64_t)__ldg(maskedX + i), n);

        uint32_t s[4];
        load_block_be(seed + 16 * i, s);
        s[0] &= ~kSeedTBit;
        uint32_t t   = party;
        uint64_t acc = 0;
#pragma unroll 1
        for (uint32_t lv = 0; lv < n; lv++)
        {
            uint32_t cw[4];
            load_block_be(sCWp + 16 * lv, cw);
            const uint64_t vcw = (uint64_t)__ldg(kb + lv);
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
            const uint64_t v = block_le_prefix(st[1], ges) + (t ? vcw : 0);
            acc += party ? (0 - v) : v;
            t = tn;
        }
        const uint64_t v = block_le_prefix(s, ges) + (t ? (uint64_t)__ldg(kb + n + 2) : 0);
        acc += party ? (0 - v) : v;
        out[i] = (GE)acc;
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
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        auto         kern   = dcf_keygen_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, kDcfThreads, 1), kDcfThreads, kAesSmemTotal, stream>>>(
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
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        if (groupSize == 1)
        {
            auto kern = dcf_eval_g1_kernel<GE>;
            if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
            kern<<<grid_for(N, kDcfThreads, 1), kDcfThreads, kAesSmemTotal, stream>>>(
                (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, N);
        }
        else
        {
            auto kern = dcf_eval_kernel<GE>;
            if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
            kern<<<grid_for(N, kDcfThreads, 1), kDcfThreads, kAesSmemTotal, stream>>>(
                (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const uint8_t *)seed, (uint32_t)partyId,
                (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, (uint32_t)groupSize, N);
        }
        return launch_status();
    });
}
