// ottt.cu — one-hot truth table (OTTT): key generation and lookup-table evaluation (sm_100a).
//
// Reference behaviour: src/impl/ottt.h:9-192 (algorithm), src/kernel/ottt.h:22-101
// (validation), include/FastFss/cuda/ottt.h (ABI). A key row is 2^n bits. Evaluation:
//   E = number of set bits,  T_k = sum over set bits b of lut[((x - b) mod 2^n) + k 2^n],
// both negated for party 0. No AES: the work is a bit scan plus LUT gathers, so G lanes
// share one element's row (32-bit words when the row is 4-byte aligned) and reduce with
// warp shuffles.
#include <FastFss/cuda/ottt.h>
#include <FastFss/ottt.h>

#include "fss_device.cuh"
#include "fss_host.h"

namespace fss {

constexpr int kOtttThreads = 256;
constexpr int kOtttLMax    = 4;

template <typename GE>
__global__ void ottt_keygen_kernel(uint8_t *__restrict__ key, const GE *__restrict__ alpha, uint32_t n, size_t N)
{
    const size_t rowBytes = ((size_t)1 << n) / 8;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint64_t a = mod_bits<GE>((uint64_t)alpha[i], n);
        key[i * rowBytes + a / 8] ^= (uint8_t)(1u << (a % 8));
    }
}

template <typename GE, bool WORDS>
__global__ void __launch_bounds__(kOtttThreads)
    ottt_eval_kernel(GE *__restrict__ outE, GE *__restrict__ outT, const GE *__restrict__ maskedX,
                     const uint8_t *__restrict__ key, uint32_t party, const GE *__restrict__ lut, uint32_t lutNum,
                     uint32_t n, size_t N, uint32_t G, uint32_t j0)
{
    const size_t   dom      = (size_t)1 << n;
    const size_t   mask     = dom - 1;
    const size_t   rowBytes = dom / 8;
    const size_t   units    = WORDS ? rowBytes / 4 : rowBytes;
    const size_t   work     = ((N * G + 31) / 32) * 32;
    const uint32_t lg       = threadIdx.x % G;
    const uint32_t jcnt     = lutNum > j0 ? min((uint32_t)kOtttLMax, lutNum - j0) : 0u;
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
    {
        const size_t i      = w / G;
        const bool   active = i < N;
        uint64_t     E = 0, T[kOtttLMax];
#pragma unroll
        for (int k = 0; k < kOtttLMax; k++) T[k] = 0;
        if (active)
        {
            const size_t   x   = (size_t)(uint64_t)__ldg(maskedX + i);
            const uint8_t *row = key + i * rowBytes;
            for (size_t u = lg; u < units; u += G)
            {
                uint32_t bits = WORDS ? __ldg(reinterpret_cast<const uint32_t *>(row) + u) : (uint32_t)__ldg(row + u);
                const size_t base = u * (WORDS ? 32 : 8);
                E += (uint64_t)__popc(bits);
                while (bits)
                {
                    const uint32_t b   = (uint32_t)__ffs(bits) - 1;
                    bits &= bits - 1;
                    const size_t idx = (x - (base + b)) & mask;
#pragma unroll
                    for (int k = 0; k < kOtttLMax; k++)
                        if ((uint32_t)k < jcnt) T[k] += (uint64_t)__ldg(lut + idx + (size_t)(j0 + k) * dom);
                }
            }
        }
        for (uint32_t off = G >> 1; off > 0; off >>= 1)
        {
            E += __shfl_xor_sync(0xffffffffu, E, off);
#pragma unroll
            for (int k = 0; k < kOtttLMax; k++) T[k] += __shfl_xor_sync(0xffffffffu, T[k], off);
        }
        if (active && lg == 0)
        {
            if (party == 0)
            {
                E = 0 - E;
#pragma unroll
                for (int k = 0; k < kOtttLMax; k++) T[k] = 0 - T[k];
            }
            if (j0 == 0) outE[i] = (GE)E;
#pragma unroll
            for (int k = 0; k < kOtttLMax; k++)
                if ((uint32_t)k < jcnt) outT[i * lutNum + j0 + k] = (GE)T[k];
        }
    }
}

} // namespace fss

using namespace fss;

// Validation order: OtttKeyGenTask::check (src/kernel/ottt.h:22-37).
extern "C" FAST_FSS_API int FastFss_cuda_otttKeyGen(void *key, size_t keyDataSize, const void *alpha,
                                                    size_t alphaDataSize, size_t bitWidthIn, size_t elementSize,
                                                    size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(3 <= n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (n >= 64 || keyDataSize != N * (((size_t)1 << n) / 8)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {alpha}, {}); rc != FAST_FSS_SUCCESS) return rc;
        ottt_keygen_kernel<GE><<<grid_for(N, 256, 8), 256, 0, resolve_stream(cudaStreamPtr)>>>(
            (uint8_t *)key, (const GE *)alpha, (uint32_t)n, N);
        return launch_status();
    });
}

// Validation order: OtttLutEvalTask::check (src/kernel/ottt.h:67-101).
extern "C" FAST_FSS_API int FastFss_cuda_otttLutEval(void *sharedOutE, size_t sharedOutEDataSize, void *sharedOutT,
                                                     size_t sharedOutTDataSize, const void *maskedX,
                                                     size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                     int partyId, const void *lookUpTable, size_t lookUpTableDataSize,
                                                     size_t bitWidthIn, size_t elementSize, size_t elementNum,
                                                     void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, n = bitWidthIn;
        if (!(3 <= n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (n >= 64 || keyDataSize != N * (((size_t)1 << n) / 8)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        const size_t each = es * ((size_t)1 << n);
        if (lookUpTableDataSize % each != 0) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        const size_t lutNum = lookUpTableDataSize / each;
        if (sharedOutEDataSize != N * es) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (sharedOutTDataSize != N * es * lutNum) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOutE, sharedOutT, maskedX, lookUpTable}, {}); rc != FAST_FSS_SUCCESS) return rc;
        const size_t rowBytes = ((size_t)1 << n) / 8;
        const bool   words    = (rowBytes % 4 == 0) && (((uintptr_t)key & 3u) == 0);
        const size_t units    = words ? rowBytes / 4 : rowBytes;
        uint32_t     G        = 1;
        while (G < 32 && G < units) G <<= 1;
        cudaStream_t stream = resolve_stream(cudaStreamPtr);
        for (size_t j0 = 0; j0 < (lutNum ? lutNum : 1); j0 += kOtttLMax)
        {
            auto kern = words ? ottt_eval_kernel<GE, true> : ottt_eval_kernel<GE, false>;
            kern<<<grid_for(N * G, kOtttThreads, 8), kOtttThreads, 0, stream>>>(
                (GE *)sharedOutE, (GE *)sharedOutT, (const GE *)maskedX, (const uint8_t *)key, (uint32_t)partyId,
                (const GE *)lookUpTable, (uint32_t)lutNum, (uint32_t)n, N, G, (uint32_t)j0);
            if (launch_status() != FAST_FSS_SUCCESS) return FAST_FSS_RUNTIME_ERROR;
        }
        return FAST_FSS_SUCCESS;
    });
}
