// mic.cu — DCF-based multiple interval containment (sm_100a).
//
// Reference behaviour: src/impl/mic.h:9-109 (algorithm), src/kernel/mic.h:33-162
// (validation), include/FastFss/cuda/mic.h (ABI). The key is a DCF key with groupSize 1
// for alpha - 1 and beta = 1; z[i][q] is public per-interval correction data.
//
// Evaluation: interval q needs sp = DCF(x - 1 - L_q) and sq = DCF(x - 1 - (R_q + 1)). When the
// intervals touch, sq of interval q - 1 is sp of interval q (the reference reuses it in its
// per-element loop); here each point is walked once by its own thread and the intervals are
// formed from neighbouring points after a barrier. Intervals that do not touch are evaluated
// one thread per (element, interval), both walks side by side.
#include <FastFss/cuda/mic.h>
#include <FastFss/mic.h>

#include "dcf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "mic_core.cuh"

namespace fss {

constexpr int kMicThreads = 512;

template <typename GE>
__global__ void __launch_bounds__(kMicThreads, 1)
    mic_keygen_kernel(uint8_t *__restrict__ key, GE *__restrict__ z, const GE *__restrict__ alpha,
                      const uint8_t *__restrict__ seed0, const uint8_t *__restrict__ seed1,
                      const GE *__restrict__ left, const GE *__restrict__ right, uint32_t m, uint32_t n, uint32_t bo,
                      size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint64_t a = (uint64_t)alpha[i];
        dcf_keygen_element<GE>(A, key, N, i, (uint64_t)(GE)(a - 1), nullptr, seed0 + 16 * i, seed1 + 16 * i, n, bo,
                               1);
        // z[i] = (aP > aQ) - (aP > p) + (aQ' > q') + (aQ == 2^n - 1)  (src/impl/mic.h:24-40)
        const uint64_t MAX = mod_bits<GE>((uint64_t)(GE)~0ull, n);
        for (uint32_t q = 0; q < m; q++)
        {
            const uint64_t L = (uint64_t)left[q], R = (uint64_t)right[q];
            const uint64_t qP  = mod_bits<GE>((uint64_t)(GE)(R + 1), n);
            const uint64_t aP  = mod_bits<GE>((uint64_t)(GE)(L + a), n);
            const uint64_t aQ  = mod_bits<GE>((uint64_t)(GE)(R + a), n);
            const uint64_t aQP = mod_bits<GE>((uint64_t)(GE)(R + 1 + a), n);
            const uint64_t p   = mod_bits<GE>(L, n);
            const int64_t  v   = (int64_t)(aP > aQ) - (int64_t)(aP > p) + (int64_t)(aQP > qP) + (int64_t)(aQ == MAX);
            z[i * m + q]       = (GE)(uint64_t)v;
        }
    }
}

// Touching intervals share endpoint walks, as the reference's own loop does when it reuses sq
// of interval q - 1 as sp of interval q (src/impl/mic.h:60-105): a CTA takes E = blockDim / P
// elements at a time, thread t walks point t % P of element t / P into shared memory, and after
// a barrier thread t writes interval t % m of element t / m from the two points around it.
// Otherwise one thread per (element, interval) walks both endpoints (mic_eval_item).
template <typename GE>
__global__ void __launch_bounds__(kMicThreads, 1)
    mic_eval_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                    const GE *__restrict__ z, const uint8_t *__restrict__ seed, uint32_t party,
                    const GE *__restrict__ left, const GE *__restrict__ right, uint32_t m, uint32_t n, uint32_t bo,
                    size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    uint64_t *shares = reinterpret_cast<uint64_t *>(fss_smem + kAesSmemTotal); // blockDim entries
    uint32_t *points = reinterpret_cast<uint32_t *>(shares + blockDim.x);
    if (threadIdx.x == 0) *points = mic_points<GE>(left, right, m, n);
    __syncthreads();
    const uint32_t P = *points;
    if (P == 0 || P > blockDim.x)
    {
        const size_t work = N * m;
        for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
            out[w] = mic_eval_item<GE>(A, maskedX, key, z, seed, party, left, right, m, n, bo, N, w);
        return;
    }
    const uint32_t E = blockDim.x / P;
    for (size_t base = (size_t)blockIdx.x * E; base < N; base += (size_t)gridDim.x * E)
        mic_shared_batch<GE>(A, shares, out, maskedX, key, z, seed, party, left, right, m, n, bo, N, P, base, N, 0,
                             (unsigned long long)N * m);
}

static inline size_t dcf_key_bytes_g1(size_t n, size_t es, size_t N)
{
    return N * (16 * n + es * n + 3 * es);
}

} // namespace fss

using namespace fss;

// Validation order: DcfMICKeyGenTask::check (src/kernel/mic.h:33-68).
extern "C" FAST_FSS_API int FastFss_cuda_dcfMICKeyGen(void *key, size_t keyDataSize, void *z, size_t zDataSize,
                                                      const void *alpha, size_t alphaDataSize, const void *seed0,
                                                      size_t seedDataSize0, const void *seed1, size_t seedDataSize1,
                                                      const void *leftEndpoints, size_t leftEndpointsDataSize,
                                                      const void *rightEndpoints, size_t rightEndpointsDataSize,
                                                      size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                      size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, m = leftEndpointsDataSize / es;
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (keyDataSize != dcf_key_bytes_g1(bitWidthIn, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (zDataSize != N * es * m) return FAST_FSS_INVALID_Z_DATA_SIZE_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (seedDataSize0 != N * 16 || seedDataSize1 != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (leftEndpointsDataSize != m * es || rightEndpointsDataSize != m * es)
            return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {z, alpha, leftEndpoints, rightEndpoints}, {key, seed0, seed1}); rc != FAST_FSS_SUCCESS) return rc;
        auto kern = mic_keygen_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, aes_threads(N, kMicThreads), 1), aes_threads(N, kMicThreads), kAesSmemTotal, resolve_stream(cudaStreamPtr)>>>(
            (uint8_t *)key, (GE *)z, (const GE *)alpha, (const uint8_t *)seed0, (const uint8_t *)seed1,
            (const GE *)leftEndpoints, (const GE *)rightEndpoints, (uint32_t)m, (uint32_t)bitWidthIn,
            (uint32_t)bitWidthOut, N);
        return launch_status();
    });
}

// Validation order: DcfMICEvalTask::check (src/kernel/mic.h:114-162).
extern "C" FAST_FSS_API int FastFss_cuda_dcfMICEval(void *sharedOut, size_t sharedOutDataSize, const void *maskedX,
                                                    size_t maskedXDataSize, const void *key, size_t keyDataSize,
                                                    const void *sharedZ, size_t sharedZDataSize, const void *seed,
                                                    size_t seedDataSize, int partyId, const void *leftEndpoints,
                                                    size_t leftEndpointsDataSize, const void *rightEndpoints,
                                                    size_t rightEndpointsDataSize, size_t bitWidthIn,
                                                    size_t bitWidthOut, size_t elementSize, size_t elementNum,
                                                    void *cache, size_t cacheDataSize, void *cudaStreamPtr)
{
    (void)cache;
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, m = leftEndpointsDataSize / es, n = bitWidthIn;
        if (!(0 < n && n <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (keyDataSize != dcf_key_bytes_g1(n, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (sharedOutDataSize != N * es * m) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (sharedZDataSize != N * es * m) return FAST_FSS_INVALID_Z_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (leftEndpointsDataSize != m * es || rightEndpointsDataSize != m * es)
            return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (cacheDataSize != 0 && cacheDataSize != N * 16 * n + N * es * n) return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        if (N == 0 || m == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOut, maskedX, sharedZ, leftEndpoints, rightEndpoints}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        auto kern = mic_eval_kernel<GE>;
        // tables, then one share per thread and the point count (mic_eval_kernel)
        constexpr int smem = kAesSmemTotal + kMicThreads * 8 + 16;
        if (!ensure_smem(reinterpret_cast<const void *>(kern), smem)) return FAST_FSS_RUNTIME_ERROR;
        const int threads = aes_threads(N * m, kMicThreads);
        kern<<<grid_for(N * m, threads, 1), threads, kAesSmemTotal + threads * 8 + 16, resolve_stream(cudaStreamPtr)>>>(
            (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const GE *)sharedZ, (const uint8_t *)seed,
            (uint32_t)partyId, (const GE *)leftEndpoints, (const GE *)rightEndpoints, (uint32_t)m, (uint32_t)n,
            (uint32_t)bitWidthOut, N);
        return launch_status();
    });
}
