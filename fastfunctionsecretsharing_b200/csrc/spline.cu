// spline.cu — DCF-based piecewise-polynomial (spline) key generation and evaluation (sm_100a).
//
// Reference behaviour: src/impl/spline.h:89-253 (algorithm), src/kernel/spline.h:39-207
// (validation), include/FastFss/cuda/spline.h (ABI). The key is a vector DCF key with
// groupSize g = m (d + 1) for alpha - 1 whose payload beta holds every interval's
// polynomial shifted by alpha; e = correction * beta.
//
// Evaluation. The reference evaluates the full g-vector DCF at every endpoint and then uses
// only interval q's d + 1 values of it (src/impl/spline.h:226-249). Here each interval is
// handled by its own lane of a G-lane group, which walks the two DCF paths of interval q
// (x - 1 - L_q and x - 1 - (R_q + 1)) and reads only slot q's values out of each level's
// convert stream: the AES-CTR blocks holding slot q are produced under one extra key schedule
// per level (not all ceil(ges g / 16) blocks of the stream).
// Coefficient sums are reduced across the group with warp shuffles and lane 0 evaluates the
// polynomial. Shares are bit-identical to the reference; nothing is written to the cache.
#include <FastFss/cuda/spline.h>
#include <FastFss/spline.h>

#include "dcf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "spline_core.cuh"

namespace fss {

constexpr int kSplineThreads     = 256; // key generation
constexpr int kSplineEvalThreads = 256; // evaluation: 8 warps per SM, registers unconstrained

// splineShiftPolynomialCoefficients (src/impl/spline.h:89-117), writing d + 1 values.
template <typename GE>
__device__ __forceinline__ void spline_shift(GE *out, const GE *coeffs, uint64_t shift, uint32_t d, uint32_t bo)
{
    const uint64_t negShift = mod_bits<GE>((uint64_t)(GE)(0 - shift), bo);
    for (uint32_t i = 0; i <= d; i++) out[i] = 0;
    for (uint32_t i = d + 1; i > 0; --i)
    {
        const uint64_t c = (uint64_t)coeffs[i - 1];
        for (uint32_t j = d; j > 0; --j) out[j] = (GE)((uint64_t)out[j - 1] + (uint64_t)out[j] * negShift);
        out[0] = (GE)((uint64_t)out[0] * negShift + c);
    }
    for (uint32_t i = 0; i <= d; i++) out[i] = (GE)mod_bits<GE>((uint64_t)out[i], bo);
}

template <typename GE>
__global__ void __launch_bounds__(kSplineThreads, 1)
    spline_keygen_kernel(uint8_t *__restrict__ key, GE *__restrict__ e, GE *__restrict__ beta,
                         const GE *__restrict__ alpha, const uint8_t *__restrict__ seed0,
                         const uint8_t *__restrict__ seed1, const GE *__restrict__ coeffs, uint32_t d,
                         const GE *__restrict__ left, const GE *__restrict__ right, uint32_t m, uint32_t n,
                         uint32_t bo, size_t N)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const uint32_t cn = d + 1, g = m * cn;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint64_t a  = (uint64_t)alpha[i];
        GE            *bi = beta + i * g;
        for (uint32_t q = 0; q < m; q++) spline_shift<GE>(bi + q * cn, coeffs + (size_t)q * cn, a, d, bo);
        dcf_keygen_element<GE>(A, key, N, i, (uint64_t)(GE)(a - 1), bi, seed0 + 16 * i, seed1 + 16 * i, n, bo, g);
        const uint64_t maxValue = mod_bits<GE>((uint64_t)(GE)~0ull, n);
        for (uint32_t q = 0; q < m; q++)
        {
            const uint64_t L   = mod_bits<GE>((uint64_t)left[q], n);
            const uint64_t R   = mod_bits<GE>((uint64_t)right[q], n);
            const uint64_t Rp  = mod_bits<GE>((uint64_t)(GE)(R + 1), n);
            const uint64_t aL  = mod_bits<GE>((uint64_t)(GE)(L + a), n);
            const uint64_t aR  = mod_bits<GE>((uint64_t)(GE)(R + a), n);
            const uint64_t aRp = mod_bits<GE>((uint64_t)(GE)(Rp + a), n);
            const uint64_t corr =
                (uint64_t)((int64_t)(aL > aR) - (int64_t)(aL > L) + (int64_t)(aRp > Rp) + (int64_t)(aR == maxValue));
            for (uint32_t j = 0; j < cn; j++)
                e[i * g + q * cn + j] = (GE)mod_bits<GE>((uint64_t)(GE)(corr * (uint64_t)bi[q * cn + j]), bo);
        }
    }
}

template <typename GE>
__global__ void __launch_bounds__(kSplineEvalThreads, 1)
    spline_eval_kernel(GE *__restrict__ out, const GE *__restrict__ maskedX, const uint8_t *__restrict__ key,
                       const GE *__restrict__ sharedE, const GE *__restrict__ sharedBeta,
                       const uint8_t *__restrict__ seed, uint32_t party, const GE *__restrict__ left,
                       const GE *__restrict__ right, uint32_t m, uint32_t d, uint32_t n, uint32_t bo, size_t N,
                       uint32_t G)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    const size_t work = ((N * G + 31) / 32) * 32; // whole warps stay in the loop (shuffles)
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < work; w += (size_t)gridDim.x * blockDim.x)
        spline_eval_group<GE>(A, out, maskedX, key, sharedE, sharedBeta, seed, party, left, right, m, d, n, bo, N, G,
                              w / G, (uint32_t)(w % G), w / G < N);
}

static inline size_t dcf_key_bytes(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n + es * n * g + es + es + es * g);
}

static inline size_t spline_cache_bytes(size_t n, size_t m, size_t d, size_t es, size_t N)
{
    const size_t g = m * (d + 1);
    return N * 16 * n + N * es * n * g + N * es * (2 * g + d + 1);
}

} // namespace fss

using namespace fss;

// Validation order: DcfSplineKeyGenTask::check (src/kernel/spline.h:39-91).
extern "C" FAST_FSS_API int FastFss_cuda_dcfSplineKeyGen(
    void *key, size_t keyDataSize, void *e, size_t eDataSize, void *beta, size_t betaDataSize, const void *alpha,
    size_t alphaDataSize, const void *seed0, size_t seedDataSize0, const void *seed1, size_t seedDataSize1,
    const void *coefficients, size_t coefficientsDataSize, size_t degree, const void *leftEndpoints,
    size_t leftEndpointsDataSize, const void *rightEndpoints, size_t rightEndpointsDataSize, size_t intervalNum,
    size_t bitWidthIn, size_t bitWidthOut, size_t elementSize, size_t elementNum, void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, m = intervalNum, g = m * (degree + 1);
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (m == 0) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (keyDataSize != dcf_key_bytes(bitWidthIn, g, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (eDataSize != N * es * g) return FAST_FSS_INVALID_Z_DATA_SIZE_ERROR;
        if (betaDataSize != N * es * g) return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        if (alphaDataSize != N * es) return FAST_FSS_INVALID_ALPHA_DATA_SIZE_ERROR;
        if (seedDataSize0 != N * 16 || seedDataSize1 != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (leftEndpointsDataSize != m * es) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (rightEndpointsDataSize != m * es) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (coefficientsDataSize != m * (degree + 1) * es) return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {e, beta, alpha, coefficients, leftEndpoints, rightEndpoints}, {key, seed0, seed1}); rc != FAST_FSS_SUCCESS) return rc;
        auto kern = spline_keygen_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N, aes_threads(N, kSplineThreads), 1), aes_threads(N, kSplineThreads), kAesSmemTotal,
                 resolve_stream(cudaStreamPtr)>>>(
            (uint8_t *)key, (GE *)e, (GE *)beta, (const GE *)alpha, (const uint8_t *)seed0, (const uint8_t *)seed1,
            (const GE *)coefficients, (uint32_t)degree, (const GE *)leftEndpoints, (const GE *)rightEndpoints,
            (uint32_t)m, (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, N);
        return launch_status();
    });
}

// Validation order: DcfSplineEvalTask::check (src/kernel/spline.h:145-207); the cache must
// be present and of the reference's size, although it is not used.
extern "C" FAST_FSS_API int FastFss_cuda_dcfSplineEval(
    void *sharedOut, size_t sharedOutDataSize, const void *maskedX, size_t maskedXDataSize, const void *key,
    size_t keyDataSize, const void *sharedE, size_t sharedEDataSize, const void *sharedBeta, size_t sharedBetaDataSize,
    const void *seed, size_t seedDataSize, int partyId, const void *leftEndpoints, size_t leftEndpointsDataSize,
    const void *rightEndpoints, size_t rightEndpointsDataSize, size_t intervalNum, size_t degree, size_t bitWidthIn,
    size_t bitWidthOut, size_t elementSize, size_t elementNum, void *cache, size_t cacheDataSize,
    void *cudaStreamPtr)
{
    return dispatch_es(elementSize, [&](auto tag) -> int {
        using GE        = decltype(tag);
        const size_t es = sizeof(GE), N = elementNum, m = intervalNum, g = m * (degree + 1);
        if (!(0 < bitWidthIn && bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (!(0 < bitWidthOut && bitWidthOut <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
        if (partyId != 0 && partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
        if (m == 0) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (keyDataSize != dcf_key_bytes(bitWidthIn, g, es, N)) return FAST_FSS_INVALID_KEY_DATA_SIZE_ERROR;
        if (sharedOutDataSize != N * es) return FAST_FSS_INVALID_SHARED_OUT_DATA_SIZE_ERROR;
        if (maskedXDataSize != N * es) return FAST_FSS_INVALID_MASKED_X_DATA_SIZE_ERROR;
        if (sharedEDataSize != N * es * g) return FAST_FSS_INVALID_Z_DATA_SIZE_ERROR;
        if (sharedBetaDataSize != N * es * g) return FAST_FSS_INVALID_BETA_DATA_SIZE_ERROR;
        if (seedDataSize != N * 16) return FAST_FSS_INVALID_SEED_DATA_SIZE_ERROR;
        if (leftEndpointsDataSize != m * es) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (rightEndpointsDataSize != m * es) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
        if (cache == nullptr || cacheDataSize != spline_cache_bytes(bitWidthIn, m, degree, es, N))
            return FAST_FSS_INVALID_CACHE_DATA_SIZE_ERROR;
        if (N == 0) return FAST_FSS_SUCCESS;
        if (int rc = check_alignment(es, {sharedOut, maskedX, sharedE, sharedBeta, leftEndpoints, rightEndpoints}, {key, seed}); rc != FAST_FSS_SUCCESS) return rc;
        uint32_t G = 1;
        while (G < 32 && G < m) G <<= 1;
        auto kern = spline_eval_kernel<GE>;
        if (!prepare_aes_kernel(kern)) return FAST_FSS_RUNTIME_ERROR;
        kern<<<grid_for(N * G, aes_threads(N * G, kSplineEvalThreads), 1), aes_threads(N * G, kSplineEvalThreads),
                 kAesSmemTotal, resolve_stream(cudaStreamPtr)>>>(
            (GE *)sharedOut, (const GE *)maskedX, (const uint8_t *)key, (const GE *)sharedE, (const GE *)sharedBeta,
            (const uint8_t *)seed, (uint32_t)partyId, (const GE *)leftEndpoints, (const GE *)rightEndpoints,
            (uint32_t)m, (uint32_t)degree, (uint32_t)bitWidthIn, (uint32_t)bitWidthOut, N, G);
        return launch_status();
    });
}
