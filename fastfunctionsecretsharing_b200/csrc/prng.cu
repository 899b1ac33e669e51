// prng.cu — AES-128-CTR generator (FastFss_cuda_prng*), sm_100a.
//
// Reference behaviour: include/FastFss/cuda/prng.h:12-25, src/cuda/prng.cu:24-185 and the
// CPU twin src/cpu/prng.cpp:20-147. Output byte stream: block i = AES_seed(counter + i) with
// the 128-bit counter as two little-endian uint64 (carry from the low into the high word);
// a trailing partial block keeps its first bytes; the counter then advances by the number of
// blocks used, carry included. The advance follows the CPU implementation
// (counter.hi += (counter.lo_new < blocks)); the reference CUDA kernel derives the carry from
// the old low word (src/cuda/prng.cu:84-86), which differs from its CPU twin only when the
// low word wraps.
//
// The generator state lives in device memory owned by the handle: {seed, counter, next}.
// Gen is asynchronous on the caller's stream: the kernel writes the advanced counter to
// `next` and a stream-ordered 16-byte device copy moves it to `counter` (no host sync).
// Every thread expands the (shared) key once into registers and encrypts its blocks with
// the shared-memory T-tables.
#include <FastFss/cuda/prng.h>
#include <FastFss/errors.h>

#include "fss_device.cuh"
#include "fss_host.h"

namespace fss {

struct PrngState
{
    unsigned char seed[16];
    unsigned char counter[16];
    unsigned char next[16];
};

constexpr int kPrngThreads = 512;

__global__ void __launch_bounds__(kPrngThreads, 1)
    prng_ctr_kernel(PrngState *__restrict__ st, uint8_t *__restrict__ dst, size_t bytes, bool aligned16)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    uint32_t key[4];
    load_block_be(st->seed, key);
    // round keys once per thread
    uint32_t rk[11][4];
#pragma unroll
    for (int c = 0; c < 4; c++) rk[0][c] = key[c];
    constexpr uint32_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
#pragma unroll
    for (int r = 0; r < 10; r++)
    {
#pragma unroll
        for (int c = 0; c < 4; c++) rk[r + 1][c] = rk[r][c];
        key_step(A, rk[r + 1], RCON[r]);
    }
    const unsigned long long c0 = reinterpret_cast<const unsigned long long *>(st->counter)[0];
    const unsigned long long c1 = reinterpret_cast<const unsigned long long *>(st->counter)[1];
    const size_t             nblk = (bytes + 15) / 16;
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += (size_t)gridDim.x * blockDim.x)
    {
        const unsigned long long lo = c0 + (unsigned long long)b;
        const unsigned long long hi = c1 + (lo < c0 ? 1ull : 0ull);
        uint32_t                 s[4];
        s[0] = bswap32((uint32_t)lo) ^ rk[0][0];
        s[1] = bswap32((uint32_t)(lo >> 32)) ^ rk[0][1];
        s[2] = bswap32((uint32_t)hi) ^ rk[0][2];
        s[3] = bswap32((uint32_t)(hi >> 32)) ^ rk[0][3];
#pragma unroll
        for (int r = 1; r < 10; r++) enc_round(A, s, rk[r]);
        enc_last(A, s, rk[10]);
        uint8_t *p = dst + 16 * b;
        if (16 * b + 16 <= bytes && aligned16)
        {
            store_block_be(p, s);
        }
        else
        {
            const size_t lim = bytes - 16 * b < 16 ? bytes - 16 * b : 16;
            for (size_t k = 0; k < lim; k++) p[k] = (uint8_t)block_byte(s, (int)k);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        const unsigned long long nlo                             = c0 + (unsigned long long)nblk;
        reinterpret_cast<unsigned long long *>(st->next)[0] = nlo;
        reinterpret_cast<unsigned long long *>(st->next)[1] = c1 + (nlo < (unsigned long long)nblk ? 1ull : 0ull);
    }
}

} // namespace fss

using namespace fss;

extern "C" FAST_FSS_API void *FastFss_cuda_prngInit()
{
    void *p = nullptr;
    if (cudaMalloc(&p, sizeof(PrngState)) != cudaSuccess) return nullptr;
    if (cudaMemset(p, 0, sizeof(PrngState)) != cudaSuccess)
    {
        cudaFree(p);
        return nullptr;
    }
    return p;
}

extern "C" FAST_FSS_API void FastFss_cuda_prngRelease(void *prng)
{
    if (prng) cudaFree(prng);
}

extern "C" FAST_FSS_API int FastFss_cuda_prngSetCurrentSeed(void *prng, const void *hostSeed128bit,
                                                            const void *hostCounter128bit)
{
    if (prng == nullptr || hostSeed128bit == nullptr) return FAST_FSS_PRNG_INPUT_INVALID_ARGUMENT;
    PrngState *st = (PrngState *)prng;
    if (cudaMemcpy(st->seed, hostSeed128bit, 16, cudaMemcpyHostToDevice) != cudaSuccess) return FAST_FSS_RUNTIME_ERROR;
    cudaError_t e = hostCounter128bit ? cudaMemcpy(st->counter, hostCounter128bit, 16, cudaMemcpyHostToDevice)
                                      : cudaMemset(st->counter, 0, 16);
    return e == cudaSuccess ? FAST_FSS_SUCCESS : FAST_FSS_RUNTIME_ERROR;
}

extern "C" FAST_FSS_API int FastFss_cuda_prngGetCurrentSeed(const void *prng, void *hostSeed128bit,
                                                            void *hostCounter128bit)
{
    if (prng == nullptr || hostSeed128bit == nullptr) return FAST_FSS_PRNG_INPUT_INVALID_ARGUMENT;
    const PrngState *st = (const PrngState *)prng;
    if (cudaMemcpy(hostSeed128bit, st->seed, 16, cudaMemcpyDeviceToHost) != cudaSuccess) return FAST_FSS_RUNTIME_ERROR;
    if (hostCounter128bit && cudaMemcpy(hostCounter128bit, st->counter, 16, cudaMemcpyDeviceToHost) != cudaSuccess)
        return FAST_FSS_RUNTIME_ERROR;
    return FAST_FSS_SUCCESS;
}

extern "C" FAST_FSS_API int FastFss_cuda_prngGen(void *prng, void *deviceDst, size_t bitWidth, size_t elementSize,
                                                 size_t elementNum, void *cudaStreamPtr)
{
    if (prng == nullptr || deviceDst == nullptr) return FAST_FSS_PRNG_INPUT_INVALID_ARGUMENT;
    if (bitWidth == 0 || bitWidth > elementSize * 8) return FAST_FSS_PRNG_INVALID_BIT_WIDTH;
    const size_t bytes = elementNum * elementSize;
    if (bytes == 0) return FAST_FSS_SUCCESS;
    PrngState   *st     = (PrngState *)prng;
    cudaStream_t stream = resolve_stream(cudaStreamPtr);
    if (!prepare_aes_kernel(prng_ctr_kernel)) return FAST_FSS_RUNTIME_ERROR;
    const size_t nblk = (bytes + 15) / 16;
    prng_ctr_kernel<<<grid_for(nblk, kPrngThreads, 1), kPrngThreads, kAesSmemTotal, stream>>>(
        st, (uint8_t *)deviceDst, bytes, ((uintptr_t)deviceDst & 15u) == 0);
    if (launch_status() != FAST_FSS_SUCCESS) return FAST_FSS_RUNTIME_ERROR;
    if (cudaMemcpyAsync(st->counter, st->next, 16, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        return FAST_FSS_RUNTIME_ERROR;
    return FAST_FSS_SUCCESS;
}
