// probe.cu — measured denominator for the AES roofline (see include/FastFss/b200/diag.h).
#include <FastFss/b200/diag.h>

#include "fss_device.cuh"
#include "fss_host.h"

namespace fss {

constexpr int kProbeThreads = 512;

__global__ void __launch_bounds__(kProbeThreads, 1) smem_lookup_probe_kernel(uint32_t *sink, uint32_t iters)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    uint32_t c[8];
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = (threadIdx.x * 2654435761u) ^ (uint32_t)(k * 0x9e3779b9u) ^ blockIdx.x;
#pragma unroll 1
    for (uint32_t it = 0; it < iters; it++)
    {
#pragma unroll
        for (int k = 0; k < 8; k++) c[k] ^= te<0, 1>(A, c[k]);
    }
    uint32_t r = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) r ^= c[k];
    sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = r;
}

} // namespace fss

using namespace fss;

extern "C" FAST_FSS_API int FastFss_b200_smCount(void)
{
    return sm_count();
}

extern "C" FAST_FSS_API int FastFss_b200_smemLookupProbe(void *sink, size_t sinkBytes, unsigned iterations,
                                                         unsigned long long *lookups, void *cudaStreamPtr)
{
    const unsigned grid = (unsigned)sm_count();
    if (sink == nullptr || sinkBytes < (size_t)4 * kProbeThreads * grid) return FAST_FSS_RUNTIME_ERROR;
    if (!prepare_aes_kernel(smem_lookup_probe_kernel)) return FAST_FSS_RUNTIME_ERROR;
    smem_lookup_probe_kernel<<<grid, kProbeThreads, kAesSmemTotal, resolve_stream(cudaStreamPtr)>>>(
        (uint32_t *)sink, iterations);
    if (lookups) *lookups = (unsigned long long)grid * kProbeThreads * 8ull * iterations;
    return launch_status();
}
