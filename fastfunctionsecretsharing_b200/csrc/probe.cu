// probe.cu — measured denominator for the AES roofline (see include/FastFss/b200/diag.h).
#include <FastFss/b200/diag.h>

#include "fss_device.cuh"
#include "fss_host.h"

namespace fss {

constexpr int kProbeThreads = 512;

// Issues 16 independent conflict-free table lookups per iteration (lane l reads bank l of
// rows it*7 .. it*7 + 15 of the Te0|Te1 region), with one address update per iteration, so
// the shared-memory pipe, not address arithmetic, bounds the rate.
__global__ void __launch_bounds__(kProbeThreads, 1) smem_lookup_probe_kernel(uint32_t *sink, uint32_t iters)
{
    aes_tables_build();
    const uint32_t lane4 = (threadIdx.x & 31u) << 2;
    uint32_t       acc0 = 0, acc1 = 0;
#pragma unroll 1
    for (uint32_t it = 0; it < iters; it++)
    {
        const uint32_t addr = (((it * 7u) & 0xEFu) << 8) | lane4;
#pragma unroll
        for (int k = 0; k < 16; k += 2)
        {
            acc0 ^= *reinterpret_cast<const uint32_t *>(fss_smem + addr + k * 256);
            acc1 ^= *reinterpret_cast<const uint32_t *>(fss_smem + addr + (k + 1) * 256);
        }
    }
    sink[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = acc0 ^ acc1;
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
    if (lookups) *lookups = (unsigned long long)grid * kProbeThreads * 16ull * iterations;
    return launch_status();
}
