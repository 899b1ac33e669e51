// fss_host.h — host-side plumbing shared by the C-ABI entry points: element-size dispatch,
// stream resolution, grid sizing and launch-error reporting.
#pragma once

#include <FastFss/errors.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <mutex>
#include <set>
#include <utility>

namespace fss {

// The reference dispatches elementSize over {1,2,4,8,16,24,32} (src/impl/def.h:38-45);
// this library implements the built-in widths. Others get the reference's default-case
// error code.
template <typename F>
inline int dispatch_es(std::size_t elementSize, F &&f)
{
    switch (elementSize)
    {
        case 1: return f(std::uint8_t{});
        case 2: return f(std::uint16_t{});
        case 4: return f(std::uint32_t{});
        case 8: return f(std::uint64_t{});
        default: return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
}

// Stream convention of the reference (src/kernel/parallel_execute.h:164-168).
inline cudaStream_t resolve_stream(void *cudaStreamPtr)
{
    return cudaStreamPtr ? *static_cast<cudaStream_t *>(cudaStreamPtr) : cudaStreamPerThread;
}

inline int current_device()
{
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

inline int sm_count()
{
    static std::mutex mu;
    static int        cache[64] = {0};
    const int         dev       = current_device();
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0)
    {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

// Raises a kernel's dynamic shared-memory limit once per (kernel, device).
inline bool ensure_smem(const void *kernel, int bytes)
{
    static std::mutex                              mu;
    static std::set<std::pair<const void *, int>> done;
    const int                                      dev = current_device();
    std::lock_guard<std::mutex>                    lock(mu);
    if (done.count({kernel, dev})) return true;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    done.insert({kernel, dev});
    return true;
}

// Grid for an element-parallel kernel: enough CTAs to cover `work` items, capped at
// `perSm` resident CTAs on every SM (the kernels loop grid-stride beyond that).
inline unsigned grid_for(std::size_t work, int threads, int perSm)
{
    std::size_t need = (work + (std::size_t)threads - 1) / (std::size_t)threads;
    std::size_t cap  = (std::size_t)sm_count() * (std::size_t)perSm;
    if (need > cap) need = cap;
    if (need == 0) need = 1;
    return (unsigned)need;
}

// CTA size for an AES kernel (one CTA per SM, `maxThreads` threads at most) over `work` items
// taken grid-stride: the smallest whole number of warps that still covers the work in the
// same number of passes k = ceil(work / (SMs * maxThreads)), so that the last pass is not a
// partial wave on a few SMs and a small launch runs on every SM instead of a few full ones
// (at least 64 threads).
inline int aes_threads(std::size_t work, int maxThreads)
{
    const std::size_t sms   = (std::size_t)sm_count();
    const std::size_t full  = sms * (std::size_t)maxThreads;
    const std::size_t k     = work == 0 ? 1 : (work + full - 1) / full;
    std::size_t       t     = (work + sms * k - 1) / (sms * k);
    t                       = ((t + 31) / 32) * 32;
    if (t < 64) t = 64;
    if (t > (std::size_t)maxThreads) t = (std::size_t)maxThreads;
    return (int)t;
}

// Every AES kernel takes the replicated T-tables (kAesSmemTotal bytes of dynamic shared
// memory, declared in fss_device.cuh).
template <typename K>
inline bool prepare_aes_kernel(K kernel)
{
    return ensure_smem(reinterpret_cast<const void *>(kernel), 2 * 65536 + 256);
}

// Kernels read keys and seeds as 16-byte vectors and ring elements at their natural width;
// the reference requires 16-byte aligned keys (include/FastFss/cuda/dcf.h:25-26) and leaves
// misaligned buffers undefined. Here they are refused before any launch.
inline bool aligned_to(const void *p, std::size_t a)
{
    return ((std::uintptr_t)p & (a - 1)) == 0;
}

inline int check_alignment(std::size_t es, std::initializer_list<const void *> ring,
                           std::initializer_list<const void *> blocks)
{
    for (const void *p : ring)
        if (!aligned_to(p, es)) return FAST_FSS_RUNTIME_ERROR;
    for (const void *p : blocks)
        if (!aligned_to(p, 16)) return FAST_FSS_RUNTIME_ERROR;
    return FAST_FSS_SUCCESS;
}

inline int launch_status()
{
    return cudaGetLastError() == cudaSuccess ? FAST_FSS_SUCCESS : FAST_FSS_RUNTIME_ERROR;
}

} // namespace fss
