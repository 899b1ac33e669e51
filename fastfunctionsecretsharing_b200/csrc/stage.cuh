// stage.cuh — asynchronous (TMA) global -> shared copies completed on a shared-memory mbarrier
// (sm_90+ `cp.async.bulk.tensor` and `mbarrier` PTX), used to stage per-warp key data. Every wait is
// bounded: after about a second the caller gets `false` and must record the timeout and stop
// using the stage.
#pragma once

#include <stdint.h>

namespace fss {

constexpr uint64_t kStageWaitNs    = 1000000000ull; // give up on a copy after 1 s
constexpr uint32_t kStageWaitLimit = 1u << 26;      // and after this many polls in any case

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes initialised barriers visible to the asynchronous (bulk copy) proxy.
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of copies to complete on this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity; false if it did not complete within
// kStageWaitNs (or kStageWaitLimit polls).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < kStageWaitLimit; it++)
    {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kStageWaitNs) return false;
    }
    return false;
}

// One box of a 2-D tiled tensor map (`map`: generic address of a __grid_constant__ CUtensorMap)
// at element coordinates (x, y) into shared `dst`, completing on `bar`. x times the element
// size must be a multiple of 16 bytes. No multicast.
__device__ __forceinline__ void tensor_copy_2d_g2s(uint32_t dst, const void *map, int32_t x, int32_t y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Orders this thread's earlier shared-memory accesses before later bulk-copy writes.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

} // namespace fss
