// region_a_stage.cuh — per-warp staging of region A of a DCF or DPF key (one row of n 16-byte
// correction words per element, 16 n bytes apart) through shared memory.
//
// A warp evaluates 32 consecutive elements (a tile) at a time. kStageLevels levels of the 32
// rows arrive together by one TMA copy of a 64-byte x 32-row box of a 2-D tensor map over
// region A; two stages per warp are used in turn, so the next levels arrive while these are
// evaluated, and every lane reads its row with conflict-free 16-byte shared loads instead of
// one scattered global load per lane and level. The copy uses the 64-byte swizzle (16-byte
// chunk k of row r lands in chunk k ^ ((r >> 1) & 3)), which puts the 8 rows of a load phase
// in 8 different bank groups. Waits are bounded (stage.cuh): on a time-out the caller stops,
// drains and counts the failure.
#pragma once

#include <cuda.h>

#include "fss_device.cuh"
#include "stage.cuh"

namespace fss {

constexpr int kStageLevels    = 4;
constexpr int kStageRowBytes  = 16 * kStageLevels;                   // 64: the swizzle span
constexpr int kStageBytes     = 32 * kStageRowBytes;                 // 2048 per stage
constexpr int kStageBase      = (kAesSmemTotal + 1023) / 1024 * 1024; // stages 1024-byte aligned
constexpr int kWarpStageBytes = 2 * kStageBytes;

// Dynamic shared memory of a CTA of `warps` warps: tables, stages, then 2 mbarriers per warp.
constexpr int stage_smem_bytes(int warps)
{
    return kStageBase + warps * kWarpStageBytes + warps * 16;
}

// True if this CTA's dynamic shared window starts where the swizzled stages line up (it does
// on every launch seen; checked so that a misaligned copy is never issued).
__device__ __forceinline__ bool stage_window_ok()
{
    return (smem_u32(fss_smem + kStageBase) & 1023u) == 0;
}

struct RegionAStage
{
    const CUtensorMap *map;
    uint8_t           *ws;
    uint32_t           st0, bar0, swz, lane, C, ic, ib, b, parity;
    size_t             tiles, tstride, iT;

    // Every lane of the warp calls this; it issues the first two copies.
    __device__ __forceinline__ void init(const CUtensorMap *m, uint32_t n, size_t N, size_t tile0, size_t stride)
    {
        const uint32_t warp = threadIdx.x >> 5, W = blockDim.x >> 5;
        map                 = m;
        lane                = threadIdx.x & 31u;
        ws                  = fss_smem + kStageBase + (size_t)warp * kWarpStageBytes;
        st0                 = smem_u32(ws);
        bar0                = smem_u32(fss_smem + kStageBase + (size_t)W * kWarpStageBytes + 16 * warp);
        swz                 = 16u * ((lane >> 1) & 3u);
        C                   = (n + kStageLevels - 1) / kStageLevels;
        tiles               = (N + 31) / 32;
        tstride             = stride;
        iT                  = tile0;
        ic = ib = b = parity = 0;
        if (lane == 0)
        {
            mbar_init(bar0, 1);
            mbar_init(bar0 + 8, 1);
            mbar_init_fence();
        }
        __syncwarp();
        issue();
        issue();
    }

    // Copies the next chunk in consumption order: chunk ic of tile iT, then on to tile
    // iT + tstride after the last chunk of a tile. Warp-uniform.
    __device__ __forceinline__ void issue()
    {
        if (iT >= tiles) return;
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
        {
            // the whole box counts, rows past N and levels past n included (zero filled)
            mbar_arrive_expect_tx(bar0 + 8 * ib, kStageBytes);
            tensor_copy_2d_g2s(st0 + ib * kStageBytes, map, (int32_t)(ic * kStageRowBytes), (int32_t)(iT * 32),
                               bar0 + 8 * ib);
        }
        ib ^= 1u;
        if (++ic == C)
        {
            ic = 0;
            iT += tstride;
        }
    }

    // Waits for the chunk about to be evaluated; false if its copy did not arrive in time.
    __device__ __forceinline__ bool wait()
    {
        if (!mbar_wait_bounded(bar0 + 8 * b, (parity >> b) & 1u)) return false;
        parity ^= 1u << b;
        return true;
    }

    // Level j (< kStageLevels) of this lane's row in the current chunk, as big-endian words.
    __device__ __forceinline__ void level(uint32_t j, uint32_t cw[4]) const
    {
        const uint4 raw = *reinterpret_cast<const uint4 *>(ws + b * kStageBytes + lane * kStageRowBytes +
                                                           ((16u * j) ^ swz));
        cw[0] = bswap32(raw.x), cw[1] = bswap32(raw.y), cw[2] = bswap32(raw.z), cw[3] = bswap32(raw.w);
    }

    // The current chunk has been read: its stage is refilled two chunks ahead.
    __device__ __forceinline__ void next()
    {
        issue();
        b ^= 1u;
    }

    // After a failed wait: bounded waits for whatever is still in flight to this warp's stages.
    __device__ __forceinline__ void drain()
    {
        mbar_wait_bounded(bar0, parity & 1u);
        mbar_wait_bounded(bar0 + 8, (parity >> 1) & 1u);
    }
};

} // namespace fss
