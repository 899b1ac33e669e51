// region_a_map.h — host side of region_a_stage.cuh: the 2-D tensor map over region A of a key
// (rows = elements, 16 n bytes each; x counted in bytes), boxes of 64 bytes x 32 rows with the
// 64-byte swizzle. The driver's encoder is looked up once per process.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace fss {

inline bool encode_region_a_map(CUtensorMap *map, const void *key, std::size_t n, std::size_t N)
{
    static std::once_flag                    once;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    std::call_once(once, [] {
        void                            *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        else
            cudaGetLastError();
    });
    if (encode == nullptr || N == 0 || N >= (1ull << 32) || ((std::size_t)key & 15u) != 0) return false;
    const cuuint64_t dims[2]    = {(cuuint64_t)(16 * n), (cuuint64_t)N};
    const cuuint64_t strides[1] = {(cuuint64_t)(16 * n)};
    const cuuint32_t box[2]     = {64u, 32u};
    const cuuint32_t estr[2]    = {1u, 1u};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(key), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace fss
