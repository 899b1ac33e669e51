// sizes.cpp — host-only key/cache size queries and the zip/unzip entry points.
//
// Values and validation follow the reference's src/{dcf,dpf,grotto,mic,spline,ottt}.cpp with
// the size formulas of src/impl/*.h. Element sizes the reference cannot dispatch take its
// default case (src/impl/def.h:38-45): INVALID_ELEMENT_SIZE (and a size of SIZE_MAX) for
// DCF/DPF, a size of 0 and success for Grotto/MIC/spline. Zip/Unzip are not implemented by the reference
// (src/dcf.cpp:10-34) and return FAST_FSS_RUNTIME_ERROR here too.
#include <FastFss/dcf.h>
#include <FastFss/dpf.h>
#include <FastFss/errors.h>
#include <FastFss/grotto.h>
#include <FastFss/mic.h>
#include <FastFss/ottt.h>
#include <FastFss/spline.h>

#include <cstddef>

namespace {

// The widths the reference's dispatch knows (src/impl/def.h:38-45). Size queries are pure
// arithmetic, so they answer for the wide-integer widths too; the kernels support 1..8.
bool known_es(size_t es)
{
    return es == 1 || es == 2 || es == 4 || es == 8 || es == 16 || es == 24 || es == 32;
}

size_t dcf_key(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n + es * n * g + es + es + es * g);
}

size_t dcf_cache(size_t n, size_t g, size_t es, size_t N)
{
    return N * (16 * n) + N * es * n * g;
}

} // namespace

extern "C" {

FAST_FSS_API int FastFss_dcfKeyZip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_dcfKeyUnzip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_dcfGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                           size_t groupSize, size_t elementSize, size_t elementNum)
{
    if (!(0 < bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!(0 < bitWidthOut && bitWidthOut <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *keyDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *keyDataSize = dcf_key(bitWidthIn, groupSize, elementSize, elementNum);
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                 size_t groupSize, size_t elementSize, size_t elementNum)
{
    (void)groupSize, (void)elementNum;
    if (!(0 < bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!(0 < bitWidthOut && bitWidthOut <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *keyDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *keyDataSize = 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                             size_t groupSize, size_t elementSize, size_t elementNum)
{
    if (!(0 < bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!(0 < bitWidthOut && bitWidthOut <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *cacheDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *cacheDataSize = dcf_cache(bitWidthIn, groupSize, elementSize, elementNum);
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dpfKeyZip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_dpfKeyUnzip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

// src/dpf.cpp checks only the upper bound of the widths.
FAST_FSS_API int FastFss_dpfGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                           size_t groupSize, size_t elementSize, size_t elementNum)
{
    if (bitWidthIn > elementSize * 8 || bitWidthOut > elementSize * 8) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *keyDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *keyDataSize = elementNum * (16 * bitWidthIn + 2 * elementSize + elementSize * groupSize);
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dpfGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                 size_t groupSize, size_t elementSize, size_t elementNum)
{
    (void)groupSize, (void)elementNum;
    if (bitWidthIn > elementSize * 8 || bitWidthOut > elementSize * 8) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *keyDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *keyDataSize = 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dpfGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t elementSize,
                                             size_t elementNum)
{
    if (bitWidthIn > elementSize * 8) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (!known_es(elementSize))
    {
        *cacheDataSize = (size_t)-1;
        return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    }
    *cacheDataSize = elementNum * 16 * bitWidthIn;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_grottoKeyZip(void *, size_t, const void *, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_grottoKeyUnzip(void *, size_t, const void *, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_grottoGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementSize,
                                              size_t elementNum)
{
    if (!(6 <= bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    *keyDataSize = known_es(elementSize) ? elementNum * (16 * (bitWidthIn - 6) + 8 + 2 * elementSize) : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_grottoGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementSize,
                                                    size_t elementNum)
{
    (void)elementNum;
    if (!(6 <= bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    *keyDataSize = known_es(elementSize) ? (size_t)-1 : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_grottoGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t elementSize,
                                                size_t elementNum)
{
    if (!(6 <= bitWidthIn && bitWidthIn <= elementSize * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    *cacheDataSize = known_es(elementSize) ? elementNum * (16 * (bitWidthIn - 6) + (bitWidthIn - 6)) : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfMICKeyZip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_dcfMICKeyUnzip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

// src/mic.cpp validates nothing but the element size.
FAST_FSS_API int FastFss_dcfMICGetCacheDataSize(size_t *cacheDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                size_t elementSize, size_t elementNum)
{
    (void)bitWidthOut;
    *cacheDataSize = known_es(elementSize) ? dcf_cache(bitWidthIn, 1, elementSize, elementNum) : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfMICGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                              size_t elementSize, size_t elementNum)
{
    (void)bitWidthOut;
    *keyDataSize = known_es(elementSize) ? dcf_key(bitWidthIn, 1, elementSize, elementNum) : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfMICGetZippedKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t bitWidthOut,
                                                    size_t elementSize, size_t elementNum)
{
    (void)bitWidthIn, (void)bitWidthOut, (void)elementSize, (void)elementNum;
    *keyDataSize = 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfSplineKeyZip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t, size_t,
                                         size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

FAST_FSS_API int FastFss_dcfSplineKeyUnzip(void *, size_t, const void *, size_t, size_t, size_t, size_t, size_t,
                                           size_t, size_t)
{
    return FAST_FSS_RUNTIME_ERROR;
}

// src/spline.cpp validates nothing but the element size (src/impl/spline.h:27-48).
FAST_FSS_API int FastFss_dcfSplineGetCacheDataSize(size_t *cacheDataSize, size_t degree, size_t intervalNum,
                                                   size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                   size_t elementNum)
{
    (void)bitWidthOut;
    if (!known_es(elementSize))
    {
        *cacheDataSize = 0;
        return FAST_FSS_SUCCESS;
    }
    const size_t g = intervalNum * (degree + 1);
    *cacheDataSize = dcf_cache(bitWidthIn, g, elementSize, elementNum) +
                     elementNum * elementSize * (2 * g + degree + 1);
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfSplineGetKeyDataSize(size_t *keyDataSize, size_t degree, size_t intervalNum,
                                                 size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                 size_t elementNum)
{
    (void)bitWidthOut;
    *keyDataSize =
        known_es(elementSize) ? dcf_key(bitWidthIn, intervalNum * (degree + 1), elementSize, elementNum) : 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_dcfSplineGetZippedKeyDataSize(size_t *keyDataSize, size_t degree, size_t intervalNum,
                                                       size_t bitWidthIn, size_t bitWidthOut, size_t elementSize,
                                                       size_t elementNum)
{
    (void)degree, (void)intervalNum, (void)bitWidthIn, (void)bitWidthOut, (void)elementSize, (void)elementNum;
    *keyDataSize = 0;
    return FAST_FSS_SUCCESS;
}

FAST_FSS_API int FastFss_otttGetKeyDataSize(size_t *keyDataSize, size_t bitWidthIn, size_t elementNum)
{
    if (!(3 <= bitWidthIn)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    *keyDataSize = elementNum * ((size_t)1 << bitWidthIn) / 8;
    return FAST_FSS_SUCCESS;
}

} // extern "C"
