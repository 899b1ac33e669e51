// config.cpp — FastFss_cuda_{set,get}GridDim and the fine-grain threshold
// (include/FastFss/cuda/config.h:18-30 and src/cuda/config.cpp:6-70 of the reference): the
// same defaults (128, 64), the same -2 for non-positive values, guarded by a mutex. The
// kernels of this library size their grids from the SM count, so the values are stored and
// reported only.
#include <FastFss/cuda/config.h>

#include <mutex>

namespace {
int        gGridDim   = 128;
int        gThreshold = 64;
std::mutex gMutex;
} // namespace

extern "C" FAST_FSS_API int FastFss_cuda_setGridDim(int dim)
{
    std::lock_guard<std::mutex> lock(gMutex);
    if (dim <= 0) return -2;
    gGridDim = dim;
    return 0;
}

extern "C" FAST_FSS_API int FastFss_cuda_getGridDim()
{
    std::lock_guard<std::mutex> lock(gMutex);
    return gGridDim;
}

extern "C" FAST_FSS_API int FastFss_cuda_setFineGrainParallelGridDimThreshold(int dim)
{
    std::lock_guard<std::mutex> lock(gMutex);
    if (dim <= 0) return -2;
    gThreshold = dim;
    return 0;
}

extern "C" FAST_FSS_API int FastFss_cuda_getFineGrainParallelGridDimThreshold()
{
    std::lock_guard<std::mutex> lock(gMutex);
    return gThreshold;
}
