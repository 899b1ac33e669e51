/* Batched evaluation in one persistent launch (extension of this library; the reference
 * evaluates one request per call).
 *
 * A batch is a list of independent evaluation requests ("ops") of different kinds, element
 * sizes, bit widths and element counts. FastFss_cuda_batchPrepare validates the ops, cuts
 * them into tiles of roughly equal AES work and uploads a descriptor table into the caller's
 * device workspace. FastFss_cuda_batchLaunch then runs one persistent kernel (one CTA per SM)
 * whose CTAs claim tiles from a device-side work queue (an atomic tile counter in the
 * workspace) until the batch is drained; it issues only a 8-byte memset and a kernel launch
 * on the stream, so it can be captured in a CUDA graph and replayed. Every op produces
 * exactly the shares its per-call entry point produces (FastFss_cuda_dcfEval with groupSize
 * 1, FastFss_cuda_dpfEval with groupSize 1, FastFss_cuda_dcfMICEval,
 * FastFss_cuda_dcfSplineEval, FastFss_cuda_grottoEval); buffers follow those layouts.
 *
 * The workspace holds the queue and the descriptors: it must not be used by two launches
 * that overlap on the GPU. Errors: FAST_FSS_INVALID_ELEMENT_SIZE_ERROR,
 * FAST_FSS_INVALID_BITWIDTH_ERROR, FAST_FSS_INVALID_PARTY_ID_ERROR,
 * FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR (spline with no interval),
 * FAST_FSS_RUNTIME_ERROR (unknown kind, null buffer, workspace too small, CUDA failure). */
#ifndef FAST_FSS_B200_BATCH_H
#define FAST_FSS_B200_BATCH_H

#include <FastFss/api.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum FastFssBatchKind
{
    FAST_FSS_BATCH_DCF_EVAL     = 1, /* groupSize 1 */
    FAST_FSS_BATCH_DPF_EVAL     = 2, /* groupSize 1 */
    FAST_FSS_BATCH_DCF_MIC_EVAL = 3,
    FAST_FSS_BATCH_SPLINE_EVAL  = 4,
    FAST_FSS_BATCH_GROTTO_EVAL  = 5,
};

typedef struct FastFssBatchOp
{
    int32_t     kind;
    int32_t     partyId;
    uint32_t    elementSize;
    uint32_t    bitWidthIn;
    uint32_t    bitWidthOut;
    uint32_t    intervalNum; /* MIC, spline */
    uint32_t    degree;      /* spline */
    uint32_t    equalBound;  /* Grotto */
    uint64_t    elementNum;
    void       *sharedOut;
    const void *maskedX;
    const void *key;
    const void *seed;
    const void *aux0; /* MIC: sharedZ; spline: sharedE */
    const void *aux1; /* spline: sharedBeta */
    const void *leftEndpoints;
    const void *rightEndpoints;
} FastFssBatchOp;

typedef struct FastFssBatchTuning
{
    uint32_t ctaThreads;  /* 256 or 512; 0 selects 256 */
    uint32_t tileLookups; /* target AES table lookups per tile (at least one item per thread);
                             0 selects 1 << 26 */
    uint32_t order;       /* 0: costliest ops' tiles first; 1: caller order */
    uint32_t reserved;
} FastFssBatchTuning;

typedef struct FastFssBatchPlan
{
    uint64_t totalTiles;
    uint64_t totalItems;
    double   lookups; /* estimated AES table lookups of the whole batch */
    uint32_t opNum;
    uint32_t ctaThreads;
} FastFssBatchPlan;

FAST_FSS_API size_t FastFss_cuda_batchWorkspaceSize(size_t opNum);

FAST_FSS_API int FastFss_cuda_batchPrepare(const FastFssBatchOp *ops, size_t opNum, const FastFssBatchTuning *tuning,
                                           void *workspace, size_t workspaceSize, FastFssBatchPlan *plan,
                                           void *cudaStreamPtr);

FAST_FSS_API int FastFss_cuda_batchLaunch(const FastFssBatchPlan *plan, void *workspace, size_t workspaceSize,
                                          void *cudaStreamPtr);

/* FastFss_cuda_batchEvalNoAlloc — no counterpart in the reference.
 *
 * The same batched evaluation as FastFss_cuda_batchPrepare + FastFss_cuda_batchLaunch, for
 * callers that cannot allocate device memory and have no workspace to lend: a runtime that
 * reserves all device memory up front for its own pool (where any further cudaMalloc fails or
 * fragments that pool), or a latency-critical loop that must not pay cudaMalloc's implicit
 * device synchronisation. The work queue and the descriptor table live in a fixed array of
 * device memory inside this library (FAST_FSS_BATCH_NOALLOC_SCRATCH_BYTES bytes, held by every
 * GPU that loads the library until the process exits), so the call allocates nothing; the
 * caller still passes every input and output buffer through the ops.
 *
 * Limits and behaviour:
 *  - at most FAST_FSS_BATCH_NOALLOC_MAX_OPS ops per call; more return
 *    FAST_FSS_BATCH_TOO_MANY_OPS_ERROR before any device work;
 *  - the first call on a device looks up that array's device address (with the device
 *    current); make that first call before any stream capture begins;
 *  - every call reuses the same array: the queue counter is reset on the stream and the
 *    descriptor table rewritten by each call, so calls that overlap on the GPU (different
 *    streams, or different host threads without ordering) race and must not be issued;
 *  - the call returns once the descriptor table has been staged for upload, which waits for
 *    work already queued on the stream; validation and results as FastFss_cuda_batchPrepare. */
#define FAST_FSS_BATCH_NOALLOC_MAX_OPS       512
#define FAST_FSS_BATCH_NOALLOC_SCRATCH_BYTES (256 + FAST_FSS_BATCH_NOALLOC_MAX_OPS * 136)
#define FAST_FSS_BATCH_TOO_MANY_OPS_ERROR    (-32)

FAST_FSS_API int FastFss_cuda_batchEvalNoAlloc(const FastFssBatchOp *ops, size_t opNum,
                                               const FastFssBatchTuning *tuning, void *cudaStreamPtr);

#ifdef __cplusplus
}
#endif

#endif
