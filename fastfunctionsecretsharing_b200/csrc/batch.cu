// batch.cu — mixed FSS evaluation requests in one persistent launch (include/FastFss/b200/batch.h).
//
// Plan (host): every op becomes `items` work items (an element, an (element, interval) pair
// for MIC, or a lane of a G-lane element group for spline) with an estimated cost in AES
// table lookups per item; items are cut into tiles of about `tileLookups` lookups, in whole
// multiples of the CTA's thread count (every thread has an item; spline lane groups never
// straddle a warp), ops are laid out costliest first and numbered by a prefix sum of their
// tile counts. A batch with fewer items than the SMs' CTAs have threads is instead cut into
// about one tile per SM (whole warps), so small batches use every SM.
//
// Kernel (device): one CTA per SM builds the replicated AES tables once, then repeatedly
// claims the next tile from the atomic counter in the workspace, finds its op by binary
// search over the tile prefix sums, and runs that op's per-item routine over the tile with
// all its threads. A CTA only ever runs one op at a time, so warps never mix kinds or widths.
// The loop ends when the counter passes the last tile (no waiting on other CTAs).
#include <FastFss/b200/batch.h>
#include <FastFss/errors.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "dcf_core.cuh"
#include "dpf_core.cuh"
#include "fss_device.cuh"
#include "fss_host.h"
#include "grotto_core.cuh"
#include "mic_core.cuh"
#include "spline_core.cuh"

namespace fss {

struct BatchOpDev
{
    uint32_t           kind, es, n, bo, m, d, party, eb, G, pad;
    unsigned long long N, items, tileItems, tileBegin;
    void              *out;
    const void        *x, *key, *seed, *aux0, *aux1, *L, *R;
};

constexpr size_t kBatchHeader    = 256; // tile counter, then padding
// after the tables: the claimed tile (16 B), then the MIC point shares (one per thread, 512 at
// most) and their count
constexpr int    kBatchSmemExtra = 16 + 512 * 8 + 16;

template <typename GE>
__device__ __forceinline__ void batch_run_tile(const AesLanes &A, const BatchOpDev &op, unsigned long long first,
                                               unsigned long long last)
{
    const uint32_t n = op.n, bo = op.bo, party = op.party;
    const size_t   N = op.N;
    GE            *out = (GE *)op.out;
    const GE      *xs  = (const GE *)op.x;
    const uint8_t *key = (const uint8_t *)op.key, *seed = (const uint8_t *)op.seed;
    switch (op.kind)
    {
        case FAST_FSS_BATCH_DCF_EVAL:
            for (unsigned long long k = first + threadIdx.x; k < last; k += blockDim.x)
            {
                DcfKeyView<GE> K;
                K.set(key, n, 1, k, N);
                out[k] = (GE)dcf_eval_g1<GE>(A, K, seed + 16 * k, party, n, bo, mod_bits<GE>((uint64_t)__ldg(xs + k), n));
            }
            break;
        case FAST_FSS_BATCH_DPF_EVAL:
            for (unsigned long long k = first + threadIdx.x; k < last; k += blockDim.x)
            {
                const GE *kb = reinterpret_cast<const GE *>(key + N * 16 * n + k * sizeof(GE) * 3);
                dpf_eval_point<GE>(A, out + k, key + k * 16 * n, kb, seed + 16 * k, party, n, bo, 1,
                                   mod_bits<GE>((uint64_t)__ldg(xs + k), n), (uint64_t)__ldg(kb),
                                   (uint64_t)__ldg(kb + 1));
            }
            break;
        case FAST_FSS_BATCH_DCF_MIC_EVAL:
        {
            // touching intervals: the elements the tile's items belong to, each point walked
            // once (mic_shared_batch); otherwise one item per thread, both walks
            uint64_t *shares = reinterpret_cast<uint64_t *>(fss_smem + kAesSmemTotal + 16);
            uint32_t *points = reinterpret_cast<uint32_t *>(shares + blockDim.x);
            if (threadIdx.x == 0) *points = mic_points<GE>((const GE *)op.L, (const GE *)op.R, op.m, n);
            __syncthreads();
            const uint32_t P = *points;
            if (P != 0 && P <= blockDim.x)
            {
                const size_t e0 = first / op.m, e1 = (last + op.m - 1) / op.m, E = blockDim.x / P;
                for (size_t base = e0; base < e1; base += E)
                    mic_shared_batch<GE>(A, shares, out, xs, key, (const GE *)op.aux0, seed, party, (const GE *)op.L,
                                         (const GE *)op.R, op.m, n, bo, N, P, base, e1, first, last);
            }
            else
            {
                for (unsigned long long k = first + threadIdx.x; k < last; k += blockDim.x)
                    out[k] = mic_eval_item<GE>(A, xs, key, (const GE *)op.aux0, seed, party, (const GE *)op.L,
                                               (const GE *)op.R, op.m, n, bo, N, k);
            }
            break;
        }
        case FAST_FSS_BATCH_SPLINE_EVAL:
        {
            // whole warps iterate together (the group reduction shuffles)
            const unsigned long long end = first + ((last - first + 31) / 32) * 32;
            for (unsigned long long k = first + threadIdx.x; k < end; k += blockDim.x)
                spline_eval_group<GE>(A, out, xs, key, (const GE *)op.aux0, (const GE *)op.aux1, seed, party,
                                      (const GE *)op.L, (const GE *)op.R, op.m, op.d, n, bo, N, op.G, k / op.G,
                                      (uint32_t)(k % op.G), k < last);
            break;
        }
        case FAST_FSS_BATCH_GROTTO_EVAL:
            for (unsigned long long k = first + threadIdx.x; k < last; k += blockDim.x)
            {
                GrottoKeyView<GE> K;
                K.set(key, n, k, N);
                out[k] = (GE)grotto_cmp<GE>(A, K, seed + 16 * k, party, n, mod_bits<GE>((uint64_t)__ldg(xs + k), n),
                                            op.eb != 0);
            }
            break;
        default: break;
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
    batch_kernel(const BatchOpDev *__restrict__ ops, uint32_t opNum, unsigned long long *counter,
                 unsigned long long totalTiles)
{
    aes_tables_build();
    AesLanes A;
    A.init();
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(fss_smem + kAesSmemTotal);
    for (;;)
    {
        if (threadIdx.x == 0) *slot = atomicAdd(counter, 1ull);
        __syncthreads();
        const unsigned long long t = *slot;
        __syncthreads();
        if (t >= totalTiles) break;
        uint32_t lo = 0, hi = opNum - 1;
        while (lo < hi)
        {
            const uint32_t mid = (lo + hi + 1) / 2;
            if (ops[mid].tileBegin <= t)
                lo = mid;
            else
                hi = mid - 1;
        }
        const BatchOpDev         &op    = ops[lo];
        const unsigned long long first = (t - op.tileBegin) * op.tileItems;
        const unsigned long long last  = first + op.tileItems < op.items ? first + op.tileItems : op.items;
        switch (op.es)
        {
            case 1: batch_run_tile<uint8_t>(A, op, first, last); break;
            case 2: batch_run_tile<uint16_t>(A, op, first, last); break;
            case 4: batch_run_tile<uint32_t>(A, op, first, last); break;
            default: batch_run_tile<uint64_t>(A, op, first, last); break;
        }
        __syncthreads();
    }
}

// Estimated AES table lookups of one work item (a key schedule is 40, a block 160).
static double item_cost(const FastFssBatchOp &o, uint32_t G)
{
    const double n = o.bitWidthIn;
    switch (o.kind)
    {
        case FAST_FSS_BATCH_DCF_EVAL: return n * 340.0;
        case FAST_FSS_BATCH_DPF_EVAL: return n * 200.0 + 200.0;
        case FAST_FSS_BATCH_DCF_MIC_EVAL: return 2.0 * n * 340.0;
        case FAST_FSS_BATCH_SPLINE_EVAL:
        {
            // whole passes: interval groups per lane and coefficient chunks per slot
            const double per_q  = (double)((o.intervalNum + G - 1) / G);
            const double chunks = (double)((o.degree + 1 + kSplineMaxC - 1) / kSplineMaxC);
            return per_q * chunks * 2.0 * n * (340.0 + 360.0);
        }
        case FAST_FSS_BATCH_GROTTO_EVAL: return (n - 6) * 200.0;
        default: return 0.0;
    }
}

static int validate(const FastFssBatchOp &o)
{
    const uint32_t es = o.elementSize;
    if (!(es == 1 || es == 2 || es == 4 || es == 8)) return FAST_FSS_INVALID_ELEMENT_SIZE_ERROR;
    if (o.kind < FAST_FSS_BATCH_DCF_EVAL || o.kind > FAST_FSS_BATCH_GROTTO_EVAL) return FAST_FSS_RUNTIME_ERROR;
    const uint32_t nmin = o.kind == FAST_FSS_BATCH_GROTTO_EVAL ? 6u : 1u;
    if (!(nmin <= o.bitWidthIn && o.bitWidthIn <= es * 8)) return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (o.kind != FAST_FSS_BATCH_GROTTO_EVAL && !(0 < o.bitWidthOut && o.bitWidthOut <= es * 8))
        return FAST_FSS_INVALID_BITWIDTH_ERROR;
    if (o.partyId != 0 && o.partyId != 1) return FAST_FSS_INVALID_PARTY_ID_ERROR;
    if (o.kind == FAST_FSS_BATCH_SPLINE_EVAL && o.intervalNum == 0) return FAST_FSS_INVALID_BOUNDARY_DATA_SIZE_ERROR;
    if (o.elementNum == 0) return FAST_FSS_SUCCESS;
    if (!o.sharedOut || !o.maskedX || !o.key || !o.seed) return FAST_FSS_RUNTIME_ERROR;
    if (o.kind == FAST_FSS_BATCH_DCF_MIC_EVAL && o.intervalNum && (!o.aux0 || !o.leftEndpoints || !o.rightEndpoints))
        return FAST_FSS_RUNTIME_ERROR;
    if (o.kind == FAST_FSS_BATCH_SPLINE_EVAL && (!o.aux0 || !o.aux1 || !o.leftEndpoints || !o.rightEndpoints))
        return FAST_FSS_RUNTIME_ERROR;
    if (int rc = check_alignment(es, {o.sharedOut, o.maskedX, o.aux0, o.aux1, o.leftEndpoints, o.rightEndpoints},
                                 {o.key, o.seed});
        rc != FAST_FSS_SUCCESS)
        return rc;
    return FAST_FSS_SUCCESS;
}

// Builds the device descriptor table; returns an error code or success.
int batch_plan(const FastFssBatchOp *ops, size_t opNum, const FastFssBatchTuning *tuning,
               std::vector<BatchOpDev> &dev, FastFssBatchPlan *plan)
{
    const uint32_t threads   = (tuning && tuning->ctaThreads == 512) ? 512u : 256u;
    const double   tileCost  = (tuning && tuning->tileLookups) ? (double)tuning->tileLookups : (double)(1u << 26);
    const bool     callOrder = tuning && tuning->order == 1;
    struct Row
    {
        BatchOpDev d;
        double     cost;
    };
    std::vector<Row> rows;
    rows.reserve(opNum);
    double lookups = 0;
    for (size_t q = 0; q < opNum; q++)
    {
        const FastFssBatchOp &o  = ops[q];
        const int             rc = validate(o);
        if (rc != FAST_FSS_SUCCESS) return rc;
        uint32_t G = 1;
        if (o.kind == FAST_FSS_BATCH_SPLINE_EVAL)
            while (G < 32 && G < o.intervalNum) G <<= 1;
        unsigned long long items = o.elementNum;
        if (o.kind == FAST_FSS_BATCH_DCF_MIC_EVAL) items = o.elementNum * o.intervalNum;
        if (o.kind == FAST_FSS_BATCH_SPLINE_EVAL) items = o.elementNum * G;
        if (items == 0) continue;
        const double c  = item_cost(o, G);
        double       ti = tileCost / (c > 1 ? c : 1);
        // a tile fills every thread of the CTA at least once (whole multiples of the CTA)
        ti = ti < threads ? threads : (ti > 1048576 ? 1048576 : ti);
        BatchOpDev d{};
        d.kind      = (uint32_t)o.kind;
        d.es        = o.elementSize;
        d.n         = o.bitWidthIn;
        d.bo        = o.bitWidthOut;
        d.m         = o.intervalNum;
        d.d         = o.degree;
        d.party     = (uint32_t)o.partyId;
        d.eb        = o.equalBound;
        d.G         = G;
        d.N         = o.elementNum;
        d.items     = items;
        d.tileItems = ((unsigned long long)ti / threads) * threads;
        d.out       = o.sharedOut;
        d.x         = o.maskedX;
        d.key       = o.key;
        d.seed      = o.seed;
        d.aux0      = o.aux0;
        d.aux1      = o.aux1;
        d.L         = o.leftEndpoints;
        d.R         = o.rightEndpoints;
        rows.push_back({d, c});
        lookups += c * (double)items;
    }
    // Tile sizes by work. k = tiles per SM at the tuned tile cost (at least 1); every op gets
    // tiles in proportion to its share of the work, so the batch splits into about k x SMs
    // tiles of similar work that the atomic queue can balance. A tile holds whole CTAs of items
    // when it is that large, else whole warps: a small batch then runs partly idle CTAs on SMs
    // that would otherwise have nothing to do, instead of a few SMs working through large tiles.
    // In a small batch (k = 1) no tile gives a thread more than one item: the ops' per-SM
    // rates differ (a DCF element is one thread's serial walk, a spline element a warp's), so
    // equal shares of lookups are not equal times; one-item tiles let the queue even them out.
    const unsigned long long sms = (unsigned long long)sm_count();
    if (!rows.empty() && lookups > 0)
    {
        const double k = std::max(1.0, std::floor(lookups / ((double)sms * tileCost)));
        for (auto &r : rows)
        {
            const double       share = r.cost * (double)r.d.items / lookups;
            const double       want  = std::max(1.0, std::round(share * k * (double)sms));
            unsigned long long ti    = (unsigned long long)std::ceil((double)r.d.items / want);
            if (k == 1.0) ti = std::min<unsigned long long>(ti, threads);
            if (ti >= threads)
                ti = std::min<unsigned long long>((ti / threads) * threads, 1048576ull);
            else
                ti = std::max<unsigned long long>(32, ((ti + 31) / 32) * 32);
            r.d.tileItems = ti;
        }
    }
    if (!callOrder)
        std::stable_sort(rows.begin(), rows.end(), [](const Row &a, const Row &b) { return a.cost > b.cost; });
    dev.clear();
    unsigned long long tiles = 0, totalItems = 0;
    for (auto &r : rows)
    {
        r.d.tileBegin = tiles;
        tiles += (r.d.items + r.d.tileItems - 1) / r.d.tileItems;
        totalItems += r.d.items;
        dev.push_back(r.d);
    }
    plan->totalTiles = tiles;
    plan->totalItems = totalItems;
    plan->lookups    = lookups;
    plan->opNum      = (uint32_t)dev.size();
    plan->ctaThreads = threads;
    return FAST_FSS_SUCCESS;
}

int batch_launch(const FastFssBatchPlan *plan, const BatchOpDev *devOps, unsigned long long *counter,
                 cudaStream_t stream)
{
    if (plan->totalTiles == 0) return FAST_FSS_SUCCESS;
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned long long), stream) != cudaSuccess)
        return FAST_FSS_RUNTIME_ERROR;
    const unsigned grid =
        (unsigned)std::min<unsigned long long>(plan->totalTiles, (unsigned long long)sm_count());
    const int smem = kAesSmemTotal + kBatchSmemExtra;
    if (plan->ctaThreads == 512)
    {
        if (!ensure_smem(reinterpret_cast<const void *>(batch_kernel<512>), smem)) return FAST_FSS_RUNTIME_ERROR;
        batch_kernel<512><<<grid, 512, smem, stream>>>(devOps, plan->opNum, counter, plan->totalTiles);
    }
    else
    {
        if (!ensure_smem(reinterpret_cast<const void *>(batch_kernel<256>), smem)) return FAST_FSS_RUNTIME_ERROR;
        batch_kernel<256><<<grid, 256, smem, stream>>>(devOps, plan->opNum, counter, plan->totalTiles);
    }
    return launch_status();
}

} // namespace fss

using namespace fss;

extern "C" FAST_FSS_API size_t FastFss_cuda_batchWorkspaceSize(size_t opNum)
{
    return kBatchHeader + opNum * sizeof(BatchOpDev);
}

extern "C" FAST_FSS_API int FastFss_cuda_batchPrepare(const FastFssBatchOp *ops, size_t opNum,
                                                      const FastFssBatchTuning *tuning, void *workspace,
                                                      size_t workspaceSize, FastFssBatchPlan *plan,
                                                      void *cudaStreamPtr)
{
    if (plan == nullptr || (opNum && ops == nullptr)) return FAST_FSS_RUNTIME_ERROR;
    std::vector<BatchOpDev> dev;
    const int               rc = batch_plan(ops, opNum, tuning, dev, plan);
    if (rc != FAST_FSS_SUCCESS) return rc;
    if (workspace == nullptr || workspaceSize < FastFss_cuda_batchWorkspaceSize(dev.size()))
        return FAST_FSS_RUNTIME_ERROR;
    if (dev.empty()) return FAST_FSS_SUCCESS;
    // pageable source: the call returns once the table has been staged, so `dev` may go away
    if (cudaMemcpyAsync((char *)workspace + kBatchHeader, dev.data(), dev.size() * sizeof(BatchOpDev),
                        cudaMemcpyHostToDevice, resolve_stream(cudaStreamPtr)) != cudaSuccess)
        return FAST_FSS_RUNTIME_ERROR;
    return FAST_FSS_SUCCESS;
}

extern "C" FAST_FSS_API int FastFss_cuda_batchLaunch(const FastFssBatchPlan *plan, void *workspace,
                                                     size_t workspaceSize, void *cudaStreamPtr)
{
    if (plan == nullptr || workspace == nullptr || workspaceSize < FastFss_cuda_batchWorkspaceSize(plan->opNum))
        return FAST_FSS_RUNTIME_ERROR;
    return batch_launch(plan, reinterpret_cast<const BatchOpDev *>((char *)workspace + kBatchHeader),
                        reinterpret_cast<unsigned long long *>(workspace), resolve_stream(cudaStreamPtr));
}

// ---------------------------------------------------------------------------------------
// No-allocation variant (FastFss_cuda_batchEvalNoAlloc in include/FastFss/b200/batch.h):
// the work queue counter and the descriptor table live in this fixed device array instead of
// a caller workspace. Host code must not use the array's name as a device address; it looks
// the address up once per device with cudaGetSymbolAddress.
// ---------------------------------------------------------------------------------------
static_assert(sizeof(fss::BatchOpDev) == 136, "descriptor size is part of the no-alloc scratch size");

static __device__ __align__(256) unsigned char g_batch_noalloc_scratch[FAST_FSS_BATCH_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void      *g_noalloc_addr[64] = {nullptr};

void *noalloc_scratch_address(int device)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= 64) return nullptr;
    if (g_noalloc_addr[device] == nullptr)
    {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_batch_noalloc_scratch) != cudaSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        g_noalloc_addr[device] = p;
    }
    return g_noalloc_addr[device];
}

} // namespace

extern "C" FAST_FSS_API int FastFss_cuda_batchEvalNoAlloc(const FastFssBatchOp *ops, size_t opNum,
                                                          const FastFssBatchTuning *tuning, void *cudaStreamPtr)
{
    if (opNum > FAST_FSS_BATCH_NOALLOC_MAX_OPS) return FAST_FSS_BATCH_TOO_MANY_OPS_ERROR;
    if (opNum && ops == nullptr) return FAST_FSS_RUNTIME_ERROR;
    std::vector<BatchOpDev> dev;
    FastFssBatchPlan        plan{};
    const int               rc = batch_plan(ops, opNum, tuning, dev, &plan);
    if (rc != FAST_FSS_SUCCESS) return rc;
    if (dev.empty()) return FAST_FSS_SUCCESS;
    unsigned char *scratch = (unsigned char *)noalloc_scratch_address(current_device());
    if (scratch == nullptr) return FAST_FSS_RUNTIME_ERROR;
    cudaStream_t stream = resolve_stream(cudaStreamPtr);
    if (cudaMemcpyAsync(scratch + kBatchHeader, dev.data(), dev.size() * sizeof(BatchOpDev), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess)
        return FAST_FSS_RUNTIME_ERROR;
    // batch_launch resets the queue counter (the first 8 bytes) on the stream before the kernel
    return batch_launch(&plan, reinterpret_cast<const BatchOpDev *>(scratch + kBatchHeader),
                        reinterpret_cast<unsigned long long *>(scratch), stream);
}
