// ---------------------------------------------------------------------------
// bh_batch.cpp -- many views in one persistent launch, its CUDA-graph form,
// and the autotuner of the tracing kernels' work distribution.
//
// No counterpart in the reference, which renders one view per call
// (src/black_hole_kernel.cu:108-134).  A batch is equivalent to calling
// launchRenderPipeline for every view in turn: same sanitising, same images.
// What changes is scheduling: the 8x4-pixel tiles of all views of a metric
// family go into one device work queue, traced by one persistent kernel
// (bh_trace.cu, batch_kernel), so small and large views share the GPU with no
// per-view launch gaps or tails.  Two launches per batch (Kerr family, then
// the spherical metrics), each with its family's register budget; the gap
// between them is one tile's duration.  Within a family views are queued by
// pixel count, largest first, so each queue ends on cheap tiles.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "bh_launch.h"
#include "bh_internal.h"

namespace {

bool isKerrModel(int m) { return m == BH_KERR || m == BH_KERR_NEWMAN; }

struct Plan
{
    std::vector<int> order;               // trace position -> view index (Kerr family first)
    std::vector<RenderParams> params;     // sanitised, by view index
    std::vector<TraceParams> table;       // trace order
    std::vector<unsigned> base;           // per family, tile prefix sums: nKerr + 1, then nSph + 1
    int nKerr = 0;
};

cudaError_t checkView(const BHView& v, const RenderParams& P)
{
    if (!v.out || !v.accum) return cudaErrorInvalidValue;
    if (P.bloomEnabled && !v.bloomB) return cudaErrorInvalidValue;
    return cudaSuccess;
}

// Sanitise every view and lay out the work queue.  With `keepOrder` the trace
// order of a previous plan is reused (graph updates keep their layout).
cudaError_t makePlan(const BHView* views, int n, Plan& pl, bool keepOrder)
{
    if (n < 0 || (n > 0 && !views)) return cudaErrorInvalidValue;
    pl.params.resize(n);
    for (int i = 0; i < n; ++i)
    {
        pl.params[i] = views[i].params;
        bhSanitizeRenderParams(&pl.params[i]);
        cudaError_t e = checkView(views[i], pl.params[i]);
        if (e != cudaSuccess) return e;
        if ((size_t)pl.params[i].width * (size_t)pl.params[i].height > (size_t)BH_MAX_RAYS)
            return cudaErrorInvalidValue;
    }
    if (!keepOrder)
    {
        pl.order.resize(n);
        for (int i = 0; i < n; ++i) pl.order[i] = i;
        auto key = [&](int i) {
            const RenderParams& P = pl.params[i];
            return (isKerrModel(P.model) ? 1e12 : 0.0) + (double)P.width * P.height;
        };
        std::stable_sort(pl.order.begin(), pl.order.end(), [&](int a, int b) { return key(a) > key(b); });
    }
    pl.nKerr = 0;
    for (int k = 0; k < n; ++k) pl.nKerr += isKerrModel(pl.params[pl.order[k]].model) ? 1 : 0;
    for (int k = 0; k < n; ++k)   // a kept order must still put the Kerr family first
        if (isKerrModel(pl.params[pl.order[k]].model) != (k < pl.nKerr)) return cudaErrorInvalidValue;
    pl.table.resize(n);
    pl.base.assign(n + 2, 0u);
    for (int k = 0; k < n; ++k)
    {
        const int i = pl.order[k];
        TraceParams t = bh_frame_params(pl.params[i], BH_OUT_ACCUM, views[i].accum);
        t.tileOrder = nullptr;
        t.counter = nullptr;
        pl.table[k] = t;
        const unsigned tiles = (unsigned)t.tilesX * (unsigned)((t.H + 3) / 4);
        const int b = k < pl.nKerr ? k : k + 1;   // the spherical prefix sums start at nKerr + 1
        pl.base[b + 1] = pl.base[b] + tiles;
    }
    return cudaSuccess;
}

cudaError_t launchPlan(const Plan& pl, const BHView* views, const TraceParams* dTable, const unsigned* dBase,
                       unsigned* counter, cudaStream_t s)
{
    const int n = (int)pl.table.size(), nK = pl.nKerr, nS = n - nK;
    int blocksK = 0, blocksS = 0;
    bhGetTuning(1, nullptr, &blocksK);
    bhGetTuning(0, nullptr, &blocksS);
    cudaError_t e = cudaSuccess;
    if (nK > 0 && (e = bh_launch_batch(true, dTable, dBase, nK, pl.base[nK], counter, blocksK, s)) != cudaSuccess)
        return e;
    if (nS > 0 && (e = bh_launch_batch(false, dTable + nK, dBase + nK + 1, nS, pl.base[n + 1], counter, blocksS,
                                       s)) != cudaSuccess)
        return e;
    for (int i = 0; i < n; ++i)
    {
        const RenderParams& P = pl.params[i];
        PostConsts pc{P.exposure, P.bloomStrength, P.bloomEnabled ? 1 : 0, P.swapRB};
        e = bh_launch_post(views[i].out, views[i].accum, views[i].bloomB, views[i].bloomA, P.width, P.height, pc, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// per-device tables of the immediate-mode batch (grown on demand)
constexpr int kMaxDevices = 64;
struct DevTables
{
    TraceParams* table = nullptr;
    unsigned* base = nullptr;
    size_t cap = 0;
};
std::mutex gLock;
DevTables gTables[kMaxDevices];

cudaError_t ensureTables(int n, DevTables** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    DevTables& t = gTables[dev];
    if (t.cap < (size_t)n)
    {
        if (t.table) cudaFree(t.table);
        if (t.base) cudaFree(t.base);
        t.table = nullptr;
        t.base = nullptr;
        t.cap = 0;
        size_t cap = std::max<size_t>(64, (size_t)n);
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&t.table), cap * sizeof(TraceParams))) != cudaSuccess) return e;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&t.base), (cap + 2) * sizeof(unsigned))) != cudaSuccess) return e;
        t.cap = cap;
    }
    *out = &t;
    return cudaSuccess;
}

}  // namespace

// ---------------------------------------------------------------------------
// immediate mode
// ---------------------------------------------------------------------------
extern "C" cudaError_t bhRenderBatch(const BHView* views, int n, cudaStream_t stream)
{
    Plan pl;
    cudaError_t e = makePlan(views, n, pl, false);
    if (e != cudaSuccess || n == 0) return e;
    std::lock_guard<std::mutex> g(gLock);
    DevTables* t = nullptr;
    if ((e = ensureTables(n, &t)) != cudaSuccess) return e;
    unsigned* counter = nullptr;
    if ((e = bh_device_counter(&counter)) != cudaSuccess) return e;
    // pageable sources: the copies are staged before the calls return
    if ((e = cudaMemcpyAsync(t->table, pl.table.data(), n * sizeof(TraceParams), cudaMemcpyHostToDevice, stream)))
        return e;
    if ((e = cudaMemcpyAsync(t->base, pl.base.data(), (n + 2) * sizeof(unsigned), cudaMemcpyHostToDevice, stream)))
        return e;
    return launchPlan(pl, views, t->table, t->base, counter, stream);
}

// ---------------------------------------------------------------------------
// CUDA-graph mode
// ---------------------------------------------------------------------------
struct BHBatchGraph
{
    int device = 0, n = 0;
    std::vector<BHView> views;
    Plan plan;
    TraceParams* dTable = nullptr;
    unsigned* dBase = nullptr;
    unsigned* dCounter = nullptr;
    unsigned char* hPinned = nullptr;     // table + base, the graph's copy source
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
};

namespace {

void stage(BHBatchGraph& G)
{
    const size_t tb = G.n * sizeof(TraceParams);
    std::copy(reinterpret_cast<const unsigned char*>(G.plan.table.data()),
              reinterpret_cast<const unsigned char*>(G.plan.table.data()) + tb, G.hPinned);
    std::copy(reinterpret_cast<const unsigned char*>(G.plan.base.data()),
              reinterpret_cast<const unsigned char*>(G.plan.base.data()) + (G.n + 2) * sizeof(unsigned),
              G.hPinned + tb);
}

void release(BHBatchGraph* G)
{
    if (!G) return;
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    if (G->done) cudaEventDestroy(G->done);
    if (G->dTable) cudaFree(G->dTable);
    if (G->dBase) cudaFree(G->dBase);
    if (G->dCounter) cudaFree(G->dCounter);
    if (G->hPinned) cudaFreeHost(G->hPinned);
    delete G;
}

}  // namespace

extern "C" cudaError_t bhBatchGraphCreate(BHBatchGraph** out, const BHView* views, int n)
{
    if (!out || n <= 0 || !views) return cudaErrorInvalidValue;
    *out = nullptr;
    BHBatchGraph* G = new BHBatchGraph();
    G->n = n;
    G->views.assign(views, views + n);
    cudaError_t e = makePlan(views, n, G->plan, false);
    cudaStream_t s = nullptr;
    const size_t tb = n * sizeof(TraceParams), bb = (n + 2) * sizeof(unsigned);
    if (e == cudaSuccess) e = cudaGetDevice(&G->device);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&G->dTable), tb);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&G->dBase), bb);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&G->dCounter), 256);
    if (e == cudaSuccess) e = cudaMallocHost(&G->hPinned, tb + bb);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&G->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) { release(G); if (s) cudaStreamDestroy(s); return e; }
    stage(*G);
    e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess)
    {
        cudaError_t le = cudaMemcpyAsync(G->dTable, G->hPinned, tb, cudaMemcpyHostToDevice, s);
        if (le == cudaSuccess) le = cudaMemcpyAsync(G->dBase, G->hPinned + tb, bb, cudaMemcpyHostToDevice, s);
        if (le == cudaSuccess) le = launchPlan(G->plan, views, G->dTable, G->dBase, G->dCounter, s);
        e = cudaStreamEndCapture(s, &G->graph);
        if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&G->exec, G->graph, 0);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) { release(G); return e; }
    *out = G;
    return cudaSuccess;
}

extern "C" cudaError_t bhBatchGraphUpdate(BHBatchGraph* G, const BHView* views, int n)
{
    if (!G || n != G->n || !views) return cudaErrorInvalidValue;
    for (int i = 0; i < n; ++i)
    {
        const BHView &a = G->views[i], &b = views[i];
        if (a.out != b.out || a.accum != b.accum || a.bloomA != b.bloomA || a.bloomB != b.bloomB ||
            a.params.width != b.params.width || a.params.height != b.params.height ||
            a.params.bloomEnabled != b.params.bloomEnabled)
            return cudaErrorInvalidValue;
    }
    Plan pl;
    pl.order = G->plan.order;
    cudaError_t e = makePlan(views, n, pl, true);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < n; ++i)   // post-processing constants are baked into the graph
    {
        const RenderParams &p0 = G->plan.params[i], &p1 = pl.params[i];
        if (p0.exposure != p1.exposure || p0.bloomStrength != p1.bloomStrength || p0.swapRB != p1.swapRB)
            return cudaErrorInvalidValue;
    }
    if ((e = cudaEventSynchronize(G->done)) != cudaSuccess) return e;   // last replay done with hPinned
    G->plan = pl;
    stage(*G);
    return cudaSuccess;
}

extern "C" cudaError_t bhBatchGraphLaunch(BHBatchGraph* G, cudaStream_t stream)
{
    if (!G) return cudaErrorInvalidValue;
    cudaError_t e = cudaGraphLaunch(G->exec, stream);
    if (e != cudaSuccess) return e;
    return cudaEventRecord(G->done, stream);
}

extern "C" void bhBatchGraphDestroy(BHBatchGraph* G)
{
    if (G && G->done) cudaEventSynchronize(G->done);
    release(G);
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
extern "C" cudaError_t bhAutotune(const RenderParams& p, int* refillMin, int* blocksPerSm, int* tileOrder,
                                  float* bestMs)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    const int family = isKerrModel(P.model) ? 1 : 0;
    int maxBlocks = 0;
    cudaError_t e = bh_trace_max_blocks(P.model, &maxBlocks);
    if (e != cudaSuccess) return e;
    float4* hdr = nullptr;
    if ((e = bh_device_alloc(reinterpret_cast<void**>(&hdr), (size_t)P.width * P.height * sizeof(float4))) != cudaSuccess) return e;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int keepR = 32, keepB = 0;
    bhGetTuning(family, &keepR, &keepB);
    const int keepO = bhGetTileOrder();
    float best = 1e30f;
    int bR = keepR, bB = keepB, bO = keepO;
    const int refills[] = {8, 16, 32};
    for (int order = 0; order <= 1 && e == cudaSuccess; ++order)
        for (int blocks = maxBlocks; blocks >= std::max(1, maxBlocks - 2) && e == cudaSuccess; --blocks)
            for (int refill : refills)
            {
                bhSetTuning(family, refill, blocks);
                bhSetTileOrder(order);
                float ms = 1e30f;
                for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep)
                {
                    cudaEventRecord(e0, s);
                    e = bhRenderHDR(hdr, P, BH_PREC_FP32, s);
                    cudaEventRecord(e1, s);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float t = 0.f;
                    cudaEventElapsedTime(&t, e0, e1);
                    if (rep > 0) ms = std::min(ms, t);   // first launch is the warm-up
                }
                if (e != cudaSuccess) break;
                if (ms < best) { best = ms; bR = refill; bB = blocks; bO = order; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    cudaFree(hdr);
    if (e != cudaSuccess)
    {
        bhSetTuning(family, keepR, keepB);
        bhSetTileOrder(keepO);
        return e;
    }
    bhSetTuning(family, bR, bB);
    bhSetTileOrder(bO);
    if (refillMin) *refillMin = bR;
    if (blocksPerSm) *blocksPerSm = bB;
    if (tileOrder) *tileOrder = bO;
    if (bestMs) *bestMs = best;
    return cudaSuccess;
}

extern "C" cudaError_t bhAutotuneBatch(const BHView* views, int n, int* blocksKerr, int* blocksSph, float* bestMs)
{
    Plan pl;
    cudaError_t e = makePlan(views, n, pl, false);
    if (e != cudaSuccess) return e;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return e;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.f;
    for (int family = 1; family >= 0 && e == cudaSuccess; --family)
    {
        std::vector<BHView> sub;
        for (int k = 0; k < n; ++k)
            if ((k < pl.nKerr) == (family == 1)) sub.push_back(views[pl.order[k]]);
        if (sub.empty()) continue;
        int maxBlocks = 0, keepR = 32, keepB = 0;
        if ((e = bh_trace_max_blocks(family ? BH_KERR : BH_SCHWARZSCHILD, &maxBlocks)) != cudaSuccess) break;
        bhGetTuning(family, &keepR, &keepB);
        float best = 1e30f;
        int bestB = keepB;
        for (int blocks = maxBlocks; blocks >= std::max(1, maxBlocks - 2) && e == cudaSuccess; --blocks)
        {
            bhSetTuning(family, keepR, blocks);
            float ms = 1e30f;
            for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep)
            {
                cudaEventRecord(e0, s);
                e = bhRenderBatch(sub.data(), (int)sub.size(), s);
                cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                if (rep > 0) ms = std::min(ms, t);   // first launch is the warm-up
            }
            if (e == cudaSuccess && ms < best) { best = ms; bestB = blocks; }
        }
        bhSetTuning(family, keepR, e == cudaSuccess ? bestB : keepB);
        if (e != cudaSuccess) break;
        total += best;
        if (family == 1 && blocksKerr) *blocksKerr = bestB;
        if (family == 0 && blocksSph) *blocksSph = bestB;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (e == cudaSuccess && bestMs) *bestMs = total;
    return e;
}
