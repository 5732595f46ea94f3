// ---------------------------------------------------------------------------
// bh_trace.cu -- persistent geodesic-tracing kernels for sm_100a.
//
// Work distribution.  A frame is a queue of rays in 8x4-pixel tiles (32
// consecutive ray ids form one tile, so rays claimed together are
// neighbouring pixels with similar paths).  The grid is persistent: as many
// 128-thread CTAs as fit stay resident on every SM, and each warp keeps 32
// rays in registers.
//
//  * Refill.  When at least `refillMin` lanes of a warp are idle the warp
//    hands them the next ray ids of its private range (one atomicAdd on the
//    frame counter claims a whole 32-ray tile) and initialises them.  Per-ray
//    initialisation is ~30 exact operations because the camera frame is
//    precomputed (CamFrame), so refilling often is cheap.
//  * Deferred shading.  A finished ray does not shade in place (that would run
//    the ~1000-instruction sky model with one lane active): its packed state
//    (key, disk radiance, transmittance and six escape-state values) is stored
//    on a per-warp ring in shared memory and the lane is free at once.
//    Whenever 32 rays are queued the whole warp rebuilds their escape
//    directions and shades them together, one per lane, fully converged.
//
// Families are separate kernels (template), so the step loop has no model
// branch; R = float is the product path, R = double the GPU accuracy oracle.
// ---------------------------------------------------------------------------
#include "bh_integrate.cuh"
#include "bh_post.cuh"
#include "bh_internal.h"
#include "bh_launch.h"

namespace {

constexpr int kQueue = 64;            // ring entries per warp (>= 2 x 32)
constexpr unsigned kChunk = 32;       // ray ids claimed per atomicAdd (one tile)

template <class R, bool STATS, int NW> struct Queue;
template <class R, int NW> struct Queue<R, false, NW> { PackedRay<R> s[NW][kQueue]; };
template <class R, int NW> struct Queue<R, true, NW> { PackedRay<R> s[NW][kQueue]; PackedStats t[NW][kQueue]; };

// ray id -> pixel (8x4 tiles, row-major tile order); false when outside the frame
BH_DEV bool ray_pixel(const TraceParams& P, unsigned rid, int& px, int& py)
{
    if (P.pixList)
    {   // BH_PIX_SKIP entries pad a list group: no ray
        const unsigned pix = __ldg(P.pixList + rid);
        py = (int)(pix / (unsigned)P.W);
        px = (int)(pix - (unsigned)py * (unsigned)P.W);
        return pix != BH_PIX_SKIP;
    }
    unsigned tile = rid >> 5, w = rid & 31u;
    if (P.tileOrder) tile = __ldg(P.tileOrder + tile);
    px = (int)((tile % (unsigned)P.tilesX) * 8u + (w & 7u));
    py = (int)((tile / (unsigned)P.tilesX) * 4u + (w >> 3));
    return px < P.W && py < P.H;
}

BH_DEV f3 ray_direction(const TraceParams& P, unsigned rid, int px, int py)
{
    if (P.dirs)
    {
        float3 d = P.dirs[rid];
        return v3(d.x, d.y, d.z);
    }
    float fx = __fdiv_rn(add_x((float)px, P.jx), (float)P.W);
    float fy = __fdiv_rn(add_x((float)py, P.jy), (float)P.H);
    return camera_ray(P, fx, fy);
}

// Shade one queued ray (sky behind it) and write it in the output mode.
template <class Ray, bool STATS>
BH_DEV void shade_slot(const TraceParams& P, const PackedRay<typename Ray::Real>& q, const PackedStats* qs)
{
    const bool horizon = (q.key & kRayHorizon) != 0u, escaped = (q.key & kRayEscaped) != 0u;
    const unsigned key = q.key & kRayKeyMask;     // pixel index; the list position in anchor mode
    int px = 0, py = 0;
    if (!P.dirs)
    {
        const unsigned pix = (P.outMode == BH_OUT_ANCHOR) ? __ldg(P.pixList + key) : key;
        py = (int)(pix / (unsigned)P.W);
        px = (int)(pix - (unsigned)py * (unsigned)P.W);
    }
    f3 esc = v3(0.f, 0.f, 0.f);
    if (escaped)
        esc = (q.key & kRayUseState) ? Ray::escape_dir(P, q) : ray_direction(P, key, px, py);
    f3 hdr = v3(q.acc[0], q.acc[1], q.acc[2]);
    if (!horizon)
    {
        f3 bg = sky_color(esc, P.gCam);
        hdr = v3(hdr.x + bg.x * q.trans, hdr.y + bg.y * q.trans, hdr.z + bg.z * q.trans);
    }
    if (!isfinite(hdr.x) || !isfinite(hdr.y) || !isfinite(hdr.z)) hdr = v3(0.f, 0.f, 0.f);

    switch (P.outMode)
    {
    case BH_OUT_ACCUM:
    {
        float4* acc = reinterpret_cast<float4*>(P.out);
        float4 pv = acc[key];
        f3 prev = v3(pv.x, pv.y, pv.z);
        if (!isfinite(prev.x) || !isfinite(prev.y) || !isfinite(prev.z)) prev = hdr;
        f3 c = accum_blend(prev, hdr, P.accumMode, P.sampleIndex);
        acc[key] = make_float4(c.x, c.y, c.z, 1.f);
        break;
    }
    case BH_OUT_RGBA:
    {
        PostConsts pc{P.exposure, 0.f, 0, P.swapRB};
        reinterpret_cast<uchar4*>(P.out)[key] = finalize_pixel(hdr, v3(0.f, 0.f, 0.f), pc, px, py);
        break;
    }
    case BH_OUT_HDR:
        reinterpret_cast<float4*>(P.out)[key] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
        break;
    case BH_OUT_ANCHOR:
    {
        BHAnchor a;
        a.escDir = make_float3(esc.x, esc.y, esc.z);
        const bool disk = q.trans < 1.f || q.acc[0] > 0.f || q.acc[1] > 0.f || q.acc[2] > 0.f;
        a.flags = (escaped ? BH_ANCHOR_ESCAPED : 0u) | (horizon ? BH_ANCHOR_HORIZON : 0u) | (disk ? BH_ANCHOR_DISK : 0u) |
                  ((q.key & kRayExhausted) ? BH_ANCHOR_INCOMPLETE : 0u);
        a.hdr = make_float3(hdr.x, hdr.y, hdr.z);
        a.trans = q.trans;
        reinterpret_cast<BHAnchor*>(P.out)[P.outIndex ? __ldg(P.outIndex + key) : key] = a;
        break;
    }
    default:
    {
        BHProbe o;
        o.outcome = escaped ? 1 : 0;
        o.cls = (q.trans < 0.5f) ? 1 : (horizon ? 0 : 2);
        o.steps = STATS ? qs->steps : 0;
        o.diskSamples = STATS ? qs->samples : 0;
        if (!escaped) esc = ray_direction(P, key, px, py);   // reference keeps the initial direction
        o.escDir[0] = esc.x; o.escDir[1] = esc.y; o.escDir[2] = esc.z;
        o.trans = q.trans;
        o.accum[0] = q.acc[0]; o.accum[1] = q.acc[1]; o.accum[2] = q.acc[2];
        o.maxHviol = STATS ? qs->maxHviol : 0.f;
        o.hdr[0] = hdr.x; o.hdr[1] = hdr.y; o.hdr[2] = hdr.z;
        o.diskR = STATS ? qs->hitR : 0.f;
        o.diskG = STATS ? qs->hitG : 0.f;
        o.drift = STATS ? qs->drift : 0.f;
        reinterpret_cast<BHProbe*>(P.out)[key] = o;
        break;
    }
    }
}

// Block size and register budget (CTAs resident per SM): the spherical FP32
// render kernel fits 72 registers (7 CTAs of 128 threads, 28 warps); the
// Kerr-Newman FP32 kernels need 80 to stay spill-free in the step loop, which
// leaves room for 25 warps: 5 CTAs of 160 threads (6 CTAs of 128 threads hold
// 24; measured 2 % slower on the 4K orbit frames); FP64 and statistics (probe)
// kernels carry more state (4 CTAs of 128).  The runtime may run fewer
// (bhSetTuning).
template <class Ray, bool STATS>
__host__ __device__ constexpr int block_of()
{
    return (Ray::kKerrFamily && sizeof(typename Ray::Real) == 4 && !STATS) ? BH_TRACE_BLOCK_KERR : BH_TRACE_BLOCK;
}

template <class Ray, bool STATS>
__host__ __device__ constexpr int min_blocks()
{
    if (sizeof(typename Ray::Real) != 4 || STATS) return 4;
    return Ray::kKerrFamily ? 5 : BH_TRACE_MIN_BLOCKS;
}

template <class Ray, bool STATS>
__global__ void __launch_bounds__(block_of<Ray, STATS>(), min_blocks<Ray, STATS>())
trace_kernel(const __grid_constant__ TraceParams P)
{
    using R = typename Ray::Real;
    __shared__ Queue<R, STATS, block_of<Ray, STATS>() / 32> Q;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu, below = (1u << lane) - 1u;
    PackedRay<R>* ring = Q.s[warp];

    const unsigned nRays = P.nRaysDev ? min(*P.nRaysDev, P.nRays) : P.nRays;
    Ray ray;
    unsigned rid = 0, key = 0;
    bool live = false;
    unsigned next = 0, end = 0;          // warp-private ray-id range (warp-uniform)
    bool drained = false;                // frame counter exhausted (warp-uniform)
    unsigned qHead = 0, qTail = 0;       // ring cursors (warp-uniform)

    while (true)
    {
        bool fin = false;
        const unsigned liveMask = __ballot_sync(FULL, live);
        const unsigned nFree = 32u - (unsigned)__popc(liveMask);
        const bool haveWork = !drained || next < end;
        if (haveWork && (liveMask == 0u || nFree >= (unsigned)P.refillMin))
        {
            // hand ids to the idle lanes, claiming a new tile if the range runs short
            unsigned avail = end - next, base = 0;
            bool claimed = false;
            if (avail < nFree && !drained)
            {
                if (lane == 0) base = atomicAdd(P.counter, kChunk);
                base = __shfl_sync(FULL, base, 0);
                claimed = true;
                if (base + kChunk >= nRays) drained = true;
            }
            if (!live)
            {
                const unsigned rank = (unsigned)__popc(~liveMask & below);
                unsigned id = (rank < avail) ? next + rank : base + (rank - avail);
                bool valid = (rank < avail) || (claimed && base < nRays);
                if (valid && id < nRays)
                {
                    int px = 0, py = 0;
                    bool inFrame = P.dirs ? true : ray_pixel(P, id, px, py);
                    if (inFrame)
                    {
                        rid = id;
                        key = (P.dirs || P.outMode == BH_OUT_ANCHOR) ? id
                                                                     : (unsigned)py * (unsigned)P.W + (unsigned)px;
                        int st = ray.init(P, ray_direction(P, id, px, py));
                        live = (st == RAY_LIVE);
                        fin = (st == RAY_DONE);
                    }
                }
            }
            if (avail >= nFree) next += nFree;
            else if (claimed && base < nRays)
            {
                end = min(base + kChunk, nRays);
                next = min(base + (nFree - avail), end);
            }
            else next = end;
        }
        else if (liveMask == 0u)
        {
            break;   // no rays left for this warp
        }

        // two steps per scheduling round: halves the ballot / refill bookkeeping
#pragma unroll 1
        for (int k = 0; k < 2; ++k)
            if (live && ray.advance(P)) { live = false; fin = true; }

        const unsigned finMask = __ballot_sync(FULL, fin);
        if (finMask)
        {
            if (fin)
            {
                const unsigned slot = (qTail + (unsigned)__popc(finMask & below)) & (kQueue - 1);
                PackedStats* st = nullptr;
                if constexpr (STATS) st = &Q.t[warp][slot];
                ray.pack(P, key, ring[slot], st);
            }
            qTail += (unsigned)__popc(finMask);
            __syncwarp();
            if (qTail - qHead >= 32u)
            {
                const unsigned slot = (qHead + lane) & (kQueue - 1);
                const PackedStats* qs = nullptr;
                if constexpr (STATS) qs = &Q.t[warp][slot];
                shade_slot<Ray, STATS>(P, ring[slot], qs);
                qHead += 32u;
                __syncwarp();
            }
        }
    }
    // shade what is left in the ring
    __syncwarp();
    if (lane < qTail - qHead)
    {
        const unsigned slot = (qHead + lane) & (kQueue - 1);
        const PackedStats* qs = nullptr;
        if constexpr (STATS) qs = &Q.t[warp][slot];
        shade_slot<Ray, STATS>(P, ring[slot], qs);
    }
}

// ---------------------------------------------------------------------------
// Batched views: one persistent launch over the tiles of many views
// ---------------------------------------------------------------------------
// One tile (32 rays) of one view, traced by a whole warp: tile-synchronous, the
// warp shades its 32 results together once every lane is done.
template <class Ray>
BH_DEV void trace_tile(const TraceParams& P, unsigned tile, unsigned lane, unsigned nRays)
{
    const unsigned rid = tile * 32u + lane;
    int px = 0, py = 0;
    const bool inFrame = rid < nRays && ray_pixel(P, rid, px, py);
    Ray ray;
    bool live = false, fin = false;
    unsigned key = 0;
    if (inFrame)
    {
        key = (P.outMode == BH_OUT_ANCHOR) ? rid : (unsigned)py * (unsigned)P.W + (unsigned)px;
        const int st = ray.init(P, ray_direction(P, rid, px, py));
        live = (st == RAY_LIVE);
        fin = (st == RAY_DONE);
    }
    while (live)
        if (ray.advance(P)) { live = false; fin = true; }
    __syncwarp();
    if (fin)
    {
        PackedRay<typename Ray::Real> q;
        ray.pack(P, key, q, nullptr);
        shade_slot<Ray, false>(P, q, nullptr);
    }
}

// One frame (or one pixel list), tile-synchronous: each warp claims 32 ray
// ids -- one 8x4 tile, or 32 consecutive list entries -- at a time (the
// counter counts tiles) and traces them to the last ray.  This is the FP32
// render path under the default work distribution (a warp refills only when
// all 32 lanes are idle); it skips trace_kernel's per-step ballots and result
// ring.  Plain frames and the surrogate's RK4 pixel lists share this kernel,
// so a pixel traced by either gets the same bits.
template <class Ray>
__global__ void __launch_bounds__(block_of<Ray, false>(), min_blocks<Ray, false>())
tile_kernel(const __grid_constant__ TraceParams P)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned nRays = P.nRaysDev ? min(*P.nRaysDev, P.nRays) : P.nRays;
    const unsigned nTiles = (nRays + 31u) / 32u;
    while (true)
    {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(P.counter, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nTiles) break;
        trace_tile<Ray>(P, t, lane, nRays);
        __syncwarp();
    }
}

// Work queue: tile g of the batch belongs to the last view v with
// tileBase[v] <= g.  A warp claims one tile at a time and copies the view's
// frame constants into shared memory when the view changes.  One kernel per
// metric family, so each runs with its family's register budget.
template <class Ray>
__global__ void __launch_bounds__(block_of<Ray, false>(), min_blocks<Ray, false>())
batch_kernel(const TraceParams* __restrict__ views, const unsigned* __restrict__ tileBase, int n,
             unsigned totalTiles, unsigned* counter)
{
    __shared__ TraceParams sp[block_of<Ray, false>() / 32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    int cur = -1;
    while (true)
    {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(counter, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= totalTiles) break;
        int lo = 0, hi = n;
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (__ldg(tileBase + mid) <= g) lo = mid; else hi = mid;
        }
        if (lo != cur)
        {
            const long long* src = reinterpret_cast<const long long*>(views + lo);
            long long* dst = reinterpret_cast<long long*>(&sp[warp]);
            for (int i = (int)lane; i < (int)(sizeof(TraceParams) / 8); i += 32) dst[i] = __ldg(src + i);
            __syncwarp();
            cur = lo;
        }
        trace_tile<Ray>(sp[warp], g - __ldg(tileBase + lo), lane, sp[warp].nRays);
        __syncwarp();
    }
}
static_assert(sizeof(TraceParams) % 8 == 0, "TraceParams is copied in 8-byte words");

template <class Ray, bool STATS>
cudaError_t launch_one(const TraceParams& P, int blocksPerSm, cudaStream_t stream)
{
    auto k = trace_kernel<Ray, STATS>;
    if constexpr (!STATS && sizeof(typename Ray::Real) == 4)
    {   // whole frames under the default work distribution: tile-synchronous
        if (P.refillMin >= 32 && !P.dirs) k = tile_kernel<Ray>;
    }
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    constexpr int block = block_of<Ray, STATS>();
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, block, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    int per = (blocksPerSm > 0 && blocksPerSm < occ) ? blocksPerSm : occ;
    long long need = ((long long)P.nRays + block - 1) / block;
    long long grid = (long long)per * sms;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, block, 0, stream>>>(P);
    return cudaGetLastError();
}

}  // namespace

cudaError_t bh_launch_trace(const TraceParams& P, int precision, bool stats, int blocksPerSm,
                            cudaStream_t stream)
{
    if (P.nRays > BH_MAX_RAYS || (!P.dirs && (size_t)P.W * (size_t)P.H > (size_t)BH_MAX_RAYS))
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(P.counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    if (P.nRays == 0) return cudaSuccess;
    const bool kerr = (P.model == 2 || P.model == 3);
    const bool dbl = (precision == BH_PREC_FP64);
    if (precision == BH_PREC_MIXED)
    {
        if (kerr) return stats ? launch_one<KerrRay<float, true, true>, true>(P, blocksPerSm, stream)
                               : launch_one<KerrRay<float, false, true>, false>(P, blocksPerSm, stream);
        return stats ? launch_one<SphRay<float, true, true>, true>(P, blocksPerSm, stream)
                     : launch_one<SphRay<float, false, true>, false>(P, blocksPerSm, stream);
    }
    if (kerr)
    {
        if (dbl) return stats ? launch_one<KerrRay<double, true>, true>(P, blocksPerSm, stream)
                              : launch_one<KerrRay<double, false>, false>(P, blocksPerSm, stream);
        return stats ? launch_one<KerrRay<float, true>, true>(P, blocksPerSm, stream)
                     : launch_one<KerrRay<float, false>, false>(P, blocksPerSm, stream);
    }
    if (dbl) return stats ? launch_one<SphRay<double, true>, true>(P, blocksPerSm, stream)
                          : launch_one<SphRay<double, false>, false>(P, blocksPerSm, stream);
    return stats ? launch_one<SphRay<float, true>, true>(P, blocksPerSm, stream)
                 : launch_one<SphRay<float, false>, false>(P, blocksPerSm, stream);
}

cudaError_t bh_launch_batch(bool kerr, const TraceParams* views, const unsigned* tileBase, int n,
                            unsigned totalTiles, unsigned* counter, int blocksPerSm, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess || totalTiles == 0) return e;
    auto k = kerr ? batch_kernel<KerrRay<float, false>> : batch_kernel<SphRay<float, false>>;
    int dev = 0, sms = 0, occ = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int block = kerr ? block_of<KerrRay<float, false>, false>() : block_of<SphRay<float, false>, false>();
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, block, 0)) != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    const int per = (blocksPerSm > 0 && blocksPerSm < occ) ? blocksPerSm : occ;
    long long grid = (long long)per * sms;
    const long long need = ((long long)totalTiles * 32 + block - 1) / block;
    if (grid > need) grid = need;
    k<<<(unsigned)grid, block, 0, stream>>>(views, tileBase, n, totalTiles, counter);
    return cudaGetLastError();
}

cudaError_t bh_trace_max_blocks(int model, int* out)
{
    const bool kerr = (model == 2 || model == 3);
    if (kerr)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, trace_kernel<KerrRay<float, false>, false>,
                                                             block_of<KerrRay<float, false>, false>(), 0);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, trace_kernel<SphRay<float, false>, false>,
                                                         block_of<SphRay<float, false>, false>(), 0);
}
