// ---------------------------------------------------------------------------
// bh_trace.cu -- persistent geodesic-tracing kernels for sm_100a.
//
// Work distribution.  A frame is a queue of rays in 8x4-pixel tiles (32
// consecutive ray ids are one tile, so a warp that refills several lanes at
// once gets neighbouring pixels with similar paths).  The grid is persistent:
// blocks_per_SM x SM-count CTAs stay resident and every warp keeps 32 rays in
// registers.  A ray that terminates leaves its lane idle; once at least
// `refillMin` lanes of a warp are idle the warp, in one converged block,
// shades and writes the finished rays and claims new ray ids for all idle
// lanes with a single atomicAdd on the frame's ray counter.  Long photon-ring
// rays therefore no longer hold 31 idle lanes hostage, which is the
// divergence that dominates a one-thread-per-pixel launch.
//
// Families are separate kernels (template), so the step loop has no model
// branch; R = float is the product path, R = double the GPU accuracy oracle.
// ---------------------------------------------------------------------------
#include "bh_integrate.cuh"
#include "bh_post.cuh"
#include "bh_internal.h"
#include "../../include/bh_launch.h"

template <bool STATS>
BH_DEV void write_ray(const TraceParams& P, unsigned rid, int px, int py, const RayResult& t)
{
    f3 hdr = t.accum;
    if (!t.horizon)
    {
        f3 bg = sky_color(t.escDir, P.gCam);
        hdr = v3(hdr.x + bg.x * t.trans, hdr.y + bg.y * t.trans, hdr.z + bg.z * t.trans);
    }
    if (!isfinite(hdr.x) || !isfinite(hdr.y) || !isfinite(hdr.z)) hdr = v3(0.f, 0.f, 0.f);

    const size_t idx = P.dirs ? (size_t)rid : (size_t)py * P.W + px;
    switch (P.outMode)
    {
    case BH_OUT_ACCUM:
    {
        float4* acc = reinterpret_cast<float4*>(P.out);
        float4 pv = acc[idx];
        f3 prev = v3(pv.x, pv.y, pv.z);
        if (!isfinite(prev.x) || !isfinite(prev.y) || !isfinite(prev.z)) prev = hdr;
        f3 c = accum_blend(prev, hdr, P.accumMode, P.sampleIndex);
        acc[idx] = make_float4(c.x, c.y, c.z, 1.f);
        break;
    }
    case BH_OUT_RGBA:
    {
        PostConsts pc{P.exposure, 0.f, 0, P.swapRB};
        reinterpret_cast<uchar4*>(P.out)[idx] = finalize_pixel(hdr, v3(0.f, 0.f, 0.f), pc, px, py);
        break;
    }
    case BH_OUT_HDR:
        reinterpret_cast<float4*>(P.out)[idx] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
        break;
    default:
    {
        BHProbe o;
        o.outcome = t.escaped ? 1 : 0;
        o.cls = (t.trans < 0.5f) ? 1 : (t.horizon ? 0 : 2);
        o.steps = t.steps;
        o.diskSamples = t.tally.samples;
        o.escDir[0] = t.escDir.x; o.escDir[1] = t.escDir.y; o.escDir[2] = t.escDir.z;
        o.trans = t.trans;
        o.accum[0] = t.accum.x; o.accum[1] = t.accum.y; o.accum[2] = t.accum.z;
        o.maxHviol = t.maxHviol;
        o.hdr[0] = hdr.x; o.hdr[1] = hdr.y; o.hdr[2] = hdr.z;
        o.diskR = t.tally.hitR; o.diskG = t.tally.hitG; o.drift = t.drift;
        reinterpret_cast<BHProbe*>(P.out)[idx] = o;
        break;
    }
    }
}

// ray id -> pixel (8x4 tiles, row-major tile order); false when outside the frame
BH_DEV bool ray_pixel(const TraceParams& P, unsigned rid, int& px, int& py)
{
    unsigned tile = rid >> 5, w = rid & 31u;
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

template <class Ray, bool STATS>
__global__ void __launch_bounds__(BH_TRACE_BLOCK)
trace_kernel(const __grid_constant__ TraceParams P)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned FULL = 0xffffffffu;
    Ray ray;
    unsigned rid = 0;
    int px = 0, py = 0;
    bool live = false, pending = false, exhausted = false;

    while (true)
    {
        const unsigned liveMask = __ballot_sync(FULL, live);
        const int nFree = 32 - __popc(liveMask);
        if (liveMask == 0u || (!exhausted && nFree >= P.refillMin))
        {
            if (pending)
            {
                RayResult t;
                ray.result(P, ray_direction(P, rid, px, py), t);
                write_ray<STATS>(P, rid, px, py, t);
                pending = false;
            }
            if (exhausted)
            {
                if (liveMask == 0u) break;
                continue;
            }
            unsigned base = 0;
            if (lane == 0) base = atomicAdd(P.counter, (unsigned)nFree);
            base = __shfl_sync(FULL, base, 0);
            if (!live)
            {
                const unsigned rank = __popc(~liveMask & ((1u << lane) - 1u));
                const unsigned id = base + rank;
                if (id < P.nRays)
                {
                    rid = id;
                    bool inFrame = true;
                    if (!P.dirs) inFrame = ray_pixel(P, rid, px, py);
                    if (inFrame)
                    {
                        int st = ray.init(P, ray_direction(P, rid, px, py));
                        live = (st == RAY_LIVE);
                        pending = (st == RAY_DONE);
                    }
                }
            }
            if (base + (unsigned)nFree >= P.nRays) exhausted = true;
            continue;
        }
        if (live && ray.advance(P))
        {
            live = false;
            pending = true;
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

template <class Ray, bool STATS>
cudaError_t launch_one(const TraceParams& P, int blocksPerSm, cudaStream_t stream)
{
    auto k = trace_kernel<Ray, STATS>;
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, BH_TRACE_BLOCK, 0);
    if (e != cudaSuccess) return e;
    if (occ < 1) occ = 1;
    int per = (blocksPerSm > 0 && blocksPerSm < occ) ? blocksPerSm : occ;
    long long need = ((long long)P.nRays + BH_TRACE_BLOCK - 1) / BH_TRACE_BLOCK;
    long long grid = (long long)per * sms;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    k<<<(unsigned)grid, BH_TRACE_BLOCK, 0, stream>>>(P);
    return cudaGetLastError();
}

}  // namespace

cudaError_t bh_launch_trace(const TraceParams& P, int precision, bool stats, int blocksPerSm,
                            cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(P.counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    if (P.nRays == 0) return cudaSuccess;
    const bool kerr = (P.model == 2 || P.model == 3);
    const bool dbl = (precision == BH_PREC_FP64);
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
