// ---------------------------------------------------------------------------
// bh_sg_anchor.cu -- resolve pass of the anchored surrogate frame.
//
// An anchored frame traces one pixel in S x S with the FP32 RK4 tracer (the
// anchors, exact pixels of the plain frame) and builds every other pixel of
// a smooth sky region from them:
//   * the escape direction is the Catmull-Rom (bicubic) interpolation of the
//     4 x 4 surrounding anchors' escape directions; its error is bounded by
//     twice the distance between the bicubic and the bilinear interpolants
//     (the bilinear error term dominates the bicubic one wherever the map is
//     smooth), plus a floor of 2e-6 rad;
//   * the pixel is accepted only if all 16 anchors escaped without touching
//     the disk, the optional cell gate (the network's probability that the
//     cell centre escapes without the disk, >= minProb) passes, the bound is below
//     epsMax, and the sky is flat within the bound: either no star of the
//     four star lattices lies within reach of the bound (an exact test on the
//     lattice cells the bound reaches and their stars), or the display values (exposure,
//     ACES, vibrance, gamma, before dither, in byte units) of the sky at the
//     direction and at four directions sqrt(2) bound away differ by less
//     than maxStep; and the pixel stays below the bloom bright-pass
//     threshold, so neither its byte nor its neighbours' bloom can move by
//     a whole step.  The sampled test costs four more sky evaluations and
//     is needed by a minority of pixels scattered over the sky, so the
//     resolve pass defers those pixels to a compact buffer and a second
//     pass (sky_sample_kernel) runs the test on full warps;
//   * the anchors are traced with a step budget that may be below the frame's
//     maxSteps (the few rays that graze the photon sphere set the anchor
//     pass's duration); an anchor that spends it is traced in full on the
//     list, and no pixel interpolates from it;
//   * a pixel whose 16 surrounding anchors were all captured without touching
//     the disk (the inside of the shadow), and whose cell centre the network
//     (when it gates) also calls captured, is black, as a captured sample is;
//   * everything else goes on the RK4 list.
// The sky is the reference's backgroundColor (trace.cuh:166-195) at the
// interpolated direction, times the transmittance 1 of a sky-only ray
// (renderSampleHDR, trace.cuh:908-926).
// No counterpart in the reference.
// ---------------------------------------------------------------------------
#include <algorithm>

#include "bh_integrate.cuh"
#include "bh_post.cuh"
#include "bh_sg_infer.h"

namespace {

constexpr float kLumBloomSafe = 0.9f;     // bright pass starts at 0.95 (post_process.cuh:76-84)

__device__ __forceinline__ void catmull_rom(float t, float w[4])
{
    const float t2 = t * t, t3 = t2 * t;
    w[0] = 0.5f * (-t3 + 2.f * t2 - t);
    w[1] = 0.5f * (3.f * t3 - 5.f * t2 + 2.f);
    w[2] = 0.5f * (-3.f * t3 + 4.f * t2 + t);
    w[3] = 0.5f * (t3 - t2);
}

// display value of one HDR colour before dither and quantisation, in byte units
// (finalize_pixel without bloom and dither: exposure, ACES, vibrance, gamma)
__device__ __forceinline__ f3 display_value(f3 hdr, float exposure)
{
    f3 c = aces_x(v3(hdr.x * exposure, hdr.y * exposure, hdr.z * exposure));
    const float lum = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
    c = v3(clampf(lum + (c.x - lum) * 1.12f, 0.f, 1.f), clampf(lum + (c.y - lum) * 1.12f, 0.f, 1.f),
           clampf(lum + (c.z - lum) * 1.12f, 0.f, 1.f));
    const float g = 1.f / 2.2f;
    return v3(255.f * __powf(c.x, g), 255.f * __powf(c.y, g), 255.f * __powf(c.z, g));
}

__device__ __forceinline__ float lum_exposed(f3 c, float exposure)
{
    return exposure * (0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z);
}

// Is the star of lattice cell `c` (integer coordinates; star_layer draws it only
// inside that cell, where d2 * sharp <= cut) farther than m + its cut radius
// from the point p (cell units)?  fc = p - c.  The cell's star position and
// magnitude use the same exact operations as star_layer.
__device__ __forceinline__ bool cell_star_clear(f3 c, f3 fc, float m, float sharp)
{
    const f3 h = hash33(c);
    const f3 dv = v3(fc.x - (0.10f + 0.80f * h.x), fc.y - (0.10f + 0.80f * h.y), fc.z - (0.10f + 0.80f * h.z));
    const float dist = sqrtf(dot3(dv, dv));
    const float mag = hash12(add_x(c.x, mul_x(91.7f, c.z)), sub_x(c.y, mul_x(33.1f, c.x)));
    const float cut = (mag > 0.9f) ? 60.f : 14.f;
    return dist - m > sqrtf(cut / sharp);
}

// Is one star lattice (trace.cuh:131-164: `cell` cells per unit direction, one
// candidate star per cell, drawn only inside its own cell) free of stars
// everywhere within `r` of the direction d?  Every cell the disc reaches is
// checked: d's own cell and, along each axis whose face lies within the
// margin, the neighbouring cell (up to 8 cells at a corner).  A disc wider than
// half a cell is not cleared.
__device__ __forceinline__ bool star_layer_clear(f3 d, float cell, float sharp, float r)
{
    const f3 p = v3(mul_x(d.x, cell), mul_x(d.y, cell), mul_x(d.z, cell));
    const f3 id = v3(floorf(p.x), floorf(p.y), floorf(p.z));
    const f3 f = v3(sub_x(p.x, id.x), sub_x(p.y, id.y), sub_x(p.z, id.z));
    const float m = 1.5f * r * cell + 1e-5f;     // the offsets reach sqrt(2) r; margin in cell units
    if (m >= 0.5f) return false;
    const int x0 = f.x < m ? -1 : 0, x1 = f.x > 1.f - m ? 1 : 0;
    const int y0 = f.y < m ? -1 : 0, y1 = f.y > 1.f - m ? 1 : 0;
    const int z0 = f.z < m ? -1 : 0, z1 = f.z > 1.f - m ? 1 : 0;
#pragma unroll 1
    for (int dz = z0; dz <= z1; ++dz)
#pragma unroll 1
        for (int dy = y0; dy <= y1; ++dy)
#pragma unroll 1
            for (int dx = x0; dx <= x1; ++dx)
            {
                const f3 c = v3(id.x + (float)dx, id.y + (float)dy, id.z + (float)dz);
                const f3 fc = v3(f.x - (float)dx, f.y - (float)dy, f.z - (float)dz);
                if (!cell_star_clear(c, fc, m, sharp)) return false;
            }
    return true;
}

// No star of the four lattices of backgroundColor within r of d: the rest of the
// sky (Milky-Way band and airglow) varies on scales of 0.1 rad and more.
__device__ __forceinline__ bool stars_clear(f3 d, float r)
{
    return star_layer_clear(d, 80.f, 320.f, r) && star_layer_clear(d, 190.f, 520.f, r) &&
           star_layer_clear(d, 420.f, 820.f, r) && star_layer_clear(d, 900.f, 1500.f, r);
}

__device__ __forceinline__ f3 unit3(f3 v)
{
    const float l = rsqrtf(fmaxf(v.x * v.x + v.y * v.y + v.z * v.z, 1e-30f));
    return v3(v.x * l, v.y * l, v.z * l);
}

// Warp-wide append of one 8x4 tile's pixels that need RK4: a warp with any
// claims a whole 32-entry group of the list, so the tracer's warps (which take
// 32 consecutive entries) trace one tile each, as coherent as in the plain
// frame; lanes without a pixel hold BH_PIX_SKIP.  `traced` counts the pixels.
__device__ __forceinline__ void push_tile(unsigned* list, unsigned* count, unsigned* traced, unsigned pix,
                                          bool want)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return;
    unsigned base = 0;
    if (lane == 0)
    {
        base = atomicAdd(count, 32u);
        atomicAdd(traced, (unsigned)__popc(m));
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    list[base + lane] = want ? pix : BH_PIX_SKIP;
}

// The pixel's sample into the accumulation buffer, blended as the tracer blends it
// (accum_blend: mode 0 replaces, modes 1 and 2 average over the frame sequence).
__device__ __forceinline__ void write_sample(const TraceParams& P, unsigned pix, f3 hdr)
{
    float4* acc = reinterpret_cast<float4*>(P.out);
    if (P.accumMode != 0 && P.sampleIndex > 0)
    {
        const float4 pv = acc[pix];
        f3 prev = v3(pv.x, pv.y, pv.z);
        if (!isfinite(prev.x) || !isfinite(prev.y) || !isfinite(prev.z)) prev = hdr;
        hdr = accum_blend(prev, hdr, P.accumMode, P.sampleIndex);
    }
    acc[pix] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
}

// Warp-wide claim of one slot per lane that wants one (all lanes call it): the
// lanes' slots are consecutive, in lane order, from one atomicAdd on `count`.
__device__ __forceinline__ unsigned warp_claim(unsigned* count, bool want)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (!m) return 0u;
    const unsigned leader = (unsigned)__ffs(m) - 1u;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (unsigned)__popc(m & ((1u << lane) - 1u));
}

// The held-out sample of the interpolated pixels: one in `stride`, hashed per frame.
__device__ __forceinline__ bool held_pick(unsigned pix, unsigned seed, int stride)
{
    if (stride <= 0) return false;
    unsigned h = pix * 0x9E3779B1u ^ (seed * 0x85EBCA77u);
    h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12;
    return (h % (unsigned)stride) == 0u;
}

// Records a held-out pixel and its interpolated HDR (all lanes call it); the
// pixel is traced after the RK4 list and compared (sg_held_compare).
__device__ __forceinline__ void push_held(const SgAnchorFrame& F, unsigned pix, f3 hdr, bool held)
{
    const unsigned k = warp_claim(F.heldCount, held);
    if (held && k < F.heldCap)
    {
        F.heldPix[k] = pix;
        F.heldPred[k] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
    }
}

// Per-frame tallies (all lanes call it): interpolated pixels, and the
// rejection reason (1..3) of the traced ones.
__device__ __forceinline__ void tally(unsigned* stats, bool resolved, int reason)
{
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        const unsigned m = __ballot_sync(0xffffffffu, k == 0 ? resolved : reason == k);
        if (lane == 0 && m) atomicAdd(stats + k, (unsigned)__popc(m));
    }
}

// anchors a 32 x 8 pixel block can reach: columns x0/S - 1 .. (x0+31)/S + 2, rows
// y0/S - 1 .. (y0+7)/S + 2 (at most 19 x 8 for S >= 2)
constexpr int kAncCols = 19, kAncRows = 8;

// One thread per pixel; 2-D blocks of 32 x 8 pixels, each warp one 8 x 4 tile
// (4 tiles across, 2 down).
// The block's anchors (escape direction and flags) are staged in shared memory
// once; each pixel then reads its 4 x 4 neighbourhood from there.
__global__ void __launch_bounds__(256, 4) anchor_resolve_kernel(const __grid_constant__ SgAnchorFrame F)
{
    __shared__ float4 sAnc[kAncRows][kAncCols];
    const TraceParams& P = F.tp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // blocks run nearest the screen centre first, so the list's first tiles hold the
    // long rays around the shadow and the tracer does not end on them
    const unsigned blk = F.blockOrder ? __ldg(F.blockOrder + blockIdx.x) : blockIdx.x;
    const unsigned bxs = (unsigned)(P.W + 31) / 32u;
    const int bx = (int)(blk % bxs), by = (int)(blk / bxs);
    const int x = bx * 32 + (warp & 3) * 8 + (lane & 7), y = by * 8 + (warp >> 2) * 4 + (lane >> 3);
    const bool inFrame = x < P.W && y < P.H;
    const int S = F.S;
    const unsigned pix = inFrame ? (unsigned)y * (unsigned)P.W + (unsigned)x : 0u;
    const int ax0 = (bx * 32) / S - 1, ay0 = (by * 8) / S - 1;
    for (int i = threadIdx.x; i < kAncRows * kAncCols; i += blockDim.x)
    {
        const int r = i / kAncCols, c = i - r * kAncCols;
        const int ax = ax0 + c, ay = ay0 + r;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ax >= 0 && ay >= 0 && ax < F.nx && ay < F.ny)
        {
            const BHAnchor& a = F.anchors[ay * F.nx + ax];
            v = make_float4(a.escDir.x, a.escDir.y, a.escDir.z, __uint_as_float(a.flags));
        }
        sAnc[r][c] = v;
    }
    __syncthreads();

    bool anchor = false, resolved = false, defer = false, incomplete = false;
    f3 hdr = v3(0.f, 0.f, 0.f);
    float4 dir = make_float4(0.f, 0.f, 0.f, 0.f);
    int reason = 0;                   // 1 anchors / cell gate, 2 error bound, 3 sky sensitivity, 4 deferred
    if (inFrame)
    {
        const int cx = x / S, cy = y / S;
        if (x == cx * S && y == cy * S)
        {   // an anchor: its own RK4 sample, unless the anchor pass's step budget ran out
            const BHAnchor& a = F.anchors[cy * F.nx + cx];
            hdr = v3(a.hdr.x, a.hdr.y, a.hdr.z);
            incomplete = (a.flags & BH_ANCHOR_INCOMPLETE) != 0u;
            anchor = !incomplete;
            reason = incomplete ? 1 : 0;
        }
        else if (cx >= 1 && cy >= 1 && cx + 2 < F.nx && cy + 2 < F.ny)
        {
            bool sky = true, dark = true;
            if (F.cellGate)
            {   // the network's class probabilities at the cell centre
                const float2 g = F.cellGate[cy * (F.nx - 1) + cx];
                sky = g.x >= F.minProb;
                dark = g.y >= F.minProb;
            }
            // anchor (cx - 1 + i, cy - 1 + j) is staged at sAnc[cy - 1 + j - ay0][cx - 1 + i - ax0];
            // the flags first, the directions re-read from shared memory where needed (keeps
            // the 16 directions out of registers)
            const float4(*st)[kAncCols] = reinterpret_cast<const float4(*)[kAncCols]>(&sAnc[cy - 1 - ay0][0]);
            const int c0i = cx - 1 - ax0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                {
                    const unsigned fl = __float_as_uint(st[j][c0i + i].w);
                    sky = sky && fl == BH_ANCHOR_ESCAPED;
                    dark = dark && fl == BH_ANCHOR_HORIZON;
                }
            reason = 1;
            if (dark)
            {   // inside the shadow: all 16 anchors captured without touching the disk, and a
                // captured ray's sample is exactly zero (renderSampleHDR, trace.cuh:916-921)
                hdr = v3(0.f, 0.f, 0.f);
                resolved = true;
                reason = 0;
            }
            else if (sky)
            {
                const float tx = (float)(x - cx * S) / (float)S, ty = (float)(y - cy * S) / (float)S;
                float wx[4], wy[4];
                catmull_rom(tx, wx);
                catmull_rom(ty, wy);
                f3 bc = v3(0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                    {
                        const float w = wy[j] * wx[i];
                        const float4 a = st[j][c0i + i];
                        bc = v3(bc.x + w * a.x, bc.y + w * a.y, bc.z + w * a.z);
                    }
                const float4 a11 = st[1][c0i + 1], a12 = st[1][c0i + 2], a21 = st[2][c0i + 1], a22 = st[2][c0i + 2];
                const f3 top = v3(a11.x + tx * (a12.x - a11.x), a11.y + tx * (a12.y - a11.y),
                                  a11.z + tx * (a12.z - a11.z));
                const f3 bot = v3(a21.x + tx * (a22.x - a21.x), a21.y + tx * (a22.y - a21.y),
                                  a21.z + tx * (a22.z - a21.z));
                const f3 bl = unit3(v3(top.x + ty * (bot.x - top.x), top.y + ty * (bot.y - top.y),
                                       top.z + ty * (bot.z - top.z)));
                bc = unit3(bc);
                const f3 df = v3(bc.x - bl.x, bc.y - bl.y, bc.z - bl.z);
                const float eps = 2.f * sqrtf(df.x * df.x + df.y * df.y + df.z * df.z) + 2e-6f;
                reason = 2;
                if (eps <= F.epsMax)
                {
                    const f3 c0 = sky_color(bc, P.gCam);
                    reason = 3;
                    if (lum_exposed(c0, P.exposure) < kLumBloomSafe && isfinite(c0.x) && isfinite(c0.y) &&
                        isfinite(c0.z))
                    {
                        if (stars_clear(normalize_x(bc), eps))
                        {   // no star within reach: flat without sampling (the common case)
                            hdr = c0;
                            resolved = true;
                            reason = 0;
                        }
                        else
                        {
                            defer = true;
                            dir = make_float4(bc.x, bc.y, bc.z, eps);
                            reason = 4;
                        }
                    }
                }
            }
        }
        else reason = 1;
    }
    if (anchor || resolved) write_sample(P, pix, hdr);

    // deferred pixels to the sample buffer; beyond its capacity they are traced
    const unsigned k = warp_claim(F.sampleCount, defer);
    if (defer && k < F.sampleCap)
    {
        F.sampleDir[k] = dir;
        F.samplePix[k] = pix;
    }
    else if (defer) reason = 3;
    const bool trace = inFrame && !anchor && !resolved && reason != 4;
    push_tile(F.list, F.listCount, F.stats + 4, pix, trace);   // held-out pixels: traced from heldPix
    push_held(F, pix, hdr, resolved && held_pick(pix, F.frameSeed, F.heldStride));
    tally(F.stats, inFrame && !anchor && resolved, inFrame && !anchor ? reason : 0);
    const unsigned mi = __ballot_sync(0xffffffffu, incomplete);
    if (lane == 0 && mi) atomicAdd(F.stats + 7, (unsigned)__popc(mi));
}

// Second pass over the deferred pixels: the sampled flatness test, one pixel per
// thread.  A flat pixel is written as in the resolve pass; the others are
// appended to the RK4 list one by one (after the resolve pass's whole tiles).
__global__ void __launch_bounds__(256) sky_sample_kernel(const __grid_constant__ SgAnchorFrame F)
{
    const TraceParams& P = F.tp;
    const unsigned n = min(*F.sampleCount, F.sampleCap);
    const unsigned lane = threadIdx.x & 31u;
    for (unsigned base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x)
    {
        const unsigned k = base + threadIdx.x;
        const bool valid = k < n;
        bool flat = false;
        f3 c0 = v3(0.f, 0.f, 0.f);
        unsigned pix = 0;
        if (valid)
        {
            const float4 e = F.sampleDir[k];
            pix = F.samplePix[k];
            const f3 bc = v3(e.x, e.y, e.z);
            const float eps = e.w;
            c0 = sky_color(bc, P.gCam);
            const f3 y0 = display_value(c0, P.exposure);
            // two unit vectors orthogonal to the direction
            const f3 ref = fabsf(bc.y) < 0.9f ? v3(0.f, 1.f, 0.f) : v3(1.f, 0.f, 0.f);
            const f3 u = unit3(v3(ref.y * bc.z - ref.z * bc.y, ref.z * bc.x - ref.x * bc.z,
                                  ref.x * bc.y - ref.y * bc.x));
            const f3 v = v3(bc.y * u.z - bc.z * u.y, bc.z * u.x - bc.x * u.z, bc.x * u.y - bc.y * u.x);
            const float r = 1.41421356f * eps;
            flat = true;
#pragma unroll 1
            for (int j = 0; j < 4 && flat; ++j)
            {
                const float su = (j == 0) ? r : (j == 1 ? -r : 0.f);
                const float sv = (j == 2) ? r : (j == 3 ? -r : 0.f);
                const f3 dk = unit3(v3(bc.x + su * u.x + sv * v.x, bc.y + su * u.y + sv * v.y,
                                       bc.z + su * u.z + sv * v.z));
                const f3 ck = sky_color(dk, P.gCam);
                const f3 yk = display_value(ck, P.exposure);
                flat = lum_exposed(ck, P.exposure) < kLumBloomSafe && fabsf(yk.x - y0.x) < F.maxStep &&
                       fabsf(yk.y - y0.y) < F.maxStep && fabsf(yk.z - y0.z) < F.maxStep;
            }
            if (flat) write_sample(P, pix, c0);
        }
        const bool trace = valid && !flat;
        const unsigned m = __ballot_sync(0xffffffffu, trace);
        const unsigned slot = warp_claim(F.listCount, trace);
        if (trace) F.list[slot] = pix;
        if (lane == 0 && m) atomicAdd(F.stats + 4, (unsigned)__popc(m));
        push_held(F, pix, c0, flat && held_pick(pix, F.frameSeed, F.heldStride));
        tally(F.stats, flat, trace ? 3 : 0);
    }
}

}  // namespace

cudaError_t sg_anchor_resolve(const SgAnchorFrame& F, cudaStream_t s)
{
    const TraceParams& P = F.tp;
    if (F.S < 2 || F.nx < 1 || F.ny < 1) return cudaErrorInvalidValue;
    const unsigned blocks = (unsigned)((P.W + 31) / 32) * (unsigned)((P.H + 7) / 8);
    anchor_resolve_kernel<<<blocks, 256, 0, s>>>(F);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || F.sampleCap == 0) return e;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned sBlocks = std::min((F.sampleCap + 255u) / 256u, (unsigned)sms * 8u);
    sky_sample_kernel<<<sBlocks, 256, 0, s>>>(F);
    return cudaGetLastError();
}
