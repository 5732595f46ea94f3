/*
 * ref_host.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference renderer's own device headers (src/trace.cuh,
 * src/metric.cuh, src/post_process.cuh of Sqhh99/Black-hole) as host C++,
 * unmodified, from where they lie in the reference tree (see oracle/Makefile;
 * the output goes to oracle/_ref/ and is never committed).  The only shim is
 * a host definition of rsqrtf, which CUDA declares for device code only.
 *
 * The functions below are OpenMP pixel loops that restate the bodies of the
 * reference kernels (src/black_hole_kernel.cu:22-103, 140-149 and the test
 * probe tests/test_main.cu:71-89) with the logic unchanged; all physics and
 * post-processing is the reference's code.  This library is the CPU
 * "reference" arm of the benchmark and pins the restated oracle
 * (oracle/bh_oracle.cpp) to the reference bit for bit.
 */
#include <cmath>
static inline float rsqrtf(float x) { return 1.f / std::sqrt(x); }

#include "render_params.h"
#include "metric.cuh"
#include "trace.cuh"
#include "post_process.cuh"

#include <cstdint>
#include <cstddef>
#include <omp.h>

/* Same layout as BHProbe in include/bh_launch.h (not included here: the
 * reference headers define names that the library header also declares). */
struct ProbeRec
{
    int outcome, cls, steps, diskSamples;
    float escDir[3];
    float trans;
    float accum[3];
    float maxHviol;
    float hdr[3];
    float diskR, diskG, drift;
};
static_assert(sizeof(ProbeRec) == 72, "ProbeRec must match BHProbe");

static int nthr(int n) { return n > 0 ? n : omp_get_max_threads(); }

static void fill(ProbeRec& o, const TraceResult& t, float3 hdr)
{
    o.outcome = t.escaped ? 1 : 0;
    o.cls = (t.trans < 0.5f) ? 1 : (t.horizon ? 0 : 2);
    o.steps = t.steps;
    o.diskSamples = 0;
    o.escDir[0] = t.escDir.x; o.escDir[1] = t.escDir.y; o.escDir[2] = t.escDir.z;
    o.trans = t.trans;
    o.accum[0] = t.accum.x; o.accum[1] = t.accum.y; o.accum[2] = t.accum.z;
    o.maxHviol = t.maxHviol;
    o.hdr[0] = hdr.x; o.hdr[1] = hdr.y; o.hdr[2] = hdr.z;
    o.diskR = 0.f; o.diskG = 0.f; o.drift = 0.f;
}

/* renderSampleHDR's shading of a finished trace (trace.cuh:917-924). */
static float3 shadeTrace(const RenderParams& P, const TraceResult& t)
{
    float gCam = cameraEnergyFactor(P);
    float3 bg = t.horizon ? make_float3(0.f, 0.f, 0.f) : backgroundColor(t.escDir, gCam);
    float3 hdr = t.accum + bg * t.trans;
    if (!std::isfinite(hdr.x) || !std::isfinite(hdr.y) || !std::isfinite(hdr.z))
        hdr = make_float3(0.f, 0.f, 0.f);
    return hdr;
}

extern "C" {

int ref_sanitize(RenderParams* p) { return sanitizeRenderParams(*p) ? 1 : 0; }

/* out: a Q rPlus rMinus rPhoton rErgo rIsco clamped naked (BHDerived layout) */
void ref_derive(int model, float* M, float* aStar, float* q, int allowNaked, float* out)
{
    BHDerived d = bhValidateAndDerive(model, *M, *aStar, *q, allowNaked != 0);
    out[0] = d.a; out[1] = d.Q; out[2] = d.rPlus; out[3] = d.rMinus;
    out[4] = d.rPhoton; out[5] = d.rErgo; out[6] = d.rIsco;
    int* flags = reinterpret_cast<int*>(out + 7);
    flags[0] = d.clamped ? 1 : 0;
    flags[1] = d.naked ? 1 : 0;
}

/* tests/test_main.cu:71-89 (probeGridKernel) plus the HDR shading. */
void ref_probe_grid(const RenderParams* p, int nx, int ny, ProbeRec* out, int nthreads)
{
    const RenderParams P = *p;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthr(nthreads))
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
        {
            float fx = (i + 0.5f) / (float)nx;
            float fy = (j + 0.5f) / (float)ny;
            float3 dir = cameraRayDir(P, fx, fy);
            TraceResult t = traceRay(P, P.camPos, dir, true);
            fill(out[(size_t)j * nx + i], t, shadeTrace(P, t));
        }
}

/* tests/test_main.cu:91-98 (probeOneKernel), batched over directions. */
void ref_probe_dirs(const RenderParams* p, const float* dirs, int n, ProbeRec* out, int nthreads)
{
    const RenderParams P = *p;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthr(nthreads))
    for (int k = 0; k < n; ++k)
    {
        float3 dir = make_float3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]);
        TraceResult t = traceRay(P, P.camPos, dir, true);
        fill(out[k], t, shadeTrace(P, t));
    }
}

/* renderSampleHDR for a list of pixel indices of a sanitised frame, with the
 * pipeline's jitter (black_hole_kernel.cu:26-27).  Writes float4 HDR. */
void ref_render_pixels(const RenderParams* p, const int* pix, int n, float* hdr, int nthreads)
{
    RenderParams P = *p;
    sanitizeRenderParams(P);
    float2 j = subpixelJitter(P.accumMode, P.sampleIndex);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthr(nthreads))
    for (int k = 0; k < n; ++k)
    {
        int px = pix[k] % P.width, py = pix[k] / P.width;
        float3 c = renderSampleHDR(P, px, py, j.x, j.y);
        hdr[4 * k + 0] = c.x; hdr[4 * k + 1] = c.y; hdr[4 * k + 2] = c.z; hdr[4 * k + 3] = 1.f;
    }
}

/* launchRenderPipeline (black_hole_kernel.cu:108-134) with the five kernel
 * bodies (:22-103) as pixel loops. */
void ref_pipeline(uint8_t* out8, float* accumf, float* bloomAf, float* bloomBf,
                  const RenderParams* p, int nthreads)
{
    RenderParams P = *p;
    sanitizeRenderParams(P);
    uchar4* out = reinterpret_cast<uchar4*>(out8);
    float4* accum = reinterpret_cast<float4*>(accumf);
    float4* bloomA = reinterpret_cast<float4*>(bloomAf);
    float4* bloomB = reinterpret_cast<float4*>(bloomBf);
    const int bw = (P.width + 1) / 2, bh = (P.height + 1) / 2;
    const int nt = nthr(nthreads);

#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int py = 0; py < P.height; ++py)                  /* renderAccumKernel */
        for (int px = 0; px < P.width; ++px)
        {
            float2 j = subpixelJitter(P.accumMode, P.sampleIndex);
            float3 cur = renderSampleHDR(P, px, py, j.x, j.y);
            int idx = py * P.width + px;
            float4 pv = accum[idx];
            float3 prev = make_float3(pv.x, pv.y, pv.z);
            if (!std::isfinite(prev.x) || !std::isfinite(prev.y) || !std::isfinite(prev.z))
                prev = cur;
            float3 c = accumBlend(prev, cur, P.accumMode, P.sampleIndex);
            accum[idx] = make_float4(c.x, c.y, c.z, 1.f);
        }
    if (P.bloomEnabled)
    {
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                       /* bloomDownsampleKernel */
            for (int x = 0; x < bw; ++x)
            {
                int x0 = x * 2, y0 = y * 2;
                int x1 = (x0 + 1 < P.width) ? x0 + 1 : x0;
                int y1 = (y0 + 1 < P.height) ? y0 + 1 : y0;
                float4 a = accum[y0 * P.width + x0];
                float4 b = accum[y0 * P.width + x1];
                float4 c = accum[y1 * P.width + x0];
                float4 d = accum[y1 * P.width + x1];
                float3 avg = make_float3(a.x + b.x + c.x + d.x, a.y + b.y + c.y + d.y,
                                         a.z + b.z + c.z + d.z) * 0.25f;
                float3 bp = bloomBrightPass(avg * P.exposure);
                bloomA[y * bw + x] = make_float4(bp.x, bp.y, bp.z, 1.f);
            }
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                       /* bloomBlurHKernel */
            for (int x = 0; x < bw; ++x)
            {
                float3 s = make_float3(0.f, 0.f, 0.f);
                for (int k = -4; k <= 4; ++k) s += fetchHalf(bloomA, x + k, y, bw, bh) * bloomGaussW(k);
                bloomB[y * bw + x] = make_float4(s.x, s.y, s.z, 1.f);
            }
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                       /* bloomBlurVKernel */
            for (int x = 0; x < bw; ++x)
            {
                float3 s = make_float3(0.f, 0.f, 0.f);
                for (int k = -4; k <= 4; ++k) s += fetchHalf(bloomB, x, y + k, bw, bh) * bloomGaussW(k);
                bloomA[y * bw + x] = make_float4(s.x, s.y, s.z, 1.f);
            }
    }
#pragma omp parallel for num_threads(nt)
    for (int py = 0; py < P.height; ++py)                  /* compositeKernel */
        for (int px = 0; px < P.width; ++px)
        {
            float4 av = accum[py * P.width + px];
            float3 hdr = make_float3(av.x, av.y, av.z);
            float3 bloom = make_float3(0.f, 0.f, 0.f);
            if (P.bloomEnabled)
                bloom = sampleHalfBilinear(bloomA, (px + 0.5f) * 0.5f, (py + 0.5f) * 0.5f, bw, bh);
            out[py * P.width + px] = finalizePixel(hdr, bloom, P, px, py);
        }
}

/* launchRenderKernel (black_hole_kernel.cu:140-163). */
void ref_render_kernel(uint8_t* out8, const RenderParams* p, int nthreads)
{
    RenderParams P = *p;
    sanitizeRenderParams(P);
    P.bloomEnabled = 0;
    uchar4* out = reinterpret_cast<uchar4*>(out8);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthr(nthreads))
    for (int py = 0; py < P.height; ++py)
        for (int px = 0; px < P.width; ++px)
        {
            float3 hdr = renderSampleHDR(P, px, py, 0.5f, 0.5f);
            out[py * P.width + px] = finalizePixel(hdr, make_float3(0.f, 0.f, 0.f), P, px, py);
        }
}

}  // extern "C"
