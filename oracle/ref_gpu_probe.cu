/*
 * ref_gpu_probe.cu -- TEST INFRASTRUCTURE ONLY.
 *
 * Probe and HDR entry points over the reference renderer's own device code
 * (src/trace.cuh of Sqhh99/Black-hole), compiled unmodified for sm_100a with
 * the reference's --use_fast_math, into oracle/_ref/libbhref_gpu.so together
 * with the unmodified src/black_hole_kernel.cu (see oracle/Makefile).  This
 * is "the reference kernel on the same box": the tests measure how far its
 * results sit from the CPU oracle, and the benchmark can time it beside the
 * new kernels.  The probe kernel restates tests/test_main.cu:71-89.
 */
#include "render_params.h"
#include "trace.cuh"
#include <cuda_runtime.h>

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

__global__ void refProbeGridKernel(ProbeRec* out, RenderParams P, int nx, int ny)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    float fx = (i + 0.5f) / (float)nx;
    float fy = (j + 0.5f) / (float)ny;
    float3 dir = cameraRayDir(P, fx, fy);
    TraceResult t = traceRay(P, P.camPos, dir, true);

    float gCam = cameraEnergyFactor(P);
    float3 bg = t.horizon ? make_float3(0.f, 0.f, 0.f) : backgroundColor(t.escDir, gCam);
    float3 hdr = t.accum + bg * t.trans;
    if (!isfinite(hdr.x) || !isfinite(hdr.y) || !isfinite(hdr.z)) hdr = make_float3(0.f, 0.f, 0.f);

    ProbeRec o;
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
    out[j * nx + i] = o;
}

/* renderSampleHDR for every pixel with a centred sample (trace.cuh:908-926). */
__global__ void refHdrKernel(float4* hdr, RenderParams P)
{
    int px = blockIdx.x * blockDim.x + threadIdx.x;
    int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= P.width || py >= P.height) return;
    float3 c = renderSampleHDR(P, px, py, 0.5f, 0.5f);
    hdr[py * P.width + px] = make_float4(c.x, c.y, c.z, 1.f);
}

extern "C" cudaError_t ref_gpu_probe_grid(ProbeRec* out, const RenderParams* p, int nx, int ny,
                                          cudaStream_t stream)
{
    dim3 block(16, 8);
    dim3 grid((nx + 15) / 16, (ny + 7) / 8);
    refProbeGridKernel<<<grid, block, 0, stream>>>(out, *p, nx, ny);
    return cudaGetLastError();
}

/* params are used as given (the caller sanitises), like the probe. */
extern "C" cudaError_t ref_gpu_render_hdr(float4* hdr, const RenderParams* p, cudaStream_t stream)
{
    dim3 block(16, 8);
    dim3 grid((p->width + 15) / 16, (p->height + 7) / 8);
    refHdrKernel<<<grid, block, 0, stream>>>(hdr, *p);
    return cudaGetLastError();
}
