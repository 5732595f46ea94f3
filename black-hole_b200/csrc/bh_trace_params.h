#pragma once
// ---------------------------------------------------------------------------
// bh_trace_params.h -- per-launch constants of the tracing kernels (host and
// device).  Built on the host from a sanitised RenderParams once per frame, so
// frame-invariant quantities (camera energy factor, capture and escape radii,
// jitter) are computed once instead of once per ray, and passed to the kernel
// as a __grid_constant__ parameter (constant-bank operands, no loads).
// ---------------------------------------------------------------------------
#include <cuda_runtime_api.h>
#include <vector_types.h>
#include <stdint.h>

enum BhOutMode
{
    BH_OUT_ACCUM = 0,   // blend the HDR sample into a float4 accumulation buffer
    BH_OUT_RGBA = 1,    // finalise straight to uchar4 (no bloom): launchRenderKernel
    BH_OUT_HDR = 2,     // write the HDR sample as float4
    BH_OUT_PROBE = 3,   // write a BHProbe record per ray
};

struct TraceParams
{
    // rays: pixels of a W x H frame in 8x4-pixel tiles, or explicit directions
    int W, H, tilesX;
    unsigned nRays;
    float jx, jy;                 // sub-pixel sample position
    const float3* dirs;           // non-null: trace these directions instead of pixels

    // camera
    float3 camPos, camFwd, camRight, camUp;
    float tanHalfFov, aspect;
    float gCam;                   // static-observer energy factor of the sky

    // metric (code units)
    int model;
    float M, a, Q;
    float rPlus, rPhoton, rCap;
    float dPhi;
    int maxSteps;

    // disk and hot spots
    int diskOn;
    float diskInner, diskOuter, diskTime, emisK, absK;
    int spotsOn;
    float spotStrength;

    // output
    int outMode;
    void* out;
    int accumMode, sampleIndex;
    float exposure;
    int swapRB;

    // work distribution
    unsigned* counter;            // ray counter, zeroed before the launch
    int refillMin;                // refill a warp when at least this many lanes are free
};
