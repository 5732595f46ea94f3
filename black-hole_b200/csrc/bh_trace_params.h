#pragma once
// ---------------------------------------------------------------------------
// bh_trace_params.h -- per-launch constants of the tracing kernels (host and
// device).  Built on the host from a sanitised RenderParams once per frame, so
// frame-invariant quantities (camera energy factor, jitter, and the whole
// static-observer tetrad at the camera) are computed once instead of once per
// ray, and passed to the kernel as a __grid_constant__ parameter.
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
    BH_OUT_ANCHOR = 4,  // pixel-list rays: write a BHAnchor record per list entry
};

// Compact record of one traced pixel of a list (BH_OUT_ANCHOR), indexed by the
// list position: the escape direction (world), outcome flags and the HDR sample.
struct BHAnchor
{
    float3 escDir;
    unsigned flags;     // BH_ANCHOR_*
    float3 hdr;
    float trans;
};
// BH_ANCHOR_INCOMPLETE: the ray spent the launch's step budget (which, for
// anchors, may be below the frame's maxSteps): its record is not the pixel's.
enum { BH_ANCHOR_ESCAPED = 1u, BH_ANCHOR_HORIZON = 2u, BH_ANCHOR_DISK = 4u, BH_ANCHOR_INCOMPLETE = 8u };

// Largest frame (pixels) or ray count of one launch: a ray's key carries its
// pixel or list position in 28 bits (16384 x 16384 pixels).
constexpr unsigned BH_MAX_RAYS = 1u << 28;

// pixel-list entry that traces nothing (pads a 32-entry group of a list)
constexpr unsigned BH_PIX_SKIP = 0xFFFFFFFFu;

// Camera-frame quantities shared by every ray of a view, in the integration
// precision T.  They are the per-ray prologue of the reference integrators
// (src/trace.cuh:213-247, 490-521, 703-739 of Sqhh99/Black-hole) with
// everything that does not depend on the ray direction hoisted out; the host
// evaluates them with the same float (or double) libm arithmetic as the
// reference, so the per-ray remainder reproduces its initial data exactly.
template <class T>
struct CamFrame
{
    // rotating family
    T r0, th0, ph0;
    T er[3], eth[3], eph[3];     // orthonormal (r, theta, phi) basis at the camera
    T gtt, gtp, gpp, A, rsq;     // metric at the camera, A = (gpp - gtp^2/gtt)^-1/2, rsq = (-gtt)^-1/2
    T sqSD, sqS;                 // sqrt(Sigma / max(Delta, 1e-6)), sqrt(Sigma)
    // spherical family
    T e1[3];                     // radial unit vector camPos / r0
    T ephS[3];                   // azimuthal unit vector of the photon-constant tetrad
    T gttS, gtpS, gppS, AS, rsqS;
    T f0, sf0, u0;               // max(f(r0), 1e-6), sqrt(f0), 1/r0
    int camAtOrigin;             // r0 < 1e-4: E = 1, Lz = 0

    // step-loop constants (the reference's expressions, evaluated once)
    T M, a, Q2, a2, a2Q2;
    T capR;                      // capture test r <= rCap * 1.002 + 1e-3
    T rFloor, rFloor105;         // max(r+, rCap), and x 1.05 (constraint monitor)
    T escR, sixM;                // 120 M, 6 M
    T k8dPhi, i22dPhi;           // 8 dPhi, 1 / (2.2 dPhi)
    T rPh15, outer13;            // 1.5 r_photon, 1.3 diskOuter
    T dPhi, hMin;                // dPhi, 0.03 dPhi (spherical step floor)
    T uHor, uEscape, invNineM;   // 1/max(rCap, 1e-6), 1/(120 M), 1/(9 M)
    T uPh;                       // 1 / max(1.5 r_photon, 3 M)
    T diskTime;
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
    const unsigned* tileOrder;    // non-null: k-th claimed tile -> tile index (trace order)
    const unsigned* pixList;      // non-null: ray k traces pixel pixList[k] (y * W + x)
    const unsigned* nRaysDev;     // non-null: the ray count is read here at kernel start
    const unsigned* outIndex;     // BH_OUT_ANCHOR, non-null: list position k writes record outIndex[k]

    CamFrame<float> cf;           // FP32 integration
    CamFrame<double> cd;          // FP64 integration
};
