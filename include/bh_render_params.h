#pragma once
/*
 * bh_render_params.h -- the per-frame parameter block of the null-geodesic
 * tracer, byte-compatible with the reference renderer's RenderParams
 * (src/render_params.h:21-87 of Sqhh99/Black-hole).
 *
 * The layout has to be identical, not merely similar: a caller of the
 * reference launchers fills this struct and passes it by reference, so the
 * drop-in library must read the same bytes at the same offsets.  Size is
 * 160 bytes, alignment 4; every offset is pinned by the static_asserts below.
 *
 * Units: G = c = 1.  M is the mass (default 0.5, so the Schwarzschild radius
 * 2M is one code unit).  aSpin = a* M is signed (a* < 0 is retrograde),
 * Qc = q M >= 0.  rPlus / rPhoton / rErgo are derived on the host
 * (bhValidateAndDerive) and re-derived by the launchers when inconsistent.
 */
#include <vector_types.h>

#ifdef __cplusplus
#define BH_DEFAULT(...) = __VA_ARGS__
#else
#define BH_DEFAULT(...)
#endif

typedef struct RenderParams
{
    /* framebuffer */
    int      width      BH_DEFAULT(1280);
    int      height     BH_DEFAULT(720);
    int      swapRB     BH_DEFAULT(0);        /* 1: write BGRA instead of RGBA */

    /* pinhole camera, world frame, spin axis +Y */
    float3   camPos     BH_DEFAULT({0.f, 0.f, 0.f});
    float3   camForward BH_DEFAULT({0.f, 0.f, -1.f});
    float3   camRight   BH_DEFAULT({1.f, 0.f, 0.f});
    float3   camUp      BH_DEFAULT({0.f, 1.f, 0.f});
    float    tanHalfFov BH_DEFAULT(0.5773503f);
    float    aspect     BH_DEFAULT(1280.f / 720.f);

    /* metric family: 0 Schwarzschild, 1 Reissner-Nordstrom, 2 Kerr, 3 Kerr-Newman */
    int      model      BH_DEFAULT(0);
    float    M          BH_DEFAULT(0.5f);
    float    aSpin      BH_DEFAULT(0.f);
    float    Qc         BH_DEFAULT(0.f);
    float    rPlus      BH_DEFAULT(1.0f);
    float    rPhoton    BH_DEFAULT(1.5f);
    float    rErgo      BH_DEFAULT(1.0f);
    int      allowNaked BH_DEFAULT(0);

    /* integration budget (quality preset) */
    float    dPhi       BH_DEFAULT(0.012f);
    int      maxSteps   BH_DEFAULT(2000);

    /* accretion disk */
    int      diskEnabled   BH_DEFAULT(1);
    float    diskInner     BH_DEFAULT(3.0f);
    float    diskOuter     BH_DEFAULT(8.0f);
    float    diskTime      BH_DEFAULT(0.f);
    float    diskEmisScale BH_DEFAULT(1.5f);
    float    diskAbsScale  BH_DEFAULT(2.2f);

    /* orbiting hot spots */
    int      hotSpotsEnabled BH_DEFAULT(1);
    float    hotSpotStrength BH_DEFAULT(0.65f);

    /* post-processing */
    float    exposure      BH_DEFAULT(1.0f);
    int      sampleIndex   BH_DEFAULT(0);  /* samples already accumulated */
    int      accumMode     BH_DEFAULT(0);  /* 0 overwrite, 1 running mean, 2 EMA */
    int      bloomEnabled  BH_DEFAULT(1);
    float    bloomStrength BH_DEFAULT(0.35f);
} RenderParams;

#undef BH_DEFAULT

#ifdef __cplusplus
#include <cstddef>
static_assert(sizeof(RenderParams) == 160, "RenderParams must stay 160 bytes");
static_assert(alignof(RenderParams) == 4, "RenderParams must stay 4-byte aligned");
static_assert(offsetof(RenderParams, camPos) == 12, "layout");
static_assert(offsetof(RenderParams, camForward) == 24, "layout");
static_assert(offsetof(RenderParams, camRight) == 36, "layout");
static_assert(offsetof(RenderParams, camUp) == 48, "layout");
static_assert(offsetof(RenderParams, tanHalfFov) == 60, "layout");
static_assert(offsetof(RenderParams, model) == 68, "layout");
static_assert(offsetof(RenderParams, aSpin) == 76, "layout");
static_assert(offsetof(RenderParams, rPlus) == 84, "layout");
static_assert(offsetof(RenderParams, allowNaked) == 96, "layout");
static_assert(offsetof(RenderParams, dPhi) == 100, "layout");
static_assert(offsetof(RenderParams, maxSteps) == 104, "layout");
static_assert(offsetof(RenderParams, diskEnabled) == 108, "layout");
static_assert(offsetof(RenderParams, diskTime) == 120, "layout");
static_assert(offsetof(RenderParams, hotSpotsEnabled) == 132, "layout");
static_assert(offsetof(RenderParams, exposure) == 140, "layout");
static_assert(offsetof(RenderParams, accumMode) == 148, "layout");
static_assert(offsetof(RenderParams, bloomStrength) == 156, "layout");
#endif
