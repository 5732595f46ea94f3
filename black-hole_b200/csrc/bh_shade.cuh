#pragma once
// ---------------------------------------------------------------------------
// bh_shade.cuh -- emission and sky shading of the tracer (float arithmetic).
//
// Physics follows the reference renderer (Sqhh99/Black-hole):
//   metric helpers            src/metric.cuh:145-199
//   blackbody colour          src/trace.cuh:101-120
//   star lattice + sky        src/trace.cuh:131-195
//   volumetric disk segment   src/trace.cuh:269-403
// The step order, constants, culls and early-outs are the reference's; the
// arithmetic is arranged for the GPU: cheap culls are tested before any square
// root, shading weights use MUFU intrinsics, and every hash input is computed
// with exact (uncontracted) operations so the procedural textures are the same.
// ---------------------------------------------------------------------------
#include "bh_math.cuh"
#include "bh_trace_params.h"

constexpr float kPiF = 3.14159265358979f;
constexpr float kTInner = 13500.f;           // disk temperature scale [K]
constexpr float kNtPeakInv = 1.f / 0.075f;   // 1 / peak of the Novikov-Thorne weight

// Keplerian angular velocity of a co-rotating equatorial circular orbit (0 if none).
BH_DEV float omega_circ(float r, float M, float a, float Q)
{
    float w2 = M * r - Q * Q;
    if (w2 <= 0.f) return 0.f;
    float sw = sqrt_a(w2);
    return __fdividef(sw, r * r + a * sw);
}

// g = 1 / [u^t (E - Omega Lz)] of a circular equatorial emitter, clamped to [0.04, 6].
BH_DEV float emitter_g(float r, float Om, float M, float a, float Q, float E, float Lz)
{
    float ir2 = __frcp_rn(r * r);
    float m2r = 2.f * M * r - Q * Q;
    float gtt = -(1.f - m2r * ir2);
    float gtp = -a * m2r * ir2;
    float gpp = r * r + a * a + m2r * a * a * ir2;
    float den = -(gtt + 2.f * Om * gtp + Om * Om * gpp);
    if (den < 1e-4f) return 0.f;
    float ut = rsqrt_f(den);
    float Eem = ut * (E - Om * Lz);
    if (Eem < 0.04f) Eem = 0.04f;
    return clampf(rcp_f(Eem), 0.04f, 6.f);
}

BH_DEV float thin_disk_flux(float r, float rIn)
{
    if (!(r > rIn) || rIn <= 0.f) return 0.f;
    float x = __fdividef(rIn, r);
    float nt = x * x * x * fmaxf(1.f - sqrt_a(x), 0.f);
    float dr = r - rIn * 1.15f;
    float sig = 0.20f * rIn;
    float peak = __expf(__fdividef(-0.5f * dr * dr, fmaxf(sig * sig, 1e-8f)));
    return nt * (0.50f + 1.00f * peak);
}

// Tanner-Helland blackbody fit, linearised (gamma 2.2).
BH_DEV_CALL f3 blackbody(float kelvin)
{
    float t = clampf(kelvin, 1200.f, 40000.f) * 0.01f;
    float r, g, b;
    if (t <= 66.f) { r = 255.f; g = 99.4708025861f * __logf(t) - 161.1195681661f; }
    else
    {
        r = 329.698727446f * __powf(t - 60.f, -0.1332047592f);
        g = 288.1221695283f * __powf(t - 60.f, -0.0755148492f);
    }
    if (t >= 66.f) b = 255.f;
    else if (t <= 19.f) b = 0.f;
    else b = 138.5177312231f * __logf(t - 10.f) - 305.0447927307f;
    const float k = 1.f / 255.f;
    float sr = clampf(r, 0.f, 255.f) * k, sg = clampf(g, 0.f, 255.f) * k, sb = clampf(b, 0.f, 255.f) * k;
    return v3(__powf(sr, 2.2f), __powf(sg, 2.2f), __powf(sb, 2.2f));
}

// One star population on a cubic lattice of `cell` cells per unit direction.
BH_DEV_CALL f3 star_layer(f3 d, float cell, float intensity, float sharp)
{
    f3 p = v3(mul_x(d.x, cell), mul_x(d.y, cell), mul_x(d.z, cell));
    f3 id = v3(floorf(p.x), floorf(p.y), floorf(p.z));
    f3 f = v3(sub_x(p.x, id.x), sub_x(p.y, id.y), sub_x(p.z, id.z));
    f3 h = hash33(id);
    f3 dv = v3(f.x - (0.10f + 0.80f * h.x), f.y - (0.10f + 0.80f * h.y), f.z - (0.10f + 0.80f * h.z));
    float d2 = dot3(dv, dv);
    float mag = hash12(add_x(id.x, mul_x(91.7f, id.z)), sub_x(id.y, mul_x(33.1f, id.x)));
    float cut = (mag > 0.9f) ? 60.f : 14.f;
    if (d2 * sharp > cut) return v3(0.f, 0.f, 0.f);
    float bright = 0.05f * __powf(mag, 9.f) + 9.0f * __powf(mag, 50.f);
    float core = __expf(-d2 * sharp);
    float glow = __expf(-d2 * sharp * 0.10f);
    float tsel = hash12(add_x(id.y, 7.3f), sub_x(id.z, 3.1f));
    f3 col = blackbody(2600.f + 12000.f * tsel * tsel);
    float lum = 0.2126f * col.x + 0.7152f * col.y + 0.0722f * col.z;
    float s = rcp_f(fmaxf(lum, 1e-4f)) * ((core + 0.08f * glow) * bright * intensity);
    return col * s;
}

// Deflected-direction sky: four star lattices, Milky-Way band, airglow, scaled by gCam^4.
BH_DEV f3 sky_color(f3 dir, float gCam)
{
    f3 d = normalize_x(dir);
    float Ts = clampf(gCam, 0.5f, 3.f);
    float Is = Ts * Ts * Ts * Ts;
    f3 c = star_layer(d, 80.f, 1.00f, 320.f);
    c = c + star_layer(d, 190.f, 0.55f, 520.f);
    c = c + star_layer(d, 420.f, 0.30f, 820.f);
    c = c + star_layer(d, 900.f, 0.14f, 1500.f);
    float k = __fdiv_rn(3.0f, add_x(1.35f, fabsf(d.y)));
    float qx = mul_x(d.x, k), qy = mul_x(d.z, k);
    float neb = fbm3(qx, qy);
    float dust = fbm3(add_x(mul_x(qx, 2.6f), 31.4f), sub_x(mul_x(qy, 2.6f), 17.2f));
    float band = __expf(-d.y * d.y * 16.f);
    float lanes = clampf(1.25f - 1.35f * dust, 0.f, 1.f);
    float w = neb * band * lanes;
    c = c + v3((0.020f + 0.030f * neb) * w, (0.024f + 0.022f * neb) * w, (0.038f + 0.014f * neb) * w);
    c = c + v3(0.0012f, 0.0015f, 0.0026f);
    return c * Is;
}

BH_DEV float wrap_pi(float d)
{
    d = fmodf(d + kPiF, 2.f * kPiF);
    if (d < 0.f) d += 2.f * kPiF;
    return d - kPiF;
}

// Per-ray disk bookkeeping kept only when the caller asks for ray statistics:
// contributing sub-samples, and the radius / emitter redshift of the first
// equatorial crossing inside the disk annulus (the "disk hit").
struct DiskTally
{
    int samples;
    float hitR, hitG;
};

// Volumetric thin-disk emission and absorption along the chord a -> b.
// (E, Lz) are the photon's conserved energy and angular momentum, tEmit the
// emission coordinate time (slow light).  Accumulates into accum / trans.
template <bool STATS>
BH_DEV void disk_segment(const TraceParams& P, float E, float Lz, f3 a, f3 b, float tEmit,
                         f3& accum, float& trans, DiskTally& tally)
{
    // vertical slab cull first: no square root for rays far from the plane
    const float maxH = 0.16f * P.diskOuter;
    if (a.y > maxH && b.y > maxH) return;
    if (a.y < -maxH && b.y < -maxH) return;

    f3 seg = b - a;
    float segLen = sqrt_a(dot3(seg, seg));
    if (segLen < 1e-7f) return;
    float rcA = sqrt_a(a.x * a.x + a.z * a.z);
    float rcB = sqrt_a(b.x * b.x + b.z * b.z);
    if (fminf(rcA, rcB) - segLen > P.diskOuter) return;
    if (fmaxf(rcA, rcB) + segLen < P.diskInner) return;

    int nSub = 1 + (int)(segLen * 6.5f);
    if (nSub > 12) nSub = 12;
    const float fsub = (float)nSub;
    const float invSub = rcp_f(fsub);
    const float ds = segLen * invSub;

    const float rin = fmaxf(P.diskInner, 1e-4f);
    const float invOut = __frcp_rn(fmaxf(P.diskOuter, rin));
    const float M = P.M, aS = P.a, Qc = P.Q;

    for (int j = 0; j < nSub; ++j)
    {
        float t = ((float)j + 0.5f) * invSub;
        f3 p = a + seg * t;
        float rc = sqrt_a(p.x * p.x + p.z * p.z);
        if (rc < rin || rc > P.diskOuter) continue;

        float H = (0.040f + 0.015f * (rc * invOut)) * rc;
        float dz = __fdividef(p.y, fmaxf(H, 1e-4f));
        if (fabsf(dz) > 2.6f) continue;

        float Fr = thin_disk_flux(rc, rin) * kNtPeakInv;
        bool wantSpots = P.spotsOn && P.spotStrength > 1e-4f && rc < rin * 1.60f;
        if (Fr < 1e-6f && !wantSpots) continue;

        float dens = __expf(-dz * dz);
        dens *= smoothstep_f(rin, rin * 1.10f, rc);
        dens *= 1.0f - smoothstep_f(P.diskOuter * 0.60f, P.diskOuter, rc);

        float omega = omega_circ(rc, M, aS, Qc);
        if (omega <= 0.f) continue;
        float g = emitter_g(rc, omega, M, aS, Qc, E, Lz);
        if (g <= 0.f) continue;

        float azim = atan2f(-p.z, p.x);
        float azr = azim - omega * tEmit;
        float n0 = fbm3(rc * 3.6f, azr * 2.3f + rc * 0.8f);
        float st = vnoise(rc * 21.f - azr * 1.7f, azr * 3.5f + rc * 2.2f);
        dens *= (0.20f + 1.30f * n0) * (0.40f + 1.00f * st);
        dens *= dens;
        float psi1 = azim - 0.55f * omega * tEmit - 1.6f * __logf(fmaxf(rc, 0.2f));
        dens *= (1.f + 0.38f * __cosf(psi1));

        float spotBoost = 0.f, spotHeat = 0.f;
        if (wantSpots)
        {
            const float rH0 = rin * 1.06f, rH1 = rin * 1.18f;
            float om0 = omega_circ(rH0, M, aS, Qc);
            float om1 = omega_circ(rH1, M, aS, Qc);
            if (om0 <= 0.f) om0 = omega;
            if (om1 <= 0.f) om1 = omega;
            const float iPhi = 1.f / (2.f * 0.18f * 0.18f);
            const float iR0 = __frcp_rn(2.f * (0.09f * rH0) * (0.09f * rH0));
            const float iR1 = __frcp_rn(2.f * (0.11f * rH1) * (0.11f * rH1));
            float dph0 = wrap_pi(azim - (om0 * tEmit + 0.4f));
            float dph1 = wrap_pi(azim - (om1 * tEmit + 0.4f + kPiF));
            float dr0 = rc - rH0, dr1 = rc - rH1;
            float fl0 = 0.72f + 0.28f * __sinf(1.7f * tEmit + 0.9f);
            float fl1 = 0.65f + 0.35f * __sinf(1.1f * tEmit + 2.3f);
            float g0 = __expf(-(dph0 * dph0) * iPhi - dr0 * dr0 * iR0 - dz * dz * 0.45f);
            float g1 = __expf(-(dph1 * dph1) * iPhi - dr1 * dr1 * iR1 - dz * dz * 0.45f);
            float S = P.spotStrength;
            spotBoost = S * (5.0f * fl0 * g0 + 3.2f * fl1 * g1);
            spotHeat = S * (0.70f * fl0 * g0 + 0.45f * fl1 * g1);
            dens += dens * 0.25f * (g0 + g1) * S;
        }
        if (dens < 1e-5f && spotBoost < 1e-4f) continue;

        float Temit = kTInner * sqrt_a(sqrt_a(clampf(Fr, 1e-6f, 1.f)));
        Temit = clampf(Temit * (1.f + 1.6f * spotHeat), 2000.f, 26000.f);
        f3 col = blackbody(clampf(Temit * g, 1200.f, 40000.f));
        float g3 = g * g * g;
        float w = dens * ds;
        float k = Fr * g3 * g * (1.f + spotBoost) * P.emisK * w;
        if (spotBoost > 1e-4f) k += spotBoost * g3 * P.emisK * 0.55f * ((0.12f + dens) * ds);
        accum = accum + col * (k * trans);

        trans *= __expf(-(P.absK * w * (1.f + 0.35f * dens)));
        if (STATS) tally.samples++;
        if (trans < 0.012f) return;
    }
}
