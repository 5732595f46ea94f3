// ---------------------------------------------------------------------------
// bh_params.cpp -- host-side black-hole derivation and parameter sanitising.
//
// Restates the reference's host logic (Sqhh99/Black-hole src/metric.cuh):
//   bhValidateAndDerive   metric.cuh:257-329   clamp a*, q; horizons, photon
//                                              orbit, ergosphere
//   bhIscoNumeric         metric.cuh:224-248   minimum of the specific orbital
//                                              energy on a 0.001 M grid
//   sanitizeRenderParams  metric.cuh:344-419   every field forced renderable
// The clamps, limits and fall-back values must be the reference's (a caller
// that passes the same RenderParams must get the same sanitised frame), so
// the sequence of tests is kept; the arithmetic is float, like the
// reference's, and this file is compiled without FMA contraction so the
// results are bit-identical to a host build of the reference.
// ---------------------------------------------------------------------------
#include <cmath>
#include "bh_launch.h"

namespace {

constexpr float kExtremal = 0.995f;   // max a*^2 + q^2 for a regular hole
constexpr float kNakedCap = 2.25f;    // max a*^2 + q^2 when naked singularities are allowed
constexpr float kSingCut = 0.05f;     // capture radius / M without a horizon

inline bool isSpinning(int model) { return model == BH_KERR || model == BH_KERR_NEWMAN; }
inline bool isCharged(int model) { return model == BH_REISSNER_NORDSTROM || model == BH_KERR_NEWMAN; }

inline float outerHorizon(float M, float a, float Q)
{
    float d = M * M - a * a - Q * Q;
    return M + std::sqrt(d < 0.f ? 0.f : d);
}

inline float innerHorizon(float M, float a, float Q)
{
    float d = M * M - a * a - Q * Q;
    return M - std::sqrt(d < 0.f ? 0.f : d);
}

// photon sphere of the spherical metrics: (3M + sqrt(9M^2 - 8Q^2)) / 2
inline float photonSphere(float M, float Q)
{
    float d = 9.f * M * M - 8.f * Q * Q;
    return 0.5f * (3.f * M + std::sqrt(d < 0.f ? 0.f : d));
}

// Bardeen's co-rotating equatorial photon orbit 2M (1 + cos(2/3 acos(-a*)))
inline float photonOrbitKerr(float M, float aStar)
{
    float x = aStar > 1.f ? 1.f : (aStar < -1.f ? -1.f : aStar);
    return 2.f * M * (1.f + std::cos((2.f / 3.f) * std::acos(-x)));
}

// Kerr orbit blended toward the spherical one by the charge (step-control marker)
inline float photonOrbitKN(float M, float aStar, float q)
{
    float rK = photonOrbitKerr(M, aStar);
    float rS = photonSphere(M, q * M);
    if (std::fabs(aStar) < 1e-5f) return rS;
    float w = q * q;
    w = w < 0.f ? 0.f : (w > 1.f ? 1.f : w);
    return (1.f - 0.35f * w) * rK + 0.35f * w * rS;
}

inline float ergoRadius(float M, float Q)
{
    float d = M * M - Q * Q;
    return M + std::sqrt(d < 0.f ? 0.f : d);
}

inline float keplerOmega(float r, float M, float a, float Q)
{
    float w2 = M * r - Q * Q;
    if (w2 <= 0.f) return 0.f;
    float sw = std::sqrt(w2);
    return sw / (r * r + a * sw);
}

// specific energy of the circular orbit at r, or +inf when none exists
inline bool orbitEnergy(float r, float M, float a, float Q, float& E)
{
    float Om = keplerOmega(r, M, a, Q);
    if (Om <= 0.f) return false;
    float r2 = r * r;
    float m2r = 2.f * M * r - Q * Q;
    float gtt = -(1.f - m2r / r2);
    float gtp = -a * m2r / r2;
    float gpp = r2 + a * a + m2r * a * a / r2;
    float den = -(gtt + 2.f * Om * gtp + Om * Om * gpp);
    if (den <= 1e-6f) return false;
    E = -(gtt + Om * gtp) / std::sqrt(den);
    return true;
}

float iscoRadius(float M, float a, float Q)
{
    const bool horizon = (M * M - a * a - Q * Q) >= 0.f;
    const float rp = horizon ? outerHorizon(M, a, Q) : kSingCut * M;
    const float rStart = rp > 1e-6f ? rp * 1.02f : 0.5f * M;
    const float rEnd = 12.f * M, dr = 0.001f * M;
    float best = 6.f * M, bestE = 1e30f;
    bool found = false;
    for (float r = rStart; r <= rEnd; r += dr)
    {
        float E;
        if (orbitEnergy(r, M, a, Q, E) && E < bestE) { bestE = E; best = r; found = true; }
    }
    if (!found) best = (6.f * M > rp * 1.5f) ? 6.f * M : rp * 1.5f;
    const float floorR = rp > 1e-6f ? rp * 1.15f : 0.5f * M;
    return best > floorR ? best : floorR;
}

BHDerived deriveHole(int model, float& M, float& aStar, float& q, bool allowNaked)
{
    BHDerived d{0.f, 0.f, 1.f, 0.f, 1.5f, 1.f, 3.f, 0, 0};
    if (!(M > 0.f) || !std::isfinite(M)) { M = 0.5f; d.clamped = 1; }
    if (!std::isfinite(aStar)) { aStar = 0.f; d.clamped = 1; }
    if (!std::isfinite(q)) { q = 0.f; d.clamped = 1; }

    const float knob = allowNaked ? std::sqrt(kNakedCap) : kExtremal;
    if (aStar < -knob) { aStar = -knob; d.clamped = 1; }
    if (aStar > knob) { aStar = knob; d.clamped = 1; }
    if (q < 0.f) { q = 0.f; d.clamped = 1; }
    if (q > knob) { q = knob; d.clamped = 1; }

    float aEff = isSpinning(model) ? aStar : 0.f;
    float qEff = isCharged(model) ? q : 0.f;
    const float bound = allowNaked ? kNakedCap : kExtremal;
    const float s2 = aEff * aEff + qEff * qEff;
    if (s2 > bound)
    {   // scale (a*, q) back onto the bound, keeping their ratio
        const float k = std::sqrt(bound / s2);
        aEff *= k;
        qEff *= k;
        if (isSpinning(model)) aStar = aEff;
        if (isCharged(model)) q = qEff;
        d.clamped = 1;
    }
    d.a = aEff * M;
    d.Q = qEff * M;

    if (M * M - d.a * d.a - d.Q * d.Q < 0.f) { d.naked = 1; d.rPlus = 0.f; d.rMinus = 0.f; }
    else { d.rPlus = outerHorizon(M, d.a, d.Q); d.rMinus = innerHorizon(M, d.a, d.Q); }
    d.rErgo = d.naked ? 0.f : ergoRadius(M, d.Q);

    if (isSpinning(model))
    {
        d.rPhoton = (model == BH_KERR_NEWMAN) ? photonOrbitKN(M, aEff, qEff) : photonOrbitKerr(M, aEff);
        if (d.rPlus > 0.f) { if (d.rPhoton < d.rPlus * 1.02f) d.rPhoton = d.rPlus * 1.02f; }
        else if (d.rPhoton < kSingCut * M * 2.f) d.rPhoton = 3.f * M;
    }
    else
    {
        d.rPhoton = photonSphere(M, d.Q);
        if (d.naked && !(d.rPhoton > 0.f)) d.rPhoton = 3.f * M;
    }
    d.rIsco = iscoRadius(M, d.a, d.Q);
    return d;
}

inline bool finiteVec(const float3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

// v := def if not finite, then clamp to [lo, hi]; records whether it changed
inline void fixRange(float& v, float lo, float hi, float def, bool& fixed)
{
    if (!std::isfinite(v)) { v = def; fixed = true; }
    if (v < lo) { v = lo; fixed = true; }
    if (v > hi) { v = hi; fixed = true; }
}

inline void fixInt(int& v, int lo, int hi, int def, bool& fixed)
{
    if (v < lo || v > hi) { v = def; fixed = true; }
}

}  // namespace

extern "C" void bhValidateAndDerive(int model, float* M, float* aStar, float* q, int allowNaked,
                                    BHDerived* out)
{
    *out = deriveHole(model, *M, *aStar, *q, allowNaked != 0);
}

extern "C" int bhSanitizeRenderParams(RenderParams* p)
{
    RenderParams& P = *p;
    bool fixed = false;
    if (P.width < 1) { P.width = 1; fixed = true; }
    if (P.height < 1) { P.height = 1; fixed = true; }
    fixRange(P.dPhi, 1e-4f, 0.1f, 0.012f, fixed);
    if (P.maxSteps < 16) { P.maxSteps = 16; fixed = true; }
    if (P.maxSteps > 200000) { P.maxSteps = 200000; fixed = true; }
    fixRange(P.exposure, 0.01f, 100.f, 1.f, fixed);
    fixRange(P.M, 1e-3f, 100.f, 0.5f, fixed);
    fixRange(P.tanHalfFov, 0.05f, 5.f, 0.5773503f, fixed);
    fixRange(P.aspect, 0.05f, 20.f, 16.f / 9.f, fixed);
    fixInt(P.model, 0, 3, 0, fixed);

    // spin / charge must be consistent with the stored horizon
    float M = P.M, aStar = P.aSpin / P.M, q = P.Qc / P.M;
    const bool naked = P.allowNaked != 0;
    const float bound = naked ? kNakedCap : kExtremal;
    if (!std::isfinite(aStar) || !std::isfinite(q) || aStar * aStar + q * q > bound + 1e-4f || q < 0.f ||
        !std::isfinite(P.rPlus) || (!naked && P.rPlus <= 0.f) || (naked && P.rPlus < 0.f))
    {
        BHDerived d = deriveHole(P.model, M, aStar, q, naked);
        P.M = M; P.aSpin = d.a; P.Qc = d.Q;
        P.rPlus = d.rPlus; P.rPhoton = d.rPhoton; P.rErgo = d.rErgo;
        fixed = true;
    }
    if (!finiteVec(P.camPos) || !finiteVec(P.camForward) || !finiteVec(P.camRight) || !finiteVec(P.camUp))
    {   // the reference's default view
        P.camPos = {13.f, 3.2f, 8.f};
        P.camForward = {-0.81f, -0.20f, -0.55f};
        P.camRight = {0.56f, 0.f, -0.83f};
        P.camUp = {-0.17f, 0.98f, -0.11f};
        fixed = true;
    }
    // keep the camera outside twice the capture radius
    const float r0 = std::sqrt(P.camPos.x * P.camPos.x + P.camPos.y * P.camPos.y + P.camPos.z * P.camPos.z);
    const float rMin = (P.rPlus > 1e-6f) ? P.rPlus * 2.0f : (kSingCut * P.M * 8.f);
    if (r0 < rMin)
    {
        const float k = rMin / (r0 > 1e-6f ? r0 : 1e-6f);
        P.camPos.x *= k; P.camPos.y *= k; P.camPos.z *= k;
        fixed = true;
    }
    const float diskLo = (P.rPlus > 1e-6f) ? P.rPlus * 1.05f : (kSingCut * P.M * 2.f);
    fixRange(P.diskInner, diskLo, 1000.f, diskLo * 3.f, fixed);
    fixRange(P.diskOuter, P.diskInner * 1.2f, 2000.f, P.diskInner * 4.f, fixed);
    if (P.sampleIndex < 0) { P.sampleIndex = 0; fixed = true; }
    if (P.sampleIndex > 65536) { P.sampleIndex = 65536; fixed = true; }
    fixInt(P.accumMode, 0, 2, 0, fixed);
    fixRange(P.bloomStrength, 0.f, 4.f, 0.35f, fixed);
    fixRange(P.diskEmisScale, 0.f, 50.f, 1.5f, fixed);
    fixRange(P.diskAbsScale, 0.f, 20.f, 2.2f, fixed);
    fixRange(P.hotSpotStrength, 0.f, 8.f, 0.65f, fixed);
    if (P.hotSpotsEnabled != 0 && P.hotSpotsEnabled != 1) { P.hotSpotsEnabled = 1; fixed = true; }
    return fixed ? 1 : 0;
}
