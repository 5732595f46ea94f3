/*
 * bh_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference tracer of Sqhh99/Black-hole, used by the
 * tests and by the CPU-baseline leg of the benchmark as the checker.  The
 * product (libbh.so) never links, loads or calls this file.
 *
 * The FP32 instantiation restates the reference arithmetic operation by
 * operation (same association, same libm calls, no FMA contraction: build
 * with -ffp-contract=off) so that it reproduces the reference compiled as
 * host code bit for bit; that claim is pinned by tests/golden (fixtures made
 * from the reference's own sources, see oracle/Makefile and
 * tests/golden/make_golden.py).  The FP64 instantiation runs the same
 * integrators in double precision and is the small-step accuracy oracle
 * (dPhi/16, 16x the step budget).  Shading (disk emissivity, starfield,
 * post-processing) is float in both, as in the reference.
 *
 * Additions that do not alter the reference logic: the count of contributing
 * disk sub-samples, the radius / redshift where transmittance first falls
 * below one half, and the drift of the conserved quantity (Carter constant
 * for Kerr-Newman, Binet first integral for the spherical metrics).
 *
 * Citations are path:line in the reference repository.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>
#include <omp.h>
#include "bh_render_params.h"
#include "bh_launch.h"

namespace {

/* ------------------------------------------------------------------------ */
/* Scalar math: one overload per precision so the FP32 path calls exactly the
 * float libm entry points the reference calls.                              */
/* ------------------------------------------------------------------------ */
inline float  Sqrt(float x)  { return sqrtf(x); }
inline double Sqrt(double x) { return sqrt(x); }
inline float  Sin(float x)   { return sinf(x); }
inline double Sin(double x)  { return sin(x); }
inline float  Cos(float x)   { return cosf(x); }
inline double Cos(double x)  { return cos(x); }
inline float  Acos(float x)  { return acosf(x); }
inline double Acos(double x) { return acos(x); }
inline float  Atan2(float y, float x)   { return atan2f(y, x); }
inline double Atan2(double y, double x) { return atan2(y, x); }
inline float  Fabs(float x)  { return fabsf(x); }
inline double Fabs(double x) { return fabs(x); }
inline float  Fmin(float a, float b)   { return fminf(a, b); }
inline double Fmin(double a, double b) { return fmin(a, b); }
inline float  Fmax(float a, float b)   { return fmaxf(a, b); }
inline double Fmax(double a, double b) { return fmax(a, b); }
/* the reference's host shim: rsqrtf(x) = 1/sqrt(x) */
inline float  Rsqrt(float x)  { return 1.f / sqrtf(x); }
inline double Rsqrt(double x) { return 1.0 / sqrt(x); }
template <class T> inline T Clamp(T x, T lo, T hi) { return Fmin(Fmax(x, lo), hi); }
template <class T> inline bool Finite(T x) { return std::isfinite(x); }

/* reference constants: trace.cuh:66-70, metric.cuh:53-58 */
constexpr float kPi        = 3.14159265358979f;
constexpr float kTInner    = 13500.f;
constexpr float kNtPeakInv = 1.f / 0.075f;
constexpr float kExtremal  = 0.995f;
constexpr float kNakedCap  = 2.25f;
constexpr float kSingCut   = 0.05f;

/* ------------------------------------------------------------------------ */
/* 3-vectors (reference vec_math.cuh:8-24 semantics)                         */
/* ------------------------------------------------------------------------ */
template <class T> struct V3 { T x, y, z; };
template <class T> inline V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T len(V3<T> a) { return Sqrt(dot(a, a)); }
template <class T> inline V3<T> unit(V3<T> a) { return a * Rsqrt(Fmax(dot(a, a), T(1e-20f))); }
template <class T> inline V3<T> divs(V3<T> a, T s) { return a * (T(1) / s); }
typedef V3<float> F3;
inline F3 fromF3(const float3& v) { return mk(v.x, v.y, v.z); }
template <class T> inline V3<T> cvt(F3 v) { return mk((T)v.x, (T)v.y, (T)v.z); }
template <class T> inline F3 tof(V3<T> v) { return mk((float)v.x, (float)v.y, (float)v.z); }

inline float fract(float x) { return x - floorf(x); }
inline float lerpf(float a, float b, float t) { return a + (b - a) * t; }
inline float smooth(float e0, float e1, float x)  /* vec_math.cuh:31-35 */
{
    float t = Clamp((x - e0) / (e1 - e0), 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}

/* ------------------------------------------------------------------------ */
/* Hashes and value noise: vec_math.cuh:46-98                                */
/* ------------------------------------------------------------------------ */
inline float hash12(float px, float py)
{
    float ax = fract(px * 0.1031f), ay = fract(py * 0.1031f), az = fract(px * 0.1031f);
    float d = ax * (ay + 33.33f) + ay * (az + 33.33f) + az * (ax + 33.33f);
    ax += d; ay += d; az += d;
    return fract((ax + ay) * az);
}

inline F3 hash33(F3 p)
{
    float x = fract(p.x * 0.1031f), y = fract(p.y * 0.1030f), z = fract(p.z * 0.0973f);
    float d = x * (y + 33.33f) + y * (x + 33.33f) + z * (z + 33.33f);
    x += d; y += d; z += d;
    return mk(fract((x + y) * z), fract((x + z) * y), fract((y + z) * x));
}

inline float vnoise(float px, float py)
{
    float ix = floorf(px), iy = floorf(py);
    float fx = px - ix, fy = py - iy;
    float ux = fx * fx * (3.f - 2.f * fx);
    float uy = fy * fy * (3.f - 2.f * fy);
    float c00 = hash12(ix, iy);
    float c10 = hash12(ix + 1.f, iy + 0.f);
    float c01 = hash12(ix + 0.f, iy + 1.f);
    float c11 = hash12(ix + 1.f, iy + 1.f);
    return lerpf(lerpf(c00, c10, ux), lerpf(c01, c11, ux), uy);
}

inline float fbm3(float px, float py)
{
    float v = 0.f, amp = 0.5f;
    for (int o = 0; o < 3; ++o)
    {
        v += amp * vnoise(px, py);
        float nx = px * 2.03f + 11.7f, ny = py * 2.01f - 5.2f;
        px = nx; py = ny;
        amp *= 0.5f;
    }
    return v;
}

/* ------------------------------------------------------------------------ */
/* Metric quantities: metric.cuh:63-199 (templated on the precision)         */
/* ------------------------------------------------------------------------ */
template <class T> inline T sigmaBL(T r, T cth, T a) { return r * r + a * a * cth * cth; }
template <class T> inline T deltaBL(T r, T M, T a, T Q) { return r * r - T(2) * M * r + a * a + Q * Q; }
template <class T> inline T sphF(T r, T M, T Q) { return T(1) - T(2) * M / r + Q * Q / (r * r); }

inline float horizonOuter(float M, float a, float Q)
{
    float d = M * M - a * a - Q * Q;
    if (d < 0.f) d = 0.f;
    return M + sqrtf(d);
}
inline float horizonInner(float M, float a, float Q)
{
    float d = M * M - a * a - Q * Q;
    if (d < 0.f) d = 0.f;
    return M - sqrtf(d);
}
inline float photonSphere(float M, float Q)            /* metric.cuh:96-101 */
{
    float d = 9.f * M * M - 8.f * Q * Q;
    if (d < 0.f) d = 0.f;
    return 0.5f * (3.f * M + sqrtf(d));
}
inline float photonOrbitKerr(float M, float aStar)     /* metric.cuh:109-115 */
{
    float x = aStar;
    if (x > 1.f) x = 1.f;
    if (x < -1.f) x = -1.f;
    return 2.f * M * (1.f + cosf((2.f / 3.f) * acosf(-x)));
}
inline float photonOrbitKN(float M, float aStar, float q)  /* metric.cuh:120-129 */
{
    float rK = photonOrbitKerr(M, aStar);
    float rS = photonSphere(M, q * M);
    if (fabsf(aStar) < 1e-5f) return rS;
    float w = q * q;
    if (w < 0.f) w = 0.f;
    if (w > 1.f) w = 1.f;
    return (1.f - 0.35f * w) * rK + 0.35f * w * rS;
}
inline float ergoEquatorial(float M, float Q)          /* metric.cuh:132-137 */
{
    float d = M * M - Q * Q;
    if (d < 0.f) d = 0.f;
    return M + sqrtf(d);
}
inline float omegaCirc(float r, float M, float a, float Q)   /* metric.cuh:145-151 */
{
    float w2 = M * r - Q * Q;
    if (w2 <= 0.f) return 0.f;
    float sw = sqrtf(w2);
    return sw / (r * r + a * sw);
}
inline void eqMetric(float r, float M, float a, float Q, float& gtt, float& gtp, float& gpp)
{                                                       /* metric.cuh:154-162 */
    float r2 = r * r;
    float m2r = 2.f * M * r - Q * Q;
    gtt = -(1.f - m2r / r2);
    gtp = -a * m2r / r2;
    gpp = r2 + a * a + m2r * a * a / r2;
}
inline float emitterG(float r, float M, float a, float Q, float E, float Lz)
{                                                       /* metric.cuh:169-185 */
    float Om = omegaCirc(r, M, a, Q);
    if (Om <= 0.f) return 0.f;
    float gtt, gtp, gpp;
    eqMetric(r, M, a, Q, gtt, gtp, gpp);
    float den = -(gtt + 2.f * Om * gtp + Om * Om * gpp);
    if (den < 1e-4f) return 0.f;
    float ut = 1.f / sqrtf(den);
    float Eem = ut * (E - Om * Lz);
    if (Eem < 0.04f) Eem = 0.04f;
    float g = 1.f / Eem;
    if (g < 0.04f) g = 0.04f;
    if (g > 6.f) g = 6.f;
    return g;
}
inline float thinDiskFlux(float r, float rIn)           /* metric.cuh:190-199 */
{
    if (!(r > rIn) || rIn <= 0.f) return 0.f;
    float x = rIn / r;
    float nt = x * x * x * fmaxf(1.f - sqrtf(x), 0.f);
    float dr = r - rIn * 1.15f;
    float sig = 0.20f * rIn;
    float peak = expf(-0.5f * dr * dr / fmaxf(sig * sig, 1e-8f));
    return nt * (0.50f + 1.00f * peak);
}

/* ------------------------------------------------------------------------ */
/* Host derivation and sanitising: metric.cuh:224-419                        */
/* ------------------------------------------------------------------------ */
float iscoNumeric(float M, float a, float Q)            /* metric.cuh:224-248 */
{
    float disc = M * M - a * a - Q * Q;
    float rp = (disc >= 0.f) ? horizonOuter(M, a, Q) : (kSingCut * M);
    float best = 6.f * M, bestE = 1e30f;
    bool found = false;
    const float r0 = (rp > 1e-6f ? rp * 1.02f : 0.5f * M);
    const float r1 = 12.f * M;
    const float step = 0.001f * M;
    for (float r = r0; r <= r1; r += step)
    {
        float Om = omegaCirc(r, M, a, Q);
        if (Om <= 0.f) continue;
        float gtt, gtp, gpp;
        eqMetric(r, M, a, Q, gtt, gtp, gpp);
        float den = -(gtt + 2.f * Om * gtp + Om * Om * gpp);
        if (den <= 1e-6f) continue;
        float E = -(gtt + Om * gtp) / std::sqrt(den);
        if (E < bestE) { bestE = E; best = r; found = true; }
    }
    if (!found) best = (6.f * M > rp * 1.5f) ? 6.f * M : rp * 1.5f;
    float lo = (rp > 1e-6f) ? rp * 1.15f : 0.5f * M;
    return best > lo ? best : lo;
}

BHDerived derive(int model, float& M, float& aStar, float& q, bool allowNaked)
{                                                       /* metric.cuh:257-329 */
    BHDerived d;
    d.a = 0.f; d.Q = 0.f; d.rPlus = 1.f; d.rMinus = 0.f; d.rPhoton = 1.5f;
    d.rErgo = 1.f; d.rIsco = 3.f; d.clamped = 0; d.naked = 0;

    if (!(M > 0.f) || !std::isfinite(M)) { M = 0.5f; d.clamped = 1; }
    if (!std::isfinite(aStar)) { aStar = 0.f; d.clamped = 1; }
    if (!std::isfinite(q)) { q = 0.f; d.clamped = 1; }

    const float knobMax = allowNaked ? std::sqrt(kNakedCap) : kExtremal;
    if (aStar < -knobMax) { aStar = -knobMax; d.clamped = 1; }
    if (aStar > knobMax) { aStar = knobMax; d.clamped = 1; }
    if (q < 0.f) { q = 0.f; d.clamped = 1; }
    if (q > knobMax) { q = knobMax; d.clamped = 1; }

    const bool spin = (model == BH_KERR || model == BH_KERR_NEWMAN);
    const bool chrg = (model == BH_REISSNER_NORDSTROM || model == BH_KERR_NEWMAN);
    float aEff = spin ? aStar : 0.f;
    float qEff = chrg ? q : 0.f;

    const float bound = allowNaked ? kNakedCap : kExtremal;
    float s2 = aEff * aEff + qEff * qEff;
    if (s2 > bound)
    {
        float scale = std::sqrt(bound / s2);
        aEff *= scale;
        qEff *= scale;
        if (spin) aStar = aEff;
        if (chrg) q = qEff;
        d.clamped = 1;
    }
    d.a = aEff * M;
    d.Q = qEff * M;

    float disc = M * M - d.a * d.a - d.Q * d.Q;
    if (disc < 0.f) { d.naked = 1; d.rPlus = 0.f; d.rMinus = 0.f; }
    else { d.rPlus = horizonOuter(M, d.a, d.Q); d.rMinus = horizonInner(M, d.a, d.Q); }
    d.rErgo = ergoEquatorial(M, d.Q);
    if (d.naked) d.rErgo = 0.f;

    if (spin)
    {
        d.rPhoton = (model == BH_KERR_NEWMAN) ? photonOrbitKN(M, aEff, qEff)
                                              : photonOrbitKerr(M, aEff);
        if (d.rPlus > 0.f)
        {
            float lo = d.rPlus * 1.02f;
            if (d.rPhoton < lo) d.rPhoton = lo;
        }
        else if (d.rPhoton < kSingCut * M * 2.f)
            d.rPhoton = 3.f * M;
    }
    else
    {
        d.rPhoton = photonSphere(M, d.Q);
        if (d.naked && !(d.rPhoton > 0.f)) d.rPhoton = 3.f * M;
    }
    d.rIsco = iscoNumeric(M, d.a, d.Q);
    return d;
}

inline bool finite3(const float3& v)
{
    return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z);
}

bool sanitize(RenderParams& P)                          /* metric.cuh:344-419 */
{
    bool fixed = false;
    auto fixf = [&](float& v, float lo, float hi, float def) {
        if (!std::isfinite(v)) { v = def; fixed = true; }
        if (v < lo) { v = lo; fixed = true; }
        if (v > hi) { v = hi; fixed = true; }
    };
    if (P.width < 1) { P.width = 1; fixed = true; }
    if (P.height < 1) { P.height = 1; fixed = true; }
    fixf(P.dPhi, 1e-4f, 0.1f, 0.012f);
    if (P.maxSteps < 16) { P.maxSteps = 16; fixed = true; }
    if (P.maxSteps > 200000) { P.maxSteps = 200000; fixed = true; }
    fixf(P.exposure, 0.01f, 100.f, 1.f);
    fixf(P.M, 1e-3f, 100.f, 0.5f);
    fixf(P.tanHalfFov, 0.05f, 5.f, 0.5773503f);
    fixf(P.aspect, 0.05f, 20.f, 16.f / 9.f);
    if (P.model < 0 || P.model > 3) { P.model = 0; fixed = true; }

    float aStar = P.aSpin / P.M, q = P.Qc / P.M, M = P.M;
    bool allowNaked = (P.allowNaked != 0);
    float bound = allowNaked ? kNakedCap : kExtremal;
    bool needFix = !std::isfinite(aStar) || !std::isfinite(q) ||
                   aStar * aStar + q * q > bound + 1e-4f || q < 0.f ||
                   !std::isfinite(P.rPlus) || (!allowNaked && P.rPlus <= 0.f) ||
                   (allowNaked && P.rPlus < 0.f);
    if (needFix)
    {
        BHDerived d = derive(P.model, M, aStar, q, allowNaked);
        P.M = M; P.aSpin = d.a; P.Qc = d.Q;
        P.rPlus = d.rPlus; P.rPhoton = d.rPhoton; P.rErgo = d.rErgo;
        fixed = true;
    }
    if (!finite3(P.camPos) || !finite3(P.camForward) || !finite3(P.camRight) || !finite3(P.camUp))
    {
        P.camPos = {13.f, 3.2f, 8.f};
        P.camForward = {-0.81f, -0.20f, -0.55f};
        P.camRight = {0.56f, 0.f, -0.83f};
        P.camUp = {-0.17f, 0.98f, -0.11f};
        fixed = true;
    }
    float r0 = std::sqrt(P.camPos.x * P.camPos.x + P.camPos.y * P.camPos.y + P.camPos.z * P.camPos.z);
    float rMin = (P.rPlus > 1e-6f) ? P.rPlus * 2.0f : (kSingCut * P.M * 8.f);
    if (r0 < rMin)
    {
        float s = rMin / (r0 > 1e-6f ? r0 : 1e-6f);
        P.camPos.x *= s; P.camPos.y *= s; P.camPos.z *= s;
        fixed = true;
    }
    float diskLo = (P.rPlus > 1e-6f) ? P.rPlus * 1.05f : (kSingCut * P.M * 2.f);
    fixf(P.diskInner, diskLo, 1000.f, diskLo * 3.f);
    fixf(P.diskOuter, P.diskInner * 1.2f, 2000.f, P.diskInner * 4.f);
    if (P.sampleIndex < 0) { P.sampleIndex = 0; fixed = true; }
    if (P.sampleIndex > 65536) { P.sampleIndex = 65536; fixed = true; }
    if (P.accumMode < 0 || P.accumMode > 2) { P.accumMode = 0; fixed = true; }
    fixf(P.bloomStrength, 0.f, 4.f, 0.35f);
    fixf(P.diskEmisScale, 0.f, 50.f, 1.5f);
    fixf(P.diskAbsScale, 0.f, 20.f, 2.2f);
    fixf(P.hotSpotStrength, 0.f, 8.f, 0.65f);
    if (P.hotSpotsEnabled != 0 && P.hotSpotsEnabled != 1) { P.hotSpotsEnabled = 1; fixed = true; }
    return fixed;
}

/* ------------------------------------------------------------------------ */
/* Camera and sky: trace.cuh:73-195, 431-438                                 */
/* ------------------------------------------------------------------------ */
inline float captureRadius(const RenderParams& P)   /* trace.cuh:73-77 */
{
    if (P.rPlus > 1e-6f) return P.rPlus;
    return kSingCut * P.M;
}

float cameraEnergy(const RenderParams& P)           /* trace.cuh:81-96 */
{
    F3 c = fromF3(P.camPos);
    float r = len(c);
    if (r < 1e-4f) return 1.f;
    if (P.model == BH_KERR || P.model == BH_KERR_NEWMAN)
    {
        float cth = Clamp(P.camPos.y / r, -1.f, 1.f);
        float Sig = sigmaBL(r, cth, P.aSpin);
        float m2r = 2.f * P.M * r - P.Qc * P.Qc;
        float gtt = -(1.f - m2r / fmaxf(Sig, 1e-8f));
        float alpha = sqrtf(fmaxf(-gtt, 1e-6f));
        return Clamp(1.f / alpha, 0.5f, 4.f);
    }
    float f = sphF(r, P.M, P.Qc);
    return Clamp(1.f / sqrtf(fmaxf(f, 1e-6f)), 0.5f, 4.f);
}

F3 blackbody(float kelvin)                          /* trace.cuh:101-120 */
{
    float t = Clamp(kelvin, 1200.f, 40000.f) / 100.f;
    float r, g, b;
    if (t <= 66.f) r = 255.f;
    else r = 329.698727446f * powf(t - 60.f, -0.1332047592f);
    if (t <= 66.f) g = 99.4708025861f * logf(t) - 161.1195681661f;
    else g = 288.1221695283f * powf(t - 60.f, -0.0755148492f);
    if (t >= 66.f) b = 255.f;
    else if (t <= 19.f) b = 0.f;
    else b = 138.5177312231f * logf(t - 10.f) - 305.0447927307f;
    float sr = Clamp(r, 0.f, 255.f) / 255.f;
    float sg = Clamp(g, 0.f, 255.f) / 255.f;
    float sb = Clamp(b, 0.f, 255.f) / 255.f;
    return mk(powf(sr, 2.2f), powf(sg, 2.2f), powf(sb, 2.2f));
}

F3 starLayer(F3 d, float cell, float intensity, float sharp)   /* trace.cuh:131-162 */
{
    F3 p = d * cell;
    F3 id = mk(floorf(p.x), floorf(p.y), floorf(p.z));
    F3 f = p - id;
    F3 h = hash33(id);
    F3 sp = mk(0.10f + 0.80f * h.x, 0.10f + 0.80f * h.y, 0.10f + 0.80f * h.z);
    F3 dv = f - sp;
    float d2 = dot(dv, dv);
    float mag = hash12(id.x + 91.7f * id.z, id.y - 33.1f * id.x);
    float cut = (mag > 0.9f) ? 60.f : 14.f;
    if (d2 * sharp > cut) return mk(0.f, 0.f, 0.f);
    float bright = 0.05f * powf(mag, 9.f) + 9.0f * powf(mag, 50.f);
    float core = expf(-d2 * sharp);
    float glow = expf(-d2 * sharp * 0.10f);
    float tsel = hash12(id.y + 7.3f, id.z - 3.1f);
    float kelvin = 2600.f + 12000.f * tsel * tsel;
    F3 col = blackbody(kelvin);
    float lum = 0.2126f * col.x + 0.7152f * col.y + 0.0722f * col.z;
    col = col * (1.f / fmaxf(lum, 1e-4f));
    return col * ((core + 0.08f * glow) * bright * intensity);
}

F3 skyColor(F3 dir, float gCam)                     /* trace.cuh:166-195 */
{
    F3 d = unit(dir);
    float Ts = Clamp(gCam, 0.5f, 3.f);
    float Is = Ts * Ts * Ts * Ts;
    F3 c = mk(0.f, 0.f, 0.f);
    c = c + starLayer(d, 80.f, 1.00f, 320.f);
    c = c + starLayer(d, 190.f, 0.55f, 520.f);
    c = c + starLayer(d, 420.f, 0.30f, 820.f);
    c = c + starLayer(d, 900.f, 0.14f, 1500.f);
    float k = 3.0f / (1.35f + fabsf(d.y));
    float qx = d.x * k, qy = d.z * k;
    float neb = fbm3(qx, qy);
    float dust = fbm3(qx * 2.6f + 31.4f, qy * 2.6f - 17.2f);
    float band = expf(-d.y * d.y * 16.f);
    float lanes = Clamp(1.25f - 1.35f * dust, 0.f, 1.f);
    c = c + (mk(0.020f, 0.024f, 0.038f) + mk(0.030f, 0.022f, 0.014f) * neb) * (neb * band * lanes);
    c = c + mk(0.0012f, 0.0015f, 0.0026f);
    return c * Is;
}

inline F3 cameraRay(const RenderParams& P, float fx, float fy)   /* trace.cuh:431-438 */
{
    float nx = fx * 2.f - 1.f;
    float ny = 1.f - fy * 2.f;
    return unit(fromF3(P.camForward) + fromF3(P.camRight) * (nx * P.tanHalfFov * P.aspect)
                + fromF3(P.camUp) * (ny * P.tanHalfFov));
}

/* ------------------------------------------------------------------------ */
/* Volumetric disk: trace.cuh:203-403                                        */
/* ------------------------------------------------------------------------ */
struct DiskPhoton { float E, Lz, a, Q; };            /* trace.cuh:203-209 */

struct DiskTally                                     /* additions: not in the reference */
{
    int samples = 0;             /* contributing disk sub-samples */
    float hitR = 0.f, hitG = 0.f; /* first equatorial crossing inside the disk annulus, g there */
};

/* Cubic Hermite interpolant over a step of length h at fraction t. */
inline double hermite(double y0, double y1, double d0, double d1, double h, double t)
{
    double t2 = t * t, t3 = t2 * t;
    return (2 * t3 - 3 * t2 + 1) * y0 + (t3 - 2 * t2 + t) * h * d0 + (3 * t2 - 2 * t3) * y1 + (t3 - t2) * h * d1;
}

/* Disk hit (addition): record the first equatorial crossing whose radius lies
 * in [diskInner, diskOuter], with the emitter redshift of the ray there. */
inline void recordHit(const RenderParams& P, DiskTally& t, double r, float E, float Lz)
{
    if (t.hitR > 0.f || !(r >= P.diskInner && r <= P.diskOuter)) return;
    float rf = (float)r;
    t.hitR = rf;
    t.hitG = emitterG(rf, P.M, P.aSpin, P.Qc, E, Lz);
}

/* Kerr-Newman: theta crosses pi/2 within the step -> bisection of the Hermite
 * interpolant of theta, r there (FP64). */
inline void kerrCrossing(const RenderParams& P, DiskTally& t, double r0, double th0, double dr0, double dth0,
                         double r1, double th1, double dr1, double dth1, double h, float E, float Lz)
{
    const double half = 1.57079632679489661923;
    const double f0 = th0 - half, f1 = th1 - half;
    if (!((f0 < 0.0) != (f1 < 0.0))) return;
    double lo = 0.0, hi = 1.0;
    for (int i = 0; i < 52; ++i)
    {
        double mid = 0.5 * (lo + hi);
        double fm = hermite(f0, f1, dth0, dth1, h, mid);
        if ((fm < 0.0) == (f0 < 0.0)) lo = mid; else hi = mid;
    }
    recordHit(P, t, hermite(r0, r1, dr0, dr1, h, 0.5 * (lo + hi)), E, Lz);
}

inline float wrapPi(float d)                         /* trace.cuh:250-255 */
{
    d = fmodf(d + kPi, 2.f * kPi);
    if (d < 0.f) d += 2.f * kPi;
    return d - kPi;
}

void diskSegment(const RenderParams& P, const DiskPhoton& ph, F3 a, F3 b, float tEmit,
                 F3& accum, float& trans, DiskTally& tally)   /* trace.cuh:269-403 */
{
    F3 seg = b - a;
    float segLen = len(seg);
    if (segLen < 1e-7f) return;

    float maxH = 0.16f * P.diskOuter;
    if (a.y > maxH && b.y > maxH) return;
    if (a.y < -maxH && b.y < -maxH) return;

    float rcA = sqrtf(a.x * a.x + a.z * a.z);
    float rcB = sqrtf(b.x * b.x + b.z * b.z);
    float rcMin = fminf(rcA, rcB), rcMax = fmaxf(rcA, rcB);
    if (rcMin - segLen > P.diskOuter) return;
    if (rcMax + segLen < P.diskInner) return;

    int nSub = 1 + (int)(segLen * 6.5f);
    if (nSub > 12) nSub = 12;
    float ds = segLen / (float)nSub;

    const float emisK = P.diskEmisScale, absK = P.diskAbsScale;
    const float rin = fmaxf(P.diskInner, 1e-4f);
    const float invOut = 1.f / fmaxf(P.diskOuter, rin);
    const float M = P.M, aS = ph.a, Qc = ph.Q;

    for (int j = 0; j < nSub; ++j)
    {
        float t = ((float)j + 0.5f) / (float)nSub;
        F3 p = a + (b - a) * t;
        float rc = sqrtf(p.x * p.x + p.z * p.z);
        if (rc < rin || rc > P.diskOuter) continue;

        float HR = 0.040f + 0.015f * (rc * invOut);
        float H = HR * rc;
        float dz = p.y / fmaxf(H, 1e-4f);
        if (fabsf(dz) > 2.6f) continue;

        float Fr = thinDiskFlux(rc, rin) * kNtPeakInv;
        bool wantSpots = P.hotSpotsEnabled && P.hotSpotStrength > 1e-4f && rc < rin * 1.60f;
        if (Fr < 1e-6f && !wantSpots) continue;

        float dens = expf(-dz * dz);
        dens *= smooth(rin, rin * 1.10f, rc);
        dens *= 1.0f - smooth(P.diskOuter * 0.60f, P.diskOuter, rc);

        float omega = omegaCirc(rc, M, aS, Qc);
        if (omega <= 0.f) continue;
        float g = emitterG(rc, M, aS, Qc, ph.E, ph.Lz);
        if (g <= 0.f) continue;

        float azim = atan2f(-p.z, p.x);
        float azr = azim - omega * tEmit;
        float n0 = fbm3(rc * 3.6f, azr * 2.3f + rc * 0.8f);
        float st = vnoise(rc * 21.f - azr * 1.7f, azr * 3.5f + rc * 2.2f);
        dens *= (0.20f + 1.30f * n0) * (0.40f + 1.00f * st);
        dens *= dens;
        float psi1 = azim - 0.55f * omega * tEmit - 1.6f * logf(fmaxf(rc, 0.2f));
        dens *= (1.f + 0.38f * cosf(psi1));

        float spotBoost = 0.f, spotHeat = 0.f;
        if (wantSpots)
        {
            const float rH0 = rin * 1.06f, rH1 = rin * 1.18f;
            float om0 = omegaCirc(rH0, M, aS, Qc);
            float om1 = omegaCirc(rH1, M, aS, Qc);
            if (om0 <= 0.f) om0 = omega;
            if (om1 <= 0.f) om1 = omega;
            const float iPhi = 1.f / (2.f * 0.18f * 0.18f);
            const float iR0 = 1.f / (2.f * (0.09f * rH0) * (0.09f * rH0));
            const float iR1 = 1.f / (2.f * (0.11f * rH1) * (0.11f * rH1));
            float dph0 = wrapPi(azim - (om0 * tEmit + 0.4f));
            float dph1 = wrapPi(azim - (om1 * tEmit + 0.4f + kPi));
            float dr0 = rc - rH0, dr1 = rc - rH1;
            float fl0 = 0.72f + 0.28f * sinf(1.7f * tEmit + 0.9f);
            float fl1 = 0.65f + 0.35f * sinf(1.1f * tEmit + 2.3f);
            float g0 = expf(-(dph0 * dph0) * iPhi - dr0 * dr0 * iR0 - dz * dz * 0.45f);
            float g1 = expf(-(dph1 * dph1) * iPhi - dr1 * dr1 * iR1 - dz * dz * 0.45f);
            float S = P.hotSpotStrength;
            spotBoost = S * (5.0f * fl0 * g0 + 3.2f * fl1 * g1);
            spotHeat = S * (0.70f * fl0 * g0 + 0.45f * fl1 * g1);
            dens += dens * 0.25f * (g0 + g1) * S;
        }
        if (dens < 1e-5f && spotBoost < 1e-4f) continue;

        float Temit = kTInner * powf(Clamp(Fr, 1e-6f, 1.f), 0.25f);
        Temit = Clamp(Temit * (1.f + 1.6f * spotHeat), 2000.f, 26000.f);
        float Tobs = Clamp(Temit * g, 1200.f, 40000.f);
        F3 col = blackbody(Tobs);
        float g3 = g * g * g;
        float emis = Fr * g3 * g * (1.f + spotBoost);

        float w = dens * ds;
        F3 add = col * (emis * emisK * w);
        if (spotBoost > 1e-4f)
        {
            float wS = (0.12f + dens) * ds;
            add = add + col * (spotBoost * g3 * emisK * 0.55f * wS);
        }
        accum = accum + add * trans;

        float tau = absK * w * (1.f + 0.35f * dens);
        trans *= expf(-tau);
        tally.samples++;
        if (trans < 0.012f) return;
    }
}

/* ------------------------------------------------------------------------ */
/* Integrators (templated on the precision T)                               */
/* ------------------------------------------------------------------------ */
struct Ray
{
    bool horizon = false, escaped = false;
    F3 escDir{0.f, 0.f, 0.f};
    F3 accum{0.f, 0.f, 0.f};
    float trans = 1.f;
    float maxHviol = 0.f;
    int steps = 0;
    DiskTally tally;
    double drift = 0.0;
};

template <class T>
void conservedEL(V3<T> o, V3<T> dir, T M, T a, T Q, T& E, T& Lz)   /* trace.cuh:213-247 */
{
    T r0 = len(o);
    if (r0 < T(1e-4f)) { E = T(1); Lz = T(0); return; }
    T cth0 = Clamp(o.y / r0, T(-1), T(1));
    T th0 = Acos(cth0);
    T ph0 = Atan2(-o.z, o.x);
    T s = Sin(th0), c = Cos(th0);
    T sp = Sin(ph0), cp = Cos(ph0);
    (void)c;
    V3<T> eph = mk(-sp, T(0), -cp);
    T dpc = dot(dir, eph);
    T s0 = s; if (s0 < T(1e-4f)) s0 = T(1e-4f);
    T s02 = s0 * s0;
    T Sig0 = sigmaBL(r0, cth0, a);
    T m2r0 = T(2) * M * r0 - Q * Q;
    T gtt = -(T(1) - m2r0 / Fmax(Sig0, T(1e-8f)));
    if (gtt > T(-1e-5f)) gtt = T(-1e-5f);
    T gtp = -a * m2r0 * s02 / Sig0;
    T gpp = (r0 * r0 + a * a + m2r0 * a * a * s02 / Sig0) * s02;
    T A = Rsqrt(Fmax(gpp - gtp * gtp / gtt, T(1e-8f)));
    T ptUp = Rsqrt(-gtt) - dpc * A * gtp / gtt;
    T pfUp = dpc * A;
    E = -(gtt * ptUp + gtp * pfUp);
    Lz = gtp * ptUp + gpp * pfUp;
    if (!(E > T(1e-6f)) || !Finite(E)) { E = T(1); Lz = T(0); }
}

template <class T>
Ray traceSpherical(const RenderParams& P, V3<T> origin, V3<T> dir, bool wantStats)   /* trace.cuh:466-611 */
{
    Ray R;
    R.escDir = tof(dir);
    const T M = (T)P.M, Qc = (T)P.Qc;
    const T Q2 = Qc * Qc;
    const T rCap = (T)captureRadius(P);
    const T uHor = T(1) / Fmax(rCap, T(1e-6f));
    const T escR = T(120) * M;
    const T uEscape = T(1) / escR;
    const T dPhi = (T)P.dPhi;

    T Eph = T(1), Lph = T(0);
    conservedEL(origin, dir, M, T(0), Qc, Eph, Lph);
    const DiskPhoton ctx = {(float)Eph, (float)Lph, 0.f, P.Qc};

    V3<T> c = origin;
    T r0 = len(c);
    V3<T> e1 = divs(c, r0);
    T ddr = dot(dir, e1);
    V3<T> perp = dir - e1 * ddr;
    T pl = len(perp);
    if (pl < T(1e-6f))                              /* trace.cuh:447-459, 500-505 */
    {
        if (dot(dir, c) < T(0)) R.horizon = true;
        R.escaped = !R.horizon;
        R.escDir = tof(dir);
        return R;
    }
    V3<T> e2 = divs(perp, pl);

    T f0 = Fmax(sphF(r0, M, Qc), T(1e-6f));
    T bImpact = Fmax(r0 * pl / Sqrt(f0), T(1e-6f));
    T u = T(1) / r0;
    T du = -Sqrt(f0) * ddr / (r0 * pl);
    T phi = T(0);
    T tFlight = T(0);
    /* Binet first integral du^2 + u^2 (1 - 2Mu + Q^2 u^2) == 1/b^2 (addition) */
    auto binet = [&](T uu, T vv) { return (double)vv * vv + (double)uu * uu * (1.0 - 2.0 * (double)M * uu + (double)Q2 * uu * uu); };
    const double I0 = binet(u, du);

    V3<T> prevPos = c;
    V3<T> dir3 = dir;
    const T invNineM = T(1) / (T(9) * M);
    T h = dPhi;
    auto acc = [M, Q2](T uu) { return T(3) * M * uu * uu - T(2) * Q2 * uu * uu * uu - uu; };

    int step = 0;
    for (; step < P.maxSteps; ++step)
    {
        T hMax = dPhi * Clamp(invNineM / u, T(1), T(6));
        h = Fmin(hMax, T(0.10f) / Fmax(Fabs(du), T(1e-6f)));
        if (h < dPhi * T(0.03f)) h = dPhi * T(0.03f);

        const T uS = u, duS = du;
        T k1u = du;
        T k1v = acc(u);
        T u2 = u + T(0.5f) * h * k1u;
        T v2 = du + T(0.5f) * h * k1v;
        T k2u = v2;
        T k2v = acc(u2);
        T u3 = u + T(0.5f) * h * k2u;
        T v3 = du + T(0.5f) * h * k2v;
        T k3u = v3;
        T k3v = acc(u3);
        T u4 = u + h * k3u;
        T v4 = du + h * k3v;
        T k4u = v4;
        T k4v = acc(u4);
        u += (h / T(6)) * (k1u + T(2) * k2u + T(2) * k3u + k4u);
        du += (h / T(6)) * (k1v + T(2) * k2v + T(2) * k3v + k4v);
        phi += h;

        if (!Finite(u) || !Finite(du)) { R.horizon = true; break; }
        if (u >= uHor) { R.horizon = true; break; }
        if (u < T(1e-4f)) { R.escaped = true; R.escDir = tof(dir3); break; }

        T r = T(1) / u;
        T cp = Cos(phi), sp = Sin(phi);
        V3<T> m = e1 * cp + e2 * sp;
        V3<T> mp = e1 * (-sp) + e2 * cp;
        T drdphi = -du / (u * u);
        V3<T> pos = m * r;
        dir3 = unit(m * drdphi + mp * r);

        T fR = Fmax(sphF(r, M, Qc), T(1e-4f));
        tFlight += h * (r * r) / (bImpact * fR);
        if (wantStats)
        {   /* disk hit (addition): the plane crosses y = 0 at phi* = atan2(-e1y, e2y) + k pi */
            const double e1y = (double)e1.y, e2y = (double)e2.y;
            if (std::fabs(e1y) + std::fabs(e2y) >= 1e-12)
            {
                const double pc = std::atan2(-e1y, e2y), pi = 3.14159265358979323846;
                const double p0 = (double)phi - (double)h;
                double ps = pc + std::ceil((p0 - pc) / pi) * pi;
                if (ps <= p0) ps += pi;
                if (ps <= (double)phi)
                {
                    double uh = hermite(uS, u, duS, du, h, (ps - p0) / (double)h);
                    if (uh > 0.0) recordHit(P, R.tally, 1.0 / uh, ctx.E, ctx.Lz);
                }
            }
        }

        if (P.diskEnabled && R.trans > 0.01f)
            diskSegment(P, ctx, tof(prevPos), tof(pos), (float)((T)P.diskTime - tFlight),
                        R.accum, R.trans, R.tally);
        prevPos = pos;

        if (u < uEscape && du < T(0)) { R.escaped = true; R.escDir = tof(dir3); break; }
    }
    R.steps = step;
    if (!R.horizon && !R.escaped)
    {
        if (u > T(1) / Fmax(T(1.5f) * (T)P.rPhoton, T(3) * M)) R.horizon = true;
        else { R.escaped = true; R.escDir = tof(dir3); }
    }
    if (I0 > 0.0) R.drift = std::fabs(binet(u, du) - I0) / I0;
    return R;
}

template <class T> struct KS { T r, th, ph, pr, pth; };

template <class T>
inline void sincosT(T x, T& s, T& c) { s = Sin(x); c = Cos(x); }   /* trace.cuh:406-413 host branch */

template <class T>
KS<T> kerrRHS(T M, T a, T Q, T E, T Lz, const KS<T>& y, T& Kout)    /* trace.cuh:620-659 */
{
    T s, cth;
    sincosT(y.th, s, cth);
    if (s < T(1e-4f)) s = T(1e-4f);
    T s2 = s * s;
    T r = y.r;
    T r2 = r * r, a2 = a * a;
    T Sig = r2 + a2 * cth * cth;
    T Del = r2 - T(2) * M * r + a2 + Q * Q;
    if (Del < T(1e-6f)) Del = T(1e-6f);
    T Pp = E * (r2 + a2) - a * Lz;
    T B = Lz / s - a * E * s;
    T W = B * B - Pp * Pp / Del;
    T K = Del * y.pr * y.pr + y.pth * y.pth + W;
    Kout = K;
    T dDel = T(2) * r - T(2) * M;
    T dP = T(2) * r * E;
    T Wr = -(T(2) * Pp * dP * Del - Pp * Pp * dDel) / (Del * Del);
    T dB = -Lz * cth / s2 - a * E * cth;
    T Wth = T(2) * B * dB;
    T invS = T(1) / Sig;
    T invS2 = invS * invS;
    KS<T> d;
    d.r = Del * y.pr * invS;
    d.th = y.pth * invS;
    d.ph = ((Lz / s2 - a * E) + a * Pp / Del) * invS;
    d.pr = T(-0.5f) * invS * (dDel * y.pr * y.pr + Wr) + r * invS2 * K;
    d.pth = T(-0.5f) * invS * Wth - a2 * s * cth * invS2 * K;
    return d;
}

template <class T>
inline V3<T> kerrToCart(T r, T th, T ph)              /* trace.cuh:665-671 */
{
    T s, c, sp, cp;
    sincosT(th, s, c);
    sincosT(ph, sp, cp);
    return mk(r * s * cp, r * c, -r * s * sp);
}

template <class T>
inline void kerrBasis(T th, T ph, V3<T>& er, V3<T>& eth, V3<T>& eph)   /* trace.cuh:673-682 */
{
    T s, c, sp, cp;
    sincosT(th, s, c);
    sincosT(ph, sp, cp);
    er = mk(s * cp, c, -s * sp);
    eth = mk(c * cp, -s, -c * sp);
    eph = mk(-sp, T(0), -cp);
}

template <class T>
inline double carterQ(const KS<T>& y, T a, T E, T Lz)   /* addition: Carter constant */
{
    double s = std::sin((double)y.th), c = std::cos((double)y.th);
    double s2 = std::max(s * s, 1e-12);
    return (double)y.pth * y.pth + c * c * ((double)Lz * Lz / s2 - (double)a * a * (double)E * E);
}

template <class T>
Ray traceKerr(const RenderParams& P, V3<T> origin, V3<T> dir, bool wantStats)   /* trace.cuh:684-890 */
{
    Ray R;
    R.escDir = tof(dir);
    const T M = (T)P.M, a = (T)P.aSpin, Q = (T)P.Qc;
    const T rp = (T)P.rPlus;
    const T rCap = (T)captureRadius(P);
    const T rFloor = Fmax(rp, rCap);
    const T escR = T(120) * M;
    const T dPhi = (T)P.dPhi;

    T r0 = len(origin);
    T cth0 = Clamp(origin.y / r0, T(-1), T(1));
    T th0 = Acos(cth0);
    T ph0 = Atan2(-origin.z, origin.x);
    V3<T> er, eth, eph;
    kerrBasis(th0, ph0, er, eth, eph);
    T drc = dot(dir, er), dtc = dot(dir, eth), dpc = dot(dir, eph);

    T s0 = Sin(th0); if (s0 < T(1e-4f)) s0 = T(1e-4f);
    T s02 = s0 * s0;
    T Sig0 = sigmaBL(r0, cth0, a);
    T Del0 = deltaBL(r0, M, a, Q);
    T m2r0 = T(2) * M * r0 - Q * Q;
    T gtt = -(T(1) - m2r0 / Sig0);
    if (gtt > T(-1e-5f)) gtt = T(-1e-5f);
    T gtp = -a * m2r0 * s02 / Sig0;
    T gpp = (r0 * r0 + a * a + m2r0 * a * a * s02 / Sig0) * s02;
    T A = Rsqrt(Fmax(gpp - gtp * gtp / gtt, T(1e-8f)));
    T ptUp = Rsqrt(-gtt) - dpc * A * gtp / gtt;
    T pfUp = dpc * A;
    T E = -(gtt * ptUp + gtp * pfUp);
    T Lz = gtp * ptUp + gpp * pfUp;

    KS<T> y;
    y.r = r0; y.th = th0; y.ph = ph0;
    y.pr = drc * Sqrt(Sig0 / Fmax(Del0, T(1e-6f)));
    y.pth = dtc * Sqrt(Sig0);
    const double Q0 = carterQ(y, a, E, Lz);

    const DiskPhoton ctx = {(float)E, (float)Lz, P.aSpin, P.Qc};
    const T E2 = E * E;
    const bool trackPos = (P.diskEnabled != 0);
    T tFlight = T(0);
    V3<T> prevPos = origin;
    V3<T> dir3 = dir;
    KS<T> dLast{};
    bool haveDeriv = false;
    int step = 0;

    /* disk hit bookkeeping (addition): start of the previous step */
    double cR = 0, cTh = 0, cDr = 0, cDth = 0, cH = 0;
    for (; step < P.maxSteps; ++step)
    {
        T Kv;
        KS<T> d1 = kerrRHS(M, a, Q, E, Lz, y, Kv);
        if (wantStats && step > 0)
            kerrCrossing(P, R.tally, cR, cTh, cDr, cDth, y.r, y.th, d1.r, d1.th, cH, ctx.E, ctx.Lz);
        if (!Finite(y.r) || !Finite(y.pr) || !Finite(y.pth) || !Finite(d1.r) || !Finite(d1.pr))
        { R.horizon = true; break; }
        if (y.r <= rCap * T(1.002f) + T(1e-3f)) { R.horizon = true; break; }
        if (wantStats && y.r > rFloor * T(1.05f))
        {
            T viol = Fabs(Kv) / (E2 * (y.r * y.r + a * a) + T(1e-12f));
            if ((float)viol > R.maxHviol) R.maxHviol = (float)viol;
        }
        if (y.r >= escR && d1.r > T(0))
        {
            V3<T> e1b, e2b, e3b;
            kerrBasis(y.th, y.ph, e1b, e2b, e3b);
            T s = Sin(y.th);
            R.escDir = tof(unit(e1b * d1.r + e2b * (y.r * d1.th) + e3b * (y.r * s * d1.ph)));
            R.escaped = true;
            break;
        }

        T h = T(1) / (Fabs(d1.r) / (T(8.0f) * dPhi * Fmax(y.r - rFloor, T(0.02f)))
                      + (Fabs(d1.th) + Fabs(d1.ph)) / (T(2.2f) * dPhi) + T(1e-5f));
        if (y.r < T(1.5f) * (T)P.rPhoton) h *= T(0.55f);
        T spd = Fabs(d1.r) + y.r * (Fabs(d1.th) + Fabs(d1.ph)) + T(1e-6f);
        T capLen;
        if (trackPos && y.r < (T)P.diskOuter * T(1.3f))
        {
            T yAbs = y.r * Fabs(Cos(y.th));
            capLen = (yAbs < T(1.8f)) ? T(1.2f) : T(2.2f);
        }
        else capLen = Fmax(T(1.2f), T(0.22f) * y.r);
        h = Fmin(h, capLen / spd);

        cR = y.r; cTh = y.th; cDr = d1.r; cDth = d1.th; cH = h;
        T kv2, kv3, kv4;
        KS<T> y2 = {y.r + T(0.5f) * h * d1.r, y.th + T(0.5f) * h * d1.th,
                    y.ph + T(0.5f) * h * d1.ph, y.pr + T(0.5f) * h * d1.pr,
                    y.pth + T(0.5f) * h * d1.pth};
        KS<T> d2 = kerrRHS(M, a, Q, E, Lz, y2, kv2);
        KS<T> y3 = {y.r + T(0.5f) * h * d2.r, y.th + T(0.5f) * h * d2.th,
                    y.ph + T(0.5f) * h * d2.ph, y.pr + T(0.5f) * h * d2.pr,
                    y.pth + T(0.5f) * h * d2.pth};
        KS<T> d3 = kerrRHS(M, a, Q, E, Lz, y3, kv3);
        KS<T> y4 = {y.r + h * d3.r, y.th + h * d3.th, y.ph + h * d3.ph,
                    y.pr + h * d3.pr, y.pth + h * d3.pth};
        KS<T> d4 = kerrRHS(M, a, Q, E, Lz, y4, kv4);

        T h6 = h / T(6);
        y.r += h6 * (d1.r + T(2) * d2.r + T(2) * d3.r + d4.r);
        y.th += h6 * (d1.th + T(2) * d2.th + T(2) * d3.th + d4.th);
        y.ph += h6 * (d1.ph + T(2) * d2.ph + T(2) * d3.ph + d4.ph);
        y.pr += h6 * (d1.pr + T(2) * d2.pr + T(2) * d3.pr + d4.pr);
        y.pth += h6 * (d1.pth + T(2) * d2.pth + T(2) * d3.pth + d4.pth);

        if (y.th < T(1e-3f)) { y.th = T(1e-3f); y.pth = Fabs(y.pth); }
        else if (y.th > (T)kPi - T(1e-3f)) { y.th = (T)kPi - T(1e-3f); y.pth = -Fabs(y.pth); }

        dLast = d4;
        haveDeriv = true;

        {   /* slow light, trace.cuh:840-851 */
            T s, cth;
            sincosT(y.th, s, cth);
            if (s < T(1e-4f)) s = T(1e-4f);
            T Sig = sigmaBL(y.r, cth, a);
            T Del = Fmax(deltaBL(y.r, M, a, Q), T(1e-5f));
            T Pp = E * (y.r * y.r + a * a) - a * Lz;
            T dtdl = (a * (Lz - a * E * s * s) + (y.r * y.r + a * a) * Pp / Del) / Fmax(Sig, T(1e-8f));
            tFlight += h * Fabs(dtdl);
        }

        if (trackPos)
        {
            V3<T> pos = kerrToCart(y.r, y.th, y.ph);
            V3<T> stepv = pos - prevPos;
            T sl = len(stepv);
            if (sl > T(1e-6f)) dir3 = stepv * (T(1) / sl);
            if (R.trans > 0.01f)
                diskSegment(P, ctx, tof(prevPos), tof(pos), (float)((T)P.diskTime - tFlight),
                            R.accum, R.trans, R.tally);
            prevPos = pos;
        }
    }
    R.steps = step;
    if (wantStats && step >= P.maxSteps && step > 0)
    {   /* budget spent: the last step's crossing */
        T Kv;
        KS<T> dEnd = kerrRHS(M, a, Q, E, Lz, y, Kv);
        kerrCrossing(P, R.tally, cR, cTh, cDr, cDth, y.r, y.th, dEnd.r, dEnd.th, cH, ctx.E, ctx.Lz);
    }
    if (!R.horizon && !R.escaped)
    {
        if (y.r < T(6) * M) R.horizon = true;
        else
        {
            R.escaped = true;
            if (haveDeriv)
            {
                V3<T> e1b, e2b, e3b;
                kerrBasis(y.th, y.ph, e1b, e2b, e3b);
                T s = Sin(y.th);
                R.escDir = tof(unit(e1b * dLast.r + e2b * (y.r * dLast.th) + e3b * (y.r * s * dLast.ph)));
            }
            else R.escDir = tof(dir3);
        }
    }
    const double Q1 = carterQ(y, a, E, Lz);
    const double scale = std::fabs(Q0) + (double)Lz * Lz + (double)a * a * (double)E * E;
    if (scale > 0.0) R.drift = std::fabs(Q1 - Q0) / scale;
    return R;
}

template <class T>
Ray traceRay(const RenderParams& P, F3 origin, F3 dir, bool wantStats)   /* trace.cuh:895-902 */
{
    if (P.model == BH_KERR || P.model == BH_KERR_NEWMAN)
        return traceKerr<T>(P, cvt<T>(origin), cvt<T>(dir), wantStats);
    return traceSpherical<T>(P, cvt<T>(origin), cvt<T>(dir), wantStats);
}

Ray traceAny(const RenderParams& P, F3 origin, F3 dir, bool wantStats, int precision)
{
    return precision == BH_PREC_FP64 ? traceRay<double>(P, origin, dir, wantStats)
                                     : traceRay<float>(P, origin, dir, wantStats);
}

F3 shade(const RenderParams& P, const Ray& t, float gCam)   /* trace.cuh:917-925 */
{
    F3 bg = t.horizon ? mk(0.f, 0.f, 0.f) : skyColor(t.escDir, gCam);
    F3 hdr = t.accum + bg * t.trans;
    if (!std::isfinite(hdr.x) || !std::isfinite(hdr.y) || !std::isfinite(hdr.z))
        hdr = mk(0.f, 0.f, 0.f);
    return hdr;
}

void fillProbe(BHProbe& o, const Ray& t, F3 hdr)
{
    o.outcome = t.escaped ? 1 : 0;
    o.cls = (t.trans < 0.5f) ? 1 : (t.horizon ? 0 : 2);
    o.steps = t.steps;
    o.diskSamples = t.tally.samples;
    o.escDir[0] = t.escDir.x; o.escDir[1] = t.escDir.y; o.escDir[2] = t.escDir.z;
    o.trans = t.trans;
    o.accum[0] = t.accum.x; o.accum[1] = t.accum.y; o.accum[2] = t.accum.z;
    o.maxHviol = t.maxHviol;
    o.hdr[0] = hdr.x; o.hdr[1] = hdr.y; o.hdr[2] = hdr.z;
    o.diskR = t.tally.hitR;
    o.diskG = t.tally.hitG;
    o.drift = (float)t.drift;
}

/* ------------------------------------------------------------------------ */
/* Post-processing: post_process.cuh:34-148, black_hole_kernel.cu:22-103     */
/* ------------------------------------------------------------------------ */
inline F3 aces(F3 x)                                     /* post_process.cuh:34-40 */
{
    const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
    F3 num = x * (x * A + mk(B, B, B));
    F3 den = x * (x * C + mk(D, D, D)) + mk(E, E, E);
    return mk(Clamp(num.x / den.x, 0.f, 1.f), Clamp(num.y / den.y, 0.f, 1.f), Clamp(num.z / den.z, 0.f, 1.f));
}

inline void jitter(int mode, int idx, float& jx, float& jy)   /* post_process.cuh:47-53 */
{
    if (mode == 0 || idx <= 0) { jx = 0.5f; jy = 0.5f; return; }
    float n = (float)idx;
    jx = fract(0.7548776662f * n + 0.5f);
    jy = fract(0.5698402909f * n + 0.5f);
}

inline F3 blend(F3 prev, F3 cur, int mode, int idx)      /* post_process.cuh:56-68 */
{
    if (mode == 0 || idx <= 0) return cur;
    if (mode == 1)
    {
        float n = (float)idx;
        return prev + (cur - prev) * (1.0f / (n + 1.0f));
    }
    return prev + (cur - prev) * 0.42f;
}

inline F3 brightPass(F3 c)                               /* post_process.cuh:76-84 */
{
    float l = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
    return c * smooth(0.95f, 2.2f, l);
}

inline float gaussW(int i)                               /* post_process.cuh:88-93 */
{
    static const float w[5] = {0.20236f, 0.17925f, 0.12458f, 0.06794f, 0.02907f};
    int k = i < 0 ? -i : i;
    return w[k > 4 ? 4 : k];
}

inline F3 fetchHalf(const float* buf, int x, int y, int bw, int bh)   /* post_process.cuh:96-104 */
{
    if (x < 0) x = 0;
    if (x >= bw) x = bw - 1;
    if (y < 0) y = 0;
    if (y >= bh) y = bh - 1;
    const float* v = buf + 4 * ((size_t)y * bw + x);
    return mk(v[0], v[1], v[2]);
}

inline F3 halfBilinear(const float* buf, float x, float y, int bw, int bh)   /* post_process.cuh:106-117 */
{
    x -= 0.5f; y -= 0.5f;
    int x0 = (int)floorf(x), y0 = (int)floorf(y);
    float tx = x - (float)x0, ty = y - (float)y0;
    F3 c00 = fetchHalf(buf, x0, y0, bw, bh);
    F3 c10 = fetchHalf(buf, x0 + 1, y0, bw, bh);
    F3 c01 = fetchHalf(buf, x0, y0 + 1, bw, bh);
    F3 c11 = fetchHalf(buf, x0 + 1, y0 + 1, bw, bh);
    F3 top = c00 + (c10 - c00) * tx;
    F3 bot = c01 + (c11 - c01) * tx;
    return top + (bot - top) * ty;
}

inline void finalize(F3 hdr, F3 bloom, const RenderParams& P, int px, int py, uint8_t* o)
{                                                        /* post_process.cuh:122-148 */
    F3 c = hdr * P.exposure;
    if (P.bloomEnabled) c = c + bloom * P.bloomStrength;
    c = aces(c);
    float lum = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
    F3 lv = mk(lum, lum, lum);
    F3 v = lv + (c - lv) * 1.12f;
    c = mk(Clamp(v.x, 0.f, 1.f), Clamp(v.y, 0.f, 1.f), Clamp(v.z, 0.f, 1.f));
    c = mk(powf(c.x, 1.0f / 2.2f), powf(c.y, 1.0f / 2.2f), powf(c.z, 1.0f / 2.2f));
    float fx = (float)px, fy = (float)py;
    float d = (hash12(fx, fy) + hash12(fx + 41.3f, fy + 17.7f)) - 1.0f;
    float dd = d * (1.0f / 255.0f);
    uint8_t r8 = (uint8_t)(Clamp(c.x + dd, 0.f, 1.f) * 255.f + 0.5f);
    uint8_t g8 = (uint8_t)(Clamp(c.y + dd, 0.f, 1.f) * 255.f + 0.5f);
    uint8_t b8 = (uint8_t)(Clamp(c.z + dd, 0.f, 1.f) * 255.f + 0.5f);
    if (P.swapRB) { o[0] = b8; o[1] = g8; o[2] = r8; }
    else { o[0] = r8; o[1] = g8; o[2] = b8; }
    o[3] = 255;
}

F3 sampleHDR(const RenderParams& P, int px, int py, float jx, float jy, float gCam,
             int precision, Ray* rayOut)                 /* trace.cuh:908-926 */
{
    float fx = ((float)px + jx) / (float)P.width;
    float fy = ((float)py + jy) / (float)P.height;
    F3 dir = cameraRay(P, fx, fy);
    Ray t = traceAny(P, fromF3(P.camPos), dir, false, precision);
    if (rayOut) *rayOut = t;
    return shade(P, t, gCam);
}

int threadsOr(int n) { return n > 0 ? n : omp_get_max_threads(); }

}  // namespace

/* ========================================================================= */
/* C ABI used by the tests (ctypes)                                          */
/* ========================================================================= */
extern "C" {

int orc_sanitize(RenderParams* p) { return sanitize(*p) ? 1 : 0; }

void orc_derive(int model, float* M, float* aStar, float* q, int allowNaked, BHDerived* out)
{
    *out = derive(model, *M, *aStar, *q, allowNaked != 0);
}

float orc_camera_energy(const RenderParams* p) { return cameraEnergy(*p); }

/* Reference test probe (tests/test_main.cu:71-89): pixel-centre grid rays,
 * constraint monitor on.  `stepDiv` > 1 divides dPhi and multiplies the step
 * budget (small-step oracle).  No sanitising, as in the reference probe. */
void orc_probe_grid(const RenderParams* p, int nx, int ny, int precision, int stepDiv,
                    BHProbe* out, int nthreads)
{
    RenderParams P = *p;
    if (stepDiv > 1) { P.dPhi = P.dPhi / (float)stepDiv; P.maxSteps = P.maxSteps * stepDiv; }
    const float gCam = cameraEnergy(P);
#pragma omp parallel for schedule(dynamic, 4) num_threads(threadsOr(nthreads))
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
        {
            float fx = (i + 0.5f) / (float)nx;
            float fy = (j + 0.5f) / (float)ny;
            F3 dir = cameraRay(P, fx, fy);
            Ray t = traceAny(P, fromF3(P.camPos), dir, true, precision);
            fillProbe(out[(size_t)j * nx + i], t, shade(P, t, gCam));
        }
}

/* Arbitrary directions from the camera (tests/test_main.cu:91-98). */
void orc_probe_dirs(const RenderParams* p, const float* dirs, int n, int precision, int stepDiv,
                    BHProbe* out, int nthreads)
{
    RenderParams P = *p;
    if (stepDiv > 1) { P.dPhi = P.dPhi / (float)stepDiv; P.maxSteps = P.maxSteps * stepDiv; }
    const float gCam = cameraEnergy(P);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threadsOr(nthreads))
    for (int k = 0; k < n; ++k)
    {
        F3 dir = mk(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]);
        Ray t = traceAny(P, fromF3(P.camPos), dir, true, precision);
        fillProbe(out[k], t, shade(P, t, gCam));
    }
}

/* Selected pixels of a frame, traced exactly as the render path does
 * (sanitised params, pipeline jitter, constraint monitor off).  Used for the
 * per-frame work census and as the CPU baseline sample. */
void orc_trace_pixels(const RenderParams* p, const int* pix, int n, int precision, BHProbe* out,
                      int nthreads)
{
    RenderParams P = *p;
    sanitize(P);
    const float gCam = cameraEnergy(P);
    float jx, jy;
    jitter(P.accumMode, P.sampleIndex, jx, jy);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threadsOr(nthreads))
    for (int k = 0; k < n; ++k)
    {
        int px = pix[k] % P.width, py = pix[k] / P.width;
        Ray t;
        F3 hdr = sampleHDR(P, px, py, jx, jy, gCam, precision, &t);
        fillProbe(out[k], t, hdr);
    }
}

/* One HDR sample per pixel (renderSampleHDR), sanitised params. */
void orc_render_hdr(const RenderParams* p, int precision, float* hdr, BHProbe* rays, int nthreads)
{
    RenderParams P = *p;
    sanitize(P);
    const float gCam = cameraEnergy(P);
    float jx, jy;
    jitter(P.accumMode, P.sampleIndex, jx, jy);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threadsOr(nthreads))
    for (int py = 0; py < P.height; ++py)
        for (int px = 0; px < P.width; ++px)
        {
            size_t idx = (size_t)py * P.width + px;
            Ray t;
            F3 c = sampleHDR(P, px, py, jx, jy, gCam, precision, &t);
            hdr[4 * idx + 0] = c.x; hdr[4 * idx + 1] = c.y; hdr[4 * idx + 2] = c.z; hdr[4 * idx + 3] = 1.f;
            if (rays) fillProbe(rays[idx], t, c);
        }
}

}  // extern "C"

namespace {
/* Post-processing with already-sanitised params: black_hole_kernel.cu:41-103. */
void postImpl(uint8_t* out, const float* accum, float* bloomA, float* bloomB, const RenderParams& P,
              int nthreads)
{
    const int W = P.width, H = P.height;
    const int bw = (W + 1) / 2, bh = (H + 1) / 2;
    const int nt = threadsOr(nthreads);
    if (P.bloomEnabled)
    {
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                      /* black_hole_kernel.cu:41-62 */
            for (int x = 0; x < bw; ++x)
            {
                int x0 = x * 2, y0 = y * 2;
                int x1 = (x0 + 1 < W) ? x0 + 1 : x0;
                int y1 = (y0 + 1 < H) ? y0 + 1 : y0;
                const float* a = accum + 4 * ((size_t)y0 * W + x0);
                const float* b = accum + 4 * ((size_t)y0 * W + x1);
                const float* c = accum + 4 * ((size_t)y1 * W + x0);
                const float* d = accum + 4 * ((size_t)y1 * W + x1);
                F3 avg = mk(a[0] + b[0] + c[0] + d[0], a[1] + b[1] + c[1] + d[1],
                            a[2] + b[2] + c[2] + d[2]) * 0.25f;
                F3 bp = brightPass(avg * P.exposure);
                float* o = bloomA + 4 * ((size_t)y * bw + x);
                o[0] = bp.x; o[1] = bp.y; o[2] = bp.z; o[3] = 1.f;
            }
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                      /* black_hole_kernel.cu:64-73 */
            for (int x = 0; x < bw; ++x)
            {
                F3 s = mk(0.f, 0.f, 0.f);
                for (int k = -4; k <= 4; ++k) s = s + fetchHalf(bloomA, x + k, y, bw, bh) * gaussW(k);
                float* o = bloomB + 4 * ((size_t)y * bw + x);
                o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = 1.f;
            }
#pragma omp parallel for num_threads(nt)
        for (int y = 0; y < bh; ++y)                      /* black_hole_kernel.cu:75-84 */
            for (int x = 0; x < bw; ++x)
            {
                F3 s = mk(0.f, 0.f, 0.f);
                for (int k = -4; k <= 4; ++k) s = s + fetchHalf(bloomB, x, y + k, bw, bh) * gaussW(k);
                float* o = bloomA + 4 * ((size_t)y * bw + x);
                o[0] = s.x; o[1] = s.y; o[2] = s.z; o[3] = 1.f;
            }
    }
#pragma omp parallel for num_threads(nt)
    for (int py = 0; py < H; ++py)                        /* black_hole_kernel.cu:86-103 */
        for (int px = 0; px < W; ++px)
        {
            const float* av = accum + 4 * ((size_t)py * W + px);
            F3 bloom = mk(0.f, 0.f, 0.f);
            if (P.bloomEnabled)
                bloom = halfBilinear(bloomA, (px + 0.5f) * 0.5f, (py + 0.5f) * 0.5f, bw, bh);
            finalize(mk(av[0], av[1], av[2]), bloom, P, px, py, out + 4 * ((size_t)py * W + px));
        }
}
}  // namespace

extern "C" {

/* Post-processing of an existing accumulation buffer. */
void orc_post(uint8_t* out, const float* accum, float* bloomA, float* bloomB, const RenderParams* p,
              int nthreads)
{
    RenderParams P = *p;
    sanitize(P);
    postImpl(out, accum, bloomA, bloomB, P, nthreads);
}

/* launchRenderPipeline semantics (black_hole_kernel.cu:108-134). */
void orc_pipeline(uint8_t* out, float* accum, float* bloomA, float* bloomB, const RenderParams* p,
                  int precision, int nthreads)
{
    RenderParams P = *p;
    sanitize(P);
    const float gCam = cameraEnergy(P);
    float jx, jy;
    jitter(P.accumMode, P.sampleIndex, jx, jy);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threadsOr(nthreads))
    for (int py = 0; py < P.height; ++py)                 /* black_hole_kernel.cu:22-39 */
        for (int px = 0; px < P.width; ++px)
        {
            F3 cur = sampleHDR(P, px, py, jx, jy, gCam, precision, nullptr);
            float* a = accum + 4 * ((size_t)py * P.width + px);
            F3 prev = mk(a[0], a[1], a[2]);
            if (!std::isfinite(prev.x) || !std::isfinite(prev.y) || !std::isfinite(prev.z)) prev = cur;
            F3 c = blend(prev, cur, P.accumMode, P.sampleIndex);
            a[0] = c.x; a[1] = c.y; a[2] = c.z; a[3] = 1.f;
        }
    postImpl(out, accum, bloomA, bloomB, P, nthreads);
}

/* launchRenderKernel semantics (black_hole_kernel.cu:140-163). */
void orc_render_kernel(uint8_t* out, const RenderParams* p, int precision, int nthreads)
{
    RenderParams P = *p;
    sanitize(P);
    P.bloomEnabled = 0;
    const float gCam = cameraEnergy(P);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threadsOr(nthreads))
    for (int py = 0; py < P.height; ++py)
        for (int px = 0; px < P.width; ++px)
        {
            F3 hdr = sampleHDR(P, px, py, 0.5f, 0.5f, gCam, precision, nullptr);
            finalize(hdr, mk(0.f, 0.f, 0.f), P, px, py, out + 4 * ((size_t)py * P.width + px));
        }
}

}  // extern "C"
