// ---------------------------------------------------------------------------
// bh_camera.cpp -- camera-frame constants of a view (host, once per frame).
//
// The reference integrators begin every ray by rebuilding the same camera
// quantities: Boyer-Lindquist angles of the camera, the orthonormal basis
// there, the metric and the static-observer tetrad (Sqhh99/Black-hole
// src/trace.cuh:213-247 for the photon constants of the spherical path,
// 490-521 for its orbital-plane set-up, 703-739 for the Kerr-Newman path).
// Only the projections of the ray direction onto that frame differ per ray.
// This file evaluates the shared part once, with the reference's float (or
// double) arithmetic and libm calls, compiled without FMA contraction, so the
// device only has to apply the per-ray remainder (bh_integrate.cuh).
// ---------------------------------------------------------------------------
#include <cmath>
#include "bh_trace_params.h"

namespace {

inline float sqrtT(float x) { return std::sqrt(x); }
inline double sqrtT(double x) { return std::sqrt(x); }
inline float acosT(float x) { return std::acos(x); }
inline double acosT(double x) { return std::acos(x); }
inline float atan2T(float y, float x) { return std::atan2(y, x); }
inline double atan2T(double y, double x) { return std::atan2(y, x); }
inline float sinT(float x) { return std::sin(x); }
inline double sinT(double x) { return std::sin(x); }
inline float cosT(float x) { return std::cos(x); }
inline double cosT(double x) { return std::cos(x); }
template <class T> inline T fmaxT(T a, T b) { return std::fmax(a, b); }
template <class T> inline T fminT(T a, T b) { return std::fmin(a, b); }

template <class T>
void fill(CamFrame<T>& f, const TraceParams& t, float3 pos, float Mf, float af, float Qf)
{
    const T M = (T)Mf, a = (T)af, Q = (T)Qf;
    const T ox = (T)pos.x, oy = (T)pos.y, oz = (T)pos.z;
    const T r0 = sqrtT(ox * ox + oy * oy + oz * oz);
    f.r0 = r0;

    // ---- rotating family: trace.cuh:704-739 ------------------------------------
    const T cth0 = fminT(fmaxT(oy / r0, T(-1)), T(1));
    const T th0 = acosT(cth0);
    const T ph0 = atan2T(-oz, ox);
    f.th0 = th0;
    f.ph0 = ph0;
    const T s = sinT(th0), c = cosT(th0), sp = sinT(ph0), cp = cosT(ph0);
    f.er[0] = s * cp;  f.er[1] = c;   f.er[2] = -s * sp;
    f.eth[0] = c * cp; f.eth[1] = -s; f.eth[2] = -c * sp;
    f.eph[0] = -sp;    f.eph[1] = T(0); f.eph[2] = -cp;
    {
        T s0 = s;
        if (s0 < T(1e-4f)) s0 = T(1e-4f);
        const T s02 = s0 * s0;
        const T Sig0 = r0 * r0 + a * a * cth0 * cth0;
        const T Del0 = r0 * r0 - T(2) * M * r0 + a * a + Q * Q;
        const T m2r0 = T(2) * M * r0 - Q * Q;
        T gtt = -(T(1) - m2r0 / Sig0);
        if (gtt > T(-1e-5f)) gtt = T(-1e-5f);
        const T gtp = -a * m2r0 * s02 / Sig0;
        const T gpp = (r0 * r0 + a * a + m2r0 * a * a * s02 / Sig0) * s02;
        f.gtt = gtt; f.gtp = gtp; f.gpp = gpp;
        f.A = T(1) / sqrtT(fmaxT(gpp - gtp * gtp / gtt, T(1e-8f)));
        f.rsq = T(1) / sqrtT(-gtt);
        f.sqSD = sqrtT(Sig0 / fmaxT(Del0, T(1e-6f)));
        f.sqS = sqrtT(Sig0);
    }

    // ---- spherical family: photon constants (trace.cuh:213-247, a = 0) ------------
    f.camAtOrigin = (r0 < T(1e-4f)) ? 1 : 0;
    f.ephS[0] = -sp; f.ephS[1] = T(0); f.ephS[2] = -cp;
    {
        T s0 = s;
        if (s0 < T(1e-4f)) s0 = T(1e-4f);
        const T s02 = s0 * s0;
        const T z = T(0);
        const T Sig0 = r0 * r0 + z * z * cth0 * cth0;
        const T m2r0 = T(2) * M * r0 - Q * Q;
        T gtt = -(T(1) - m2r0 / fmaxT(Sig0, T(1e-8f)));
        if (gtt > T(-1e-5f)) gtt = T(-1e-5f);
        const T gtp = -z * m2r0 * s02 / Sig0;
        const T gpp = (r0 * r0 + z * z + m2r0 * z * z * s02 / Sig0) * s02;
        f.gttS = gtt; f.gtpS = gtp; f.gppS = gpp;
        f.AS = T(1) / sqrtT(fmaxT(gpp - gtp * gtp / gtt, T(1e-8f)));
        f.rsqS = T(1) / sqrtT(-gtt);
    }
    // orbital-plane set-up (trace.cuh:490-521)
    const T inv = T(1) / r0;
    f.e1[0] = ox * inv; f.e1[1] = oy * inv; f.e1[2] = oz * inv;
    f.f0 = fmaxT(T(1) - T(2) * M / r0 + Q * Q / (r0 * r0), T(1e-6f));
    f.sf0 = sqrtT(f.f0);
    f.u0 = T(1) / r0;

    // ---- step-loop constants: trace.cuh:477-482, 537, 548-550, 607, 696-701, 761-808, 874
    const T rCap = (T)t.rCap, dPhi = (T)t.dPhi;
    f.M = M; f.a = a; f.Q2 = Q * Q; f.a2 = a * a; f.a2Q2 = f.a2 + f.Q2;
    f.capR = rCap * T(1.002f) + T(1e-3f);
    f.rFloor = fmaxT((T)t.rPlus, rCap);
    f.rFloor105 = f.rFloor * T(1.05f);
    f.escR = T(120) * M;
    f.sixM = T(6) * M;
    f.k8dPhi = T(8.0f) * dPhi;
    f.i22dPhi = T(1) / (T(2.2f) * dPhi);
    f.rPh15 = T(1.5f) * (T)t.rPhoton;
    f.outer13 = (T)t.diskOuter * T(1.3f);
    f.dPhi = dPhi;
    f.hMin = dPhi * T(0.03f);
    f.uHor = T(1) / fmaxT(rCap, T(1e-6f));
    f.uEscape = T(1) / (T(120) * M);
    f.invNineM = T(1) / (T(9) * M);
    f.uPh = T(1) / fmaxT(T(1.5f) * (T)t.rPhoton, T(3) * M);
    f.diskTime = (T)t.diskTime;
}

}  // namespace

void bh_fill_camera_frames(TraceParams& t)
{
    fill(t.cf, t, t.camPos, t.M, t.a, t.Q);
    fill(t.cd, t, t.camPos, t.M, t.a, t.Q);
}
