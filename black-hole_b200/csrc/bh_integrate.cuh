#pragma once
// ---------------------------------------------------------------------------
// bh_integrate.cuh -- the two geodesic integrators as resumable ray objects.
//
// Each integrator is split into init() / advance() / pack() so that a warp
// can hold 32 independent rays in registers and refill any lane whose ray
// ended (bh_trace.cu).  The arithmetic per step is the reference's method
// (Sqhh99/Black-hole):
//   SphRay   generalised Binet equation u'' = 3Mu^2 - 2Q^2u^3 - u, RK4 in the
//            orbital angle with the adaptive step of src/trace.cuh:466-611
//   KerrRay  Boyer-Lindquist Hamiltonian system (r, th, ph, p_r, p_th) with the
//            full dH derivatives (src/trace.cuh:620-659), static-observer
//            tetrad initial data (:704-739), adaptive affine step (:784-809),
//            RK4, pole guard, slow light and disk chords (:811-868)
// Termination tests and their order are the reference's, so step counts and
// outcomes agree ray by ray except where floating-point rounding decides.
//
// Initial data: the camera-frame part is precomputed on the host (CamFrame);
// the per-ray remainder here uses exact (correctly rounded, uncontracted)
// operations, so every ray starts from the reference's initial state bit for
// bit.  R is the integration precision (float: product path; double: GPU
// accuracy oracle).  Shading stays float in both.
//
// Arithmetic of the FP32 step: divisions by state-dependent quantities use one
// MUFU reciprocal each; sin/cos of the polar angle (at the start of a step and
// at the three RK4 stage angles) use the MUFU pair, replaced by the polynomial
// sincos_polar where |sin| < 1/16 so the pole terms keep relative accuracy; the
// pair at the start of a step is carried into the next step's first
// right-hand side, the slow-light term and the Cartesian chord; the
// ever-growing azimuth uses sincos_fast.  The escape direction is rebuilt once
// per ray with the accurate library sincos.
// ---------------------------------------------------------------------------
#include <type_traits>
#include "bh_shade.cuh"
#include "bh_internal.h"

enum { RAY_SKIP = 0, RAY_LIVE = 1, RAY_DONE = 2 };

// MIXED precision: the polar cap |sin th| < kPolarCap (0.9 deg) inside which a
// Kerr-family ray carries an FP64 state (KerrRay::polar_passage_fp64).  Measured
// on the 4K near-extremal sweep at 89 deg elevation (480x270, escape directions
// within 1e-4 rad of the FP64 integration): no cap 98.6 %, 1/64 99.79 %, 1/32
// 99.93 %, 1/16 99.93 %; frame time against FP32 at 0 / 45 / 89 deg: 1.5 / 1.6 /
// 2.4x at 1/64, 2.1 / 2.3 / 3.2x at 1/32, 2.8 / 3.2 / 4.0x at 1/16 (a warp
// waits for its lanes' FP64 passages).
constexpr float kPolarCap = 1.0f / 64.0f;

// A finished ray as it waits for shading: outcome flags, the radiance gathered
// from the disk, and the six state values from which the escape direction is
// rebuilt at shading time (so the finishing lane only stores, and the
// trigonometry runs later with the whole warp converged).  The key holds the
// ray's pixel (or list position) in its low 28 bits and four flags above:
// captured, escaped, escape direction from the state, step budget spent.
constexpr unsigned kRayHorizon = 1u << 31, kRayEscaped = 1u << 30, kRayUseState = 1u << 29,
                   kRayExhausted = 1u << 28;
constexpr unsigned kRayKeyMask = kRayExhausted - 1u;
static_assert(kRayKeyMask + 1u == BH_MAX_RAYS, "ray key width");

template <class R>
struct PackedRay
{
    unsigned key;         // pixel index or ray id | kRay* flags
    float acc[3];
    float trans;
    R f[6];               // family-specific escape state
};

struct PackedStats
{
    int steps, samples;
    float maxHviol, drift, hitR, hitG;
};

// ---- exact single operations in either precision --------------------------------
BH_DEV float xmul(float a, float b) { return __fmul_rn(a, b); }
BH_DEV double xmul(double a, double b) { return __dmul_rn(a, b); }
BH_DEV float xadd(float a, float b) { return __fadd_rn(a, b); }
BH_DEV double xadd(double a, double b) { return __dadd_rn(a, b); }
BH_DEV float xsub(float a, float b) { return __fsub_rn(a, b); }
BH_DEV double xsub(double a, double b) { return __dsub_rn(a, b); }
BH_DEV float xdiv(float a, float b) { return __fdiv_rn(a, b); }
BH_DEV double xdiv(double a, double b) { return __ddiv_rn(a, b); }
BH_DEV float xsqrt(float a) { return __fsqrt_rn(a); }
BH_DEV double xsqrt(double a) { return __dsqrt_rn(a); }
template <class R> BH_DEV R xdot(const R* e, vec3<R> d)
{
    return xadd(xadd(xmul(d.x, e[0]), xmul(d.y, e[1])), xmul(d.z, e[2]));
}

template <class R> BH_DEV const CamFrame<R>& frame_of(const TraceParams& P);
template <> BH_DEV const CamFrame<float>& frame_of<float>(const TraceParams& P) { return P.cf; }
template <> BH_DEV const CamFrame<double>& frame_of<double>(const TraceParams& P) { return P.cd; }

BH_DEV f3 camera_ray(const TraceParams& P, float fx, float fy)
{
    // reference src/trace.cuh:431-438, in exact arithmetic (bit-identical to a host build)
    float nx = sub_x(mul_x(fx, 2.f), 1.f);
    float ny = sub_x(1.f, mul_x(fy, 2.f));
    float sx = mul_x(mul_x(nx, P.tanHalfFov), P.aspect);
    float sy = mul_x(ny, P.tanHalfFov);
    f3 d = v3(add_x(add_x(P.camFwd.x, mul_x(P.camRight.x, sx)), mul_x(P.camUp.x, sy)),
              add_x(add_x(P.camFwd.y, mul_x(P.camRight.y, sx)), mul_x(P.camUp.y, sy)),
              add_x(add_x(P.camFwd.z, mul_x(P.camRight.z, sx)), mul_x(P.camUp.z, sy)));
    return normalize_x(d);
}

BH_DEV float capture_radius(const TraceParams& P)
{
    return (P.rPlus > 1e-6f) ? P.rPlus : 0.05f * P.M;
}

// sin/cos of the polar angle.  FP32: the MUFU pair (absolute error ~4e-7),
// replaced by the polynomial sincos_polar when |sin| < 1/16, so that sin keeps
// its relative accuracy near the poles where the equations divide by it.
// FP64: the library sincos.
BH_DEV void sincos_theta(float x, float& s, float& c)
{
    __sincosf(x, &s, &c);
    if (fabsf(s) < 0.0625f) sincos_polar(x, s, c);
}
BH_DEV void sincos_theta(double x, double& s, double& c) { sincos_cap(x, s, c); }

// RK4 stage angles: the same pole-accurate pair.  (A plain MUFU sine has only
// absolute accuracy, ~4e-7: near the poles the 1/sin^2 terms of the stages then
// carry ~1e-5 relative error, enough to move escape directions by ~1e-4 rad
// for cameras within a few degrees of the spin axis.)
BH_DEV void sincos_stage(float x, float& s, float& c) { sincos_theta(x, s, c); }
BH_DEV void sincos_stage(double x, double& s, double& c) { sincos_cap(x, s, c); }

// Cubic Hermite interpolant on a step: value at fraction t of the step of
// length h, from end values y0, y1 and derivatives d0, d1 (per unit parameter).
template <class T>
BH_DEV T hermite(T y0, T y1, T d0, T d1, T h, T t)
{
    T t2 = t * t, t3 = t2 * t;
    return (T(2) * t3 - T(3) * t2 + T(1)) * y0 + (t3 - T(2) * t2 + t) * h * d0 + (T(3) * t2 - T(2) * t3) * y1 +
           (t3 - t2) * h * d1;
}

// Root of the Hermite interpolant of f (f0, f1 of opposite sign) by bisection:
// the equatorial crossing of a step, located to the working precision.
template <class T>
BH_DEV T bisect_hermite(T f0, T f1, T d0, T d1, T h)
{
    T lo = T(0), hi = T(1);
    const int iters = sizeof(T) == 8 ? 52 : 24;
    for (int i = 0; i < iters; ++i)
    {
        T mid = T(0.5) * (lo + hi);
        T fm = hermite(f0, f1, d0, d1, h, mid);
        if ((fm < T(0)) == (f0 < T(0))) lo = mid; else hi = mid;
    }
    return T(0.5) * (lo + hi);
}

// First equatorial crossing of the ray inside the disk annulus: the
// "disk-hit" radius and the emitter redshift there, recorded for ray
// statistics (probe records, surrogate training targets).
BH_DEV void record_disk_hit(const TraceParams& P, DiskTally& tally, float rHit, float E, float Lz)
{
    if (tally.hitR > 0.f || !(rHit >= P.diskInner && rHit <= P.diskOuter)) return;
    float om = omega_circ(rHit, P.M, P.a, P.Q);
    tally.hitR = rHit;
    tally.hitG = (om > 0.f) ? emitter_g(rHit, om, P.M, P.a, P.Q, E, Lz) : 0.f;
}

// ===========================================================================
// Spherically symmetric metrics (Schwarzschild, Reissner-Nordstrom)
// ===========================================================================
// One RK4 step of the Binet equation in FP64 from a lower-precision state.
template <class R>
BH_DEV void binet_rk4_fp64(R& u, R& du, R h, const CamFrame<double>& F)
{
    double U = (double)u, V = (double)du, H = (double)h;
    const double m3 = 3.0 * F.M, q2 = 2.0 * F.Q2;
    auto acc = [&](double x) { return (m3 * x - q2 * x * x) * x - x; };
    const double hh = 0.5 * H;
    double k1 = acc(U);
    double u2 = U + hh * V, v2 = V + hh * k1, k2 = acc(u2);
    double u3 = U + hh * v2, v3 = V + hh * k2, k3 = acc(u3);
    double u4 = U + H * v3, v4 = V + H * k3, k4 = acc(u4);
    const double h6 = H / 6.0;
    U += h6 * (V + 2.0 * v2 + 2.0 * v3 + v4);
    V += h6 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
    u = (R)U;
    du = (R)V;
}

// Camera-frame initial data of a spherical-family ray, in precision T.
template <class T>
struct SphInit
{
    T E, Lz, e2x, e2y, e2z, invB, u, du;
    bool radial, inward;
};

template <class T>
BH_DEV SphInit<T> sph_init(const TraceParams& P, const CamFrame<T>& F, vec3<T> dir)
{
    SphInit<T> o;
    // photon E, Lz (reference src/trace.cuh:213-247 with a = 0)
    o.E = T(1); o.Lz = T(0);
    if (!F.camAtOrigin)
    {
        T dpc = xdot(F.ephS, dir);
        T ptUp = xsub(F.rsqS, xdiv(xmul(xmul(dpc, F.AS), F.gtpS), F.gttS));
        T pfUp = xmul(dpc, F.AS);
        o.E = -xadd(xmul(F.gttS, ptUp), xmul(F.gtpS, pfUp));
        o.Lz = xadd(xmul(F.gtpS, ptUp), xmul(F.gppS, pfUp));
        if (!(o.E > T(1e-6f)) || !finite_p(o.E)) { o.E = T(1); o.Lz = T(0); }
    }
    // orbital plane (reference src/trace.cuh:490-521)
    T ddr = xdot(F.e1, dir);
    T px = xsub(dir.x, xmul(F.e1[0], ddr));
    T py = xsub(dir.y, xmul(F.e1[1], ddr));
    T pz = xsub(dir.z, xmul(F.e1[2], ddr));
    T pl = xsqrt(xadd(xadd(xmul(px, px), xmul(py, py)), xmul(pz, pz)));
    o.radial = pl < T(1e-6f);
    if (o.radial)
    {   // exactly radial ray (reference src/trace.cuh:447-459, 500-505)
        const vec3<T> c = widen<T>(tof3(P.camPos));
        o.inward = xadd(xadd(xmul(dir.x, c.x), xmul(dir.y, c.y)), xmul(dir.z, c.z)) < T(0);
        return o;
    }
    o.inward = false;
    T ipl = xdiv(T(1), pl);
    o.e2x = xmul(px, ipl); o.e2y = xmul(py, ipl); o.e2z = xmul(pz, ipl);
    T bImpact = max_p(xdiv(xmul(F.r0, pl), F.sf0), T(1e-6f));
    o.invB = T(1) / bImpact;
    o.u = F.u0;
    o.du = xdiv(xmul(-F.sf0, ddr), xmul(F.r0, pl));
    return o;
}

// MIXED: FP32 state and steps; FP64 initial data, whole steps in FP64 where
// the Binet solution turns (u' would change sign within the step), and FP64
// location of the equatorial crossing.
template <class R, bool STATS, bool MIXED = false>
struct SphRay
{
    using Real = R;
    static constexpr bool kKerrFamily = false;
    R u, du, phi, tFlight, invB;
    R e2x, e2y, e2z;                  // in-plane unit vector normal to e1 (e1 is the camera's)
    R ud, dud, phid;                  // state of the last chord direction (deferred)
    float E, Lz;                      // photon constants for the disk emitter
    f3 prevPos, accum;
    float trans;
    int step;
    bool horizon, escaped, haveDir;
    DiskTally tally;
    double I0;

    BH_DEV int init(const TraceParams& P, f3 dirf)
    {
        horizon = escaped = haveDir = false;
        accum = v3(0.f, 0.f, 0.f);
        trans = 1.f;
        step = 0;
        tFlight = R(0);
        prevPos = tof3(P.camPos);
        if (STATS) { tally.samples = 0; tally.hitR = 0.f; tally.hitG = 0.f; I0 = 0.0; }
        bool radial, inward;
        if constexpr (MIXED)
        {
            SphInit<double> v = sph_init<double>(P, P.cd, widen<double>(dirf));
            radial = v.radial; inward = v.inward;
            E = (float)v.E; Lz = (float)v.Lz;
            e2x = (R)v.e2x; e2y = (R)v.e2y; e2z = (R)v.e2z; invB = (R)v.invB; u = (R)v.u; du = (R)v.du;
        }
        else
        {
            SphInit<R> v = sph_init<R>(P, frame_of<R>(P), widen<R>(dirf));
            radial = v.radial; inward = v.inward;
            E = (float)v.E; Lz = (float)v.Lz;
            e2x = v.e2x; e2y = v.e2y; e2z = v.e2z; invB = v.invB; u = v.u; du = v.du;
        }
        if (radial)
        {
            horizon = inward;
            escaped = !horizon;
            return RAY_DONE;
        }
        phi = R(0);
        if (STATS) I0 = binet((R)P.M, (R)P.Q * (R)P.Q, u, du);
        return RAY_LIVE;
    }

    BH_DEV static double binet(R M, R Q2, R uu, R vv)
    {   // first integral du^2 + u^2 (1 - 2Mu + Q^2 u^2) = 1/b^2
        double U = (double)uu, V = (double)vv;
        return V * V + U * U * (1.0 - 2.0 * (double)M * U + (double)Q2 * U * U);
    }

    // One reference loop iteration (src/trace.cuh:546-600).  Returns true when
    // the ray has terminated.
    BH_DEV bool advance(const TraceParams& P)
    {
        const CamFrame<R>& F = frame_of<R>(P);
        if (step >= P.maxSteps) { exhaust(P); return true; }
        const R M = F.M, Q2 = F.Q2, dPhi = F.dPhi;

        R hMax = dPhi * min_p(max_p(F.invNineM * rcp_p(u), R(1)), R(6));
        R h = min_p(hMax, R(0.10f) * rcp_p(max_p(abs_p(du), R(1e-6f))));
        h = max_p(h, F.hMin);

        const R u0 = u, du0 = du;
        const R m3 = R(3) * M, q2 = R(2) * Q2;
        auto acc = [&](R x) { return (m3 * x - q2 * x * x) * x - x; };
        const R k1v = acc(u);
        if (MIXED && abs_p(du) < h * abs_p(k1v))
            binet_rk4_fp64(u, du, h, P.cd);      // radial turning point
        else
        {
            R hh = R(0.5f) * h;
            R u2 = u + hh * du, v2 = du + hh * k1v;
            R k2v = acc(u2);
            R u3 = u + hh * v2, v3_ = du + hh * k2v;
            R k3v = acc(u3);
            R u4 = u + h * v3_, v4 = du + h * k3v;
            R k4v = acc(u4);
            R h6 = h * R(1.0 / 6.0);
            u += h6 * (du + R(2) * v2 + R(2) * v3_ + v4);
            du += h6 * (k1v + R(2) * k2v + R(2) * k3v + k4v);
        }
        phi += h;

        if (!finite_p(u + du)) { horizon = true; return true; }   // either non-finite (u, du stay far below the float range)
        if (u >= F.uHor) { horizon = true; return true; }
        if (u < R(1e-4f)) { escaped = true; return true; }   // previous chord direction

        R r = rcp_p(u);
        ud = u; dud = du; phid = phi; haveDir = true;
        R fR = max_p(R(1) - R(2) * M * u + Q2 * u * u, R(1e-4f));
        tFlight += h * r * r * invB * rcp_p(fR);
        if (STATS) equator_crossing(P, u0, du0, k1v, h);

        if (P.diskOn && trans > 0.01f)
        {
            R sp, cp;
            sincos_fast(phi, sp, cp);
            f3 pos = v3((float)((F.e1[0] * cp + e2x * sp) * r), (float)((F.e1[1] * cp + e2y * sp) * r),
                        (float)((F.e1[2] * cp + e2z * sp) * r));
            disk_segment<STATS>(P, E, Lz, prevPos, pos, (float)(F.diskTime - tFlight), accum, trans, tally);
            prevPos = pos;
        }
        ++step;
        if (u < F.uEscape && du < R(0)) { escaped = true; return true; }
        return false;
    }

    // Equatorial crossing inside the step (phi - h, phi]: the orbital plane meets
    // y = 0 at phi* = atan2(-e1y, e2y) + k pi; u(phi*) from the cubic Hermite
    // interpolant of the step (FP64 in MIXED and FP64 modes).
    BH_DEV void equator_crossing(const TraceParams& P, R u0, R du0, R ddu0, R h)
    {
        using T = typename std::conditional<MIXED, double, R>::type;
        const CamFrame<T>& F = frame_of<T>(P);
        const T e1y = F.e1[1], e2 = (T)e2y;
        if (abs_p(e1y) + abs_p(e2) < T(1e-12)) return;   // orbit in the equatorial plane
        const T pc = atan2(-e1y, e2), pi = T(3.14159265358979323846);
        const T p0 = (T)phi - (T)h;
        T k = ceil((p0 - pc) / pi);
        T ps = pc + k * pi;
        if (ps <= p0) ps += pi;
        if (ps > (T)phi) return;
        const T uh = hermite((T)u0, (T)u, (T)du0, (T)du, (T)h, (ps - p0) / (T)h);
        (void)ddu0;
        if (uh > T(0)) record_disk_hit(P, tally, (float)(T(1) / uh), E, Lz);
    }

    BH_DEV void exhaust(const TraceParams& P)
    {   // budget spent: reference src/trace.cuh:603-609
        if (u > frame_of<R>(P).uPh) horizon = true;
        else escaped = true;
    }

    BH_DEV void pack(const TraceParams& P, unsigned key, PackedRay<R>& q, PackedStats* st) const
    {
        const bool useState = escaped && haveDir;
        q.key = key | (horizon ? kRayHorizon : 0u) | (escaped ? kRayEscaped : 0u) | (useState ? kRayUseState : 0u) |
                (step >= P.maxSteps ? kRayExhausted : 0u);
        q.acc[0] = accum.x; q.acc[1] = accum.y; q.acc[2] = accum.z;
        q.trans = trans;
        q.f[0] = ud; q.f[1] = dud; q.f[2] = phid; q.f[3] = e2x; q.f[4] = e2y; q.f[5] = e2z;
        if (STATS)
        {
            st->steps = step; st->samples = tally.samples; st->maxHviol = 0.f;
            st->hitR = tally.hitR; st->hitG = tally.hitG;
            double I1 = (step > 0) ? binet((R)P.M, (R)P.Q * (R)P.Q, u, du) : I0;
            st->drift = (I0 > 0.0) ? (float)(fabs(I1 - I0) / I0) : 0.f;
        }
    }

    // Escape direction: the chord direction of the last step (reference
    // src/trace.cuh:581-587), rebuilt with accurate trigonometry.
    BH_DEV static f3 escape_dir(const TraceParams& P, const PackedRay<R>& q)
    {
        const CamFrame<R>& F = frame_of<R>(P);
        const R ud_ = q.f[0], dud_ = q.f[1], phid_ = q.f[2], ex = q.f[3], ey = q.f[4], ez = q.f[5];
        R sp, cp;
        sincos(phid_, &sp, &cp);
        R r = R(1) / ud_;
        R drdphi = -dud_ / (ud_ * ud_);
        R mx = F.e1[0] * cp + ex * sp, my = F.e1[1] * cp + ey * sp, mz = F.e1[2] * cp + ez * sp;
        R qx = -F.e1[0] * sp + ex * cp, qy = -F.e1[1] * sp + ey * cp, qz = -F.e1[2] * sp + ez * cp;
        return normalize_x(v3((float)(mx * drdphi + qx * r), (float)(my * drdphi + qy * r),
                              (float)(mz * drdphi + qz * r)));
    }
};

// ===========================================================================
// Rotating metrics (Kerr, Kerr-Newman): Boyer-Lindquist Hamiltonian system
// ===========================================================================
template <class R>
struct KerrDeriv { R r, th, ph, pr, pth; };

// Right-hand side of the first-order system plus the constraint K = 2 Sigma H
// (reference src/trace.cuh:620-659).  s, c: sin/cos of th (s unclamped).
// Also returns the pieces the slow-light term at the same point reuses.
template <class R>
struct KerrEval
{
    KerrDeriv<R> d;
    R K, Pp, iDelT, iS;   // iDelT: 1 / max(Delta, 1e-5), the slow-light clamp
};

// Per-ray constants of the right-hand side: products of E, Lz, a that the
// reference recomputes at every evaluation.
template <class R>
struct KerrConsts
{
    R E, Lz, aE, c1, twoE;    // c1 = E a^2 - a Lz, so P = E r^2 + c1
};

// per lane: x >= thr ? a : b
BH_DEV float  vsel_ge(float x, float thr, float a, float b)    { return x >= thr ? a : b; }
BH_DEV double vsel_ge(double x, double thr, double a, double b) { return x >= thr ? a : b; }
BH_DEV float2 vsel_ge(float2 x, float2 thr, float2 a, float2 b)
{
    return make_float2(x.x >= thr.x ? a.x : b.x, x.y >= thr.y ? a.y : b.y);
}
BH_DEV void vsincos_stage(float x, float& s, float& c)    { sincos_stage(x, s, c); }
BH_DEV void vsincos_stage(double x, double& s, double& c) { sincos_stage(x, s, c); }
BH_DEV void vsincos_stage(float2 x, float2& s, float2& c)
{
    sincos_stage(x.x, s.x, c.x);
    sincos_stage(x.y, s.y, c.y);
}

// Two updates a * x_i + y_i of one lane type with a shared coefficient: for a
// single FP32 ray the pair is one packed FMA, otherwise two lane FMAs (the
// same rounding either way).
BH_DEV void vfma_pair(float a, float x0, float x1, float y0, float y1, float& o0, float& o1)
{
    fma2_p(a, x0, x1, y0, y1, o0, o1);
}
template <class V> BH_DEV void vfma_pair(V a, V x0, V x1, V y0, V y1, V& o0, V& o1)
{
    o0 = vfma(a, x0, y0);
    o1 = vfma(a, x1, y1);
}

// V = float or double (one ray), float2 (two FP32 rays packed); S = the frame's
// scalar type.  Every operation explicit, so one ray and a packed pair give the
// same bits.  SCALED = false: the five derivatives without their common factor
// 1 / Sigma (returned in iS), for RK4 stages that fold it into the stage's
// coefficients.
template <class V, class S, bool SCALED = true>
BH_DEV KerrEval<V> kerr_rhs(const CamFrame<S>& F, const KerrConsts<V>& k, V r, V s, V c, V pr, V pth)
{
    const V M = lane<V>(F.M), a2 = lane<V>(F.a2);
    s = vmax(s, lane<V>((S)1e-4f));                                        // pole guard
    const V r2 = vmul(r, r);
    const V Sig = vfma(vmul(a2, c), c, r2);                                // r^2 + a^2 cos^2
    const V rm2M = vfma(lane<V>((S)-2.f), M, r);                           // r - 2M
    const V DelRaw = vfma(r, rm2M, lane<V>(F.a2Q2));                       // r (r - 2M) + a^2 + Q^2
    const V Del = vmax(DelRaw, lane<V>((S)1e-6f));
    const V Pp = vfma(k.E, r2, k.c1);                                      // E (r^2 + a^2) - a Lz
    const V is = vrcp(s), iS = vrcp(Sig), iDel = vrcp(Del);
    const V is2 = vmul(is, is);
    const V B = vfma(vneg(k.aE), s, vmul(k.Lz, is));                       // Lz / s - a E s
    const V PiD = vmul(Pp, iDel);
    const V W = vfma(B, B, vneg(vmul(PiD, Pp)));                           // B^2 - P^2 / Delta
    const V Dpr = vmul(Del, pr);
    KerrEval<V> o;
    o.K = vfma(Dpr, pr, vfma(pth, pth, W));                                // Delta pr^2 + pth^2 + W
    const V rmM = vsub(r, M);                                              // dDelta/dr / 2
    const V Wrh = vmul(PiD, vfma(PiD, rmM, vneg(vmul(k.twoE, r))));        // dW/dr / 2 = -P/D (dP - P/D dDelta) / 2
    const V KiS = vmul(o.K, iS);
    const V uph = vfma(lane<V>(F.a), PiD, vfma(k.Lz, is2, vneg(k.aE)));
    // dpr = -(dH/dr) = (r K / Sigma - (dDelta pr^2 + dW/dr) / 2) / Sigma
    const V upr = vfma(vneg(vmul(rmM, pr)), pr, vfma(r, KiS, vneg(Wrh)));
    // dpth = -(dH/dth) = cos (B (Lz / s^2 + a E) - a^2 s K / Sigma) / Sigma
    const V upth = vfma(B, vfma(k.Lz, is2, k.aE), vneg(vmul(vmul(a2, s), KiS)));
    if constexpr (SCALED)
    {
        o.d.r = vmul(Dpr, iS);
        o.d.th = vmul(pth, iS);
        o.d.ph = vmul(uph, iS);
        o.d.pr = vmul(iS, upr);
        o.d.pth = vmul(vmul(c, iS), upth);
    }
    else
    {
        o.d.r = Dpr;
        o.d.th = pth;
        o.d.ph = uph;
        o.d.pr = upr;
        o.d.pth = vmul(c, upth);
    }
    o.Pp = Pp;
    o.iDelT = vsel_ge(DelRaw, lane<V>((S)1e-5f), iDel, lane<V>((S)1e5f));
    o.iS = iS;
    return o;
}

// The classic RK4 step of the Kerr-Newman system from the state (r, th, ph,
// pr, pth) with step h and first right-hand side d1; d4 receives the final
// stage's derivative without its factor 1 / Sigma, iS4 that factor.
// (reference src/trace.cuh:811-838)  Stages 2-4 evaluate the right-hand side
// unscaled and fold 1 / Sigma into the stage's coefficients (2 / Sigma for the
// weighted sum, h / (2 Sigma) or h / Sigma for the next stage point), which
// saves the five products by 1 / Sigma per stage.
template <class V, class S>
BH_DEV void kerr_rk4(const CamFrame<S>& F, const KerrConsts<V>& k, V h, V& r, V& th, V& ph, V& pr, V& pth,
                     const KerrDeriv<V>& d1, KerrDeriv<V>& d4, V& iS4)
{
    const V hh = vmul(lane<V>((S)0.5f), h), two = lane<V>((S)2.f);
    V sx, cx, yr, yth, ypr, ypth;
    vfma_pair(hh, d1.r, d1.th, r, th, yr, yth);
    vfma_pair(hh, d1.pr, d1.pth, pr, pth, ypr, ypth);
    vsincos_stage(yth, sx, cx);
    KerrEval<V> e = kerr_rhs<V, S, false>(F, k, yr, sx, cx, ypr, ypth);      // stage 2
    V w = vmul(two, e.iS), a = vmul(hh, e.iS);
    V sr, sth, spr, spth, sph = vfma(w, e.d.ph, d1.ph);
    vfma_pair(w, e.d.r, e.d.th, d1.r, d1.th, sr, sth);
    vfma_pair(w, e.d.pr, e.d.pth, d1.pr, d1.pth, spr, spth);
    vfma_pair(a, e.d.r, e.d.th, r, th, yr, yth);
    vfma_pair(a, e.d.pr, e.d.pth, pr, pth, ypr, ypth);
    vsincos_stage(yth, sx, cx);
    e = kerr_rhs<V, S, false>(F, k, yr, sx, cx, ypr, ypth);                  // stage 3
    w = vmul(two, e.iS);
    a = vmul(h, e.iS);
    vfma_pair(w, e.d.r, e.d.th, sr, sth, sr, sth);
    vfma_pair(w, e.d.pr, e.d.pth, spr, spth, spr, spth);
    sph = vfma(w, e.d.ph, sph);
    vfma_pair(a, e.d.r, e.d.th, r, th, yr, yth);
    vfma_pair(a, e.d.pr, e.d.pth, pr, pth, ypr, ypth);
    vsincos_stage(yth, sx, cx);
    e = kerr_rhs<V, S, false>(F, k, yr, sx, cx, ypr, ypth);                  // stage 4
    d4 = e.d;
    iS4 = e.iS;
    const V h6 = vmul(h, lane<V>((S)(1.0 / 6.0)));
    V t0, t1, t2, t3;
    vfma_pair(iS4, d4.r, d4.th, sr, sth, t0, t1);
    vfma_pair(iS4, d4.pr, d4.pth, spr, spth, t2, t3);
    vfma_pair(h6, t0, t1, r, th, r, th);
    vfma_pair(h6, t2, t3, pr, pth, pr, pth);
    ph = vfma(h6, vfma(iS4, d4.ph, sph), ph);
}

// MIXED: FP32 state and steps; FP64 initial data (tetrad map and camera
// position), FP64 state and steps through every polar passage (|sin th| <
// kPolarCap, below), and FP64 bisection of the equatorial crossing.  (Not
// taken, measured on the near-extremal 4K sweep against the all-FP64
// integration: FP64 steps over the whole final horizon approach, 70 % more
// time for no accuracy gain; FP64 steps at radial turning points, where p_r
// would change sign within the step, 23 % more time for the same accuracy to
// five digits at every elevation.)
//
// Polar passages.  A ray that passes within a small angle th_min of the spin
// axis swings its azimuth by ~pi and reverses p_th within a few steps, and the
// step's outcome depends on th relative to th_min: a rounding error e in an
// FP32 state th becomes a relative error e / th_min of the passage (at
// th_min ~ 3e-4, an FP32 rounding of ~1e-9 changes p_th after the passage by
// ~1e-3 relative, and the escape direction by ~1e-4 rad).  FP64 arithmetic
// inside each step does not help while the state is rounded back to FP32
// between steps; what does is to carry an FP64 state from the step that enters
// the cap |sin th| < kPolarCap to the step that leaves it, so that is what
// MIXED does (polar_passage_fp64).
template <class R, bool STATS, bool MIXED = false>
struct KerrRay
{
    using Real = R;
    static constexpr bool kKerrFamily = true;
    R r, th, ph, pr, pth;   // Boyer-Lindquist state
    R s, c;                 // sin/cos of th
    KerrConsts<R> k;        // E, Lz and their products
    R tFlight;
    KerrDeriv<R> d1;        // right-hand side at the current state
    R K1;
    f3 prevPos, accum;
    float trans, maxHviol;
    int step;
    bool horizon, escaped, useDeriv;
    bool prevCart;          // prevPos holds (x, y, z); else (r sin th, y, ph) of the last point
    DiskTally tally;
    double Q0;

    // the reference's dLast (derivative of the final RK4 stage), kept only on
    // the last step the budget allows: it is needed only if that budget runs out
    BH_DEV static R* last_deriv()
    {
        __shared__ R dl[BH_TRACE_BLOCK_MAX][3];
        return dl[threadIdx.x];
    }

    BH_DEV int init(const TraceParams& P, f3 dirf)
    {   // reference src/trace.cuh:703-739: the per-ray remainder of the tetrad map
        const CamFrame<R>& F = frame_of<R>(P);
        R E, Lz;
        if constexpr (MIXED)
        {   // FP64 tetrad map, each result rounded once
            const CamFrame<double>& D = P.cd;
            const vec3<double> dir = widen<double>(dirf);
            double drc = xdot(D.er, dir), dtc = xdot(D.eth, dir), dpc = xdot(D.eph, dir);
            double ptUp = xsub(D.rsq, xdiv(xmul(xmul(dpc, D.A), D.gtp), D.gtt));
            double pfUp = xmul(dpc, D.A);
            E = (R)(-xadd(xmul(D.gtt, ptUp), xmul(D.gtp, pfUp)));
            Lz = (R)xadd(xmul(D.gtp, ptUp), xmul(D.gpp, pfUp));
            pr = (R)xmul(drc, D.sqSD);
            pth = (R)xmul(dtc, D.sqS);
            // the position too: near the poles acos(y / r) is ill-conditioned and
            // the FP32 camera angle is off by up to ~1e-5 rad
            r = (R)D.r0; th = (R)D.th0; ph = (R)D.ph0;
        }
        else
        {
            const vec3<R> dir = widen<R>(dirf);
            R drc = xdot(F.er, dir), dtc = xdot(F.eth, dir), dpc = xdot(F.eph, dir);
            R ptUp = xsub(F.rsq, xdiv(xmul(xmul(dpc, F.A), F.gtp), F.gtt));
            R pfUp = xmul(dpc, F.A);
            E = -xadd(xmul(F.gtt, ptUp), xmul(F.gtp, pfUp));
            Lz = xadd(xmul(F.gtp, ptUp), xmul(F.gpp, pfUp));
            pr = xmul(drc, F.sqSD);
            pth = xmul(dtc, F.sqS);
            r = F.r0; th = F.th0; ph = F.ph0;
        }
        k.E = E; k.Lz = Lz; k.aE = F.a * E; k.c1 = E * F.a2 - F.a * Lz; k.twoE = R(2) * E;
        sincos_theta(th, s, c);
        KerrEval<R> ev = kerr_rhs(F, k, r, s, c, pr, pth);
        d1 = ev.d;
        K1 = ev.K;

        tFlight = R(0);
        prevPos = tof3(P.camPos);
        prevCart = true;
        accum = v3(0.f, 0.f, 0.f);
        trans = 1.f;
        maxHviol = 0.f;
        step = 0;
        horizon = escaped = useDeriv = false;
        if (STATS)
        {
            tally.samples = 0; tally.hitR = 0.f; tally.hitG = 0.f;
            Q0 = carterQ(th, pth, F.a, E, Lz);
        }
        return RAY_LIVE;
    }

    // Carter constant p_th^2 + cos^2 th (Lz^2 / sin^2 th - a^2 E^2), in double.
    BH_DEV static double carterQ(R th_, R pth_, R a, R E_, R Lz_)
    {
        double sd, cd;
        sincos((double)th_, &sd, &cd);
        double s2 = fmax(sd * sd, 1e-12);
        return (double)pth_ * pth_ + cd * cd * ((double)Lz_ * Lz_ / s2 - (double)a * a * (double)E_ * E_);
    }

    // One reference loop iteration (src/trace.cuh:752-868).  The first
    // right-hand side of the step (d1) was evaluated at the end of the previous
    // iteration, where its Sigma, Delta and P also gave the slow-light term.
    // Returns true when the ray has terminated.
    BH_DEV bool advance(const TraceParams& P)
    {
        const CamFrame<R>& F = frame_of<R>(P);
        if (step >= P.maxSteps) { exhaust(P); return true; }
        // the reference's five finiteness tests (trace.cuh:757-760) as one: a NaN or
        // infinity in any of them makes the sum non-finite (finite values of these
        // quantities stay far below the float range)
        if (!finite_p(((r + pr) + (pth + d1.r)) + d1.pr))
        { horizon = true; return true; }
        if (r <= F.capR) { horizon = true; return true; }
        if (STATS && r > F.rFloor105)
        {
            float viol = (float)(abs_p(K1) / (k.E * k.E * (r * r + F.a2) + R(1e-12f)));
            maxHviol = fmaxf(maxHviol, viol);
        }
        if (r >= F.escR && d1.r > R(0)) { escaped = useDeriv = true; return true; }

        // adaptive affine step (reference src/trace.cuh:793-809)
        const R ang = abs_p(d1.th) + abs_p(d1.ph);
        // h = 1 / (|dr| / kq + ang / (2.2 dPhi) + 1e-5) with kq = 8 dPhi max(r - rFloor, 0.02),
        // formed as one quotient kq / (kq (ang / (2.2 dPhi) + 1e-5) + |dr|)
        const R kq = F.k8dPhi * max_p(r - F.rFloor, R(0.02f));
        R h = kq * rcp_p(kq * (ang * F.i22dPhi + R(1e-5f)) + abs_p(d1.r));
        if (r < F.rPh15) h *= R(0.55f);
        R spd = abs_p(d1.r) + r * ang + R(1e-6f);
        R capLen;
        if (P.diskOn && r < F.outer13)
            capLen = (r * abs_p(c) < R(1.8f)) ? R(1.2f) : R(2.2f);
        else
            capLen = max_p(R(1.2f), R(0.22f) * r);
        h = min_p(h, capLen * rcp_p(spd));

        const R rS = r, thS = th, drS = d1.r, dthS = d1.th;    // step start (crossing search)
        if constexpr (MIXED)
        {
            if (abs_p(s) < R(kPolarCap)) return polar_passage_fp64(P);
        }

        KerrDeriv<R> d4;
        R iS4;
        kerr_rk4(F, k, h, r, th, ph, pr, pth, d1, d4, iS4);
        return finish_step(P, F, h, rS, thS, drS, dthS, d4.r, d4.th, d4.ph, iS4);
    }

    BH_DEV bool polar_passage_fp64(const TraceParams& P);

    // Rest of a loop iteration after the RK4 update: pole guard, the next
    // step's first right-hand side with the slow-light term, disk chord.
    BH_DEV bool finish_step(const TraceParams& P, const CamFrame<R>& F, R h, R rS, R thS, R drS, R dthS,
                            R d4r, R d4th, R d4ph, R d4iS)
    {
        // pole reflection guard
        if (th < R(1e-3f)) { th = R(1e-3f); pth = abs_p(pth); }
        else if (th > R(kPiF - 1e-3f)) { th = R(kPiF - 1e-3f); pth = -abs_p(pth); }
        ++step;
        if (step == P.maxSteps)
        {
            R* dl = last_deriv();      // the final stage's derivative, scaled by 1 / Sigma
            dl[0] = d4r * d4iS; dl[1] = d4th * d4iS; dl[2] = d4ph * d4iS;
        }

        // next step's first right-hand side; its Sigma, Delta, P give the slow
        // light  Sigma dt/dl = a (Lz - a E sin^2) + (r^2 + a^2) P / Delta
        sincos_theta(th, s, c);
        KerrEval<R> ev = kerr_rhs(F, k, r, s, c, pr, pth);
        d1 = ev.d;
        K1 = ev.K;
        {
            const R sc = max_p(s, R(1e-4f));
            const R dtdl = (F.a * (k.Lz - k.aE * sc * sc) + (r * r + F.a2) * ev.Pp * ev.iDelT) * ev.iS;
            tFlight += h * abs_p(dtdl);
        }
        if (STATS) equator_crossing(P, h, rS, thS, drS, dthS);
        if (P.diskOn) disk_chord(P, F);
        return false;
    }

    // Cartesian point (kerrToCart, reference src/trace.cuh:665-671) from r sin th,
    // r cos th and the azimuth.  The point feeds the float disk shading, so an
    // FP64 ray forms it in float as well (the FP64 azimuth rounded once): a
    // general double sincos per step would dominate the FP64 step.
    BH_DEV static f3 cart(R rs, float y, R phi)
    {
        float sp, cp, px, pz;
        sincos_fast((float)phi, sp, cp);
        mul2_p((float)rs, -(float)rs, cp, sp, px, pz);
        return v3(px, y, pz);
    }

    // The disk chord from the previous point to the current one (reference
    // src/trace.cuh:853-866).  The chord's first test in disk_segment is the
    // vertical slab cull on the two end heights; most steps of most rays are
    // culled there, so for FP32 rays the azimuthal part of the Cartesian
    // point (a sincos and two products) is formed only when a chord can
    // reach the slab: a culled point keeps (r sin th, y, ph) and becomes
    // Cartesian only if the next chord needs it.  The values, and so the
    // chord, are the same bits as forming every point.
    BH_DEV void disk_chord(const TraceParams& P, const CamFrame<R>& F)
    {
        const R rs = r * s;
        const float y = (float)(r * c);
        if constexpr (std::is_same<R, float>::value)
        {
            const float maxH = 0.16f * P.diskOuter;
            if ((prevPos.y > maxH && y > maxH) || (prevPos.y < -maxH && y < -maxH))
            {   // culled: keep the point in polar form
                prevPos = v3((float)rs, y, (float)ph);
                prevCart = false;
                return;
            }
            if (!prevCart) prevPos = cart((R)prevPos.x, prevPos.y, (R)prevPos.z);
        }
        const f3 pos = cart(rs, y, ph);
        if (trans > 0.01f)
            disk_segment<STATS>(P, (float)k.E, (float)k.Lz, prevPos, pos, (float)(F.diskTime - tFlight), accum,
                                trans, tally);
        prevPos = pos;
        prevCart = true;
    }

    // Equatorial crossing inside the last step: bisection of the cubic Hermite
    // interpolant of theta over the step (FP64 in MIXED and FP64 modes), r there.
    BH_DEV void equator_crossing(const TraceParams& P, R h, R rS, R thS, R drS, R dthS)
    {
        using T = typename std::conditional<MIXED, double, R>::type;
        const T half = T(1.57079632679489661923);
        const T f0 = (T)thS - half, f1 = (T)th - half;
        if (!((f0 < T(0)) != (f1 < T(0)))) return;
        const T t = bisect_hermite(f0, f1, (T)dthS, (T)d1.th, (T)h);
        const T rh = hermite((T)rS, (T)r, (T)drS, (T)d1.r, (T)h, t);
        record_disk_hit(P, tally, (float)rh, (float)k.E, (float)k.Lz);
    }

    BH_DEV void exhaust(const TraceParams& P)
    {   // budget spent: reference src/trace.cuh:871-888
        if (r < frame_of<R>(P).sixM) horizon = true;
        else { escaped = true; useDeriv = step > 0; }
    }

    BH_DEV void pack(const TraceParams& P, unsigned key, PackedRay<R>& q, PackedStats* st) const
    {
        const bool useState = escaped && useDeriv;
        q.key = key | (horizon ? kRayHorizon : 0u) | (escaped ? kRayEscaped : 0u) | (useState ? kRayUseState : 0u) |
                (step >= P.maxSteps ? kRayExhausted : 0u);
        q.acc[0] = accum.x; q.acc[1] = accum.y; q.acc[2] = accum.z;
        q.trans = trans;
        q.f[0] = r; q.f[1] = th; q.f[2] = ph;
        if (useState && step >= P.maxSteps)
        {   // budget exhausted: the derivative of the last RK4 stage
            const R* dl = last_deriv();
            q.f[3] = dl[0]; q.f[4] = dl[1]; q.f[5] = dl[2];
        }
        else { q.f[3] = d1.r; q.f[4] = d1.th; q.f[5] = d1.ph; }
        if (STATS)
        {
            st->steps = step; st->samples = tally.samples; st->maxHviol = maxHviol;
            st->hitR = tally.hitR; st->hitG = tally.hitG;
            const R a = (R)P.a;
            double q1 = carterQ(th, pth, a, k.E, k.Lz);
            double scale = fabs(Q0) + (double)k.Lz * k.Lz + (double)a * a * (double)k.E * k.E;
            st->drift = scale > 0.0 ? (float)(fabs(q1 - Q0) / scale) : 0.f;
        }
    }

    // Escape direction: kerrBasis(th, ph) applied to the coordinate derivative
    // (reference src/trace.cuh:775-779, 880-884), accurate trigonometry.
    BH_DEV static f3 escape_dir(const TraceParams&, const PackedRay<R>& q)
    {
        const R r_ = q.f[0], th_ = q.f[1], ph_ = q.f[2];
        R sth, cth, sph, cph;
        sincos(th_, &sth, &cth);
        sincos(ph_, &sph, &cph);
        R vr = q.f[3], vt = r_ * q.f[4], vp = r_ * sth * q.f[5];
        return normalize_x(v3((float)(sth * cph * vr + cth * cph * vt - sph * vp),
                              (float)(cth * vr - sth * vt),
                              (float)(-sth * sph * vr - cth * sph * vt - cph * vp)));
    }
};

// MIXED polar passage: the ray continues as an FP64 ray (same method, same
// termination tests and disk chords, E and Lz as the FP32 ray holds them) with
// its state carried in FP64 from step to step, until it leaves the cap
// |sin th| < kPolarCap or terminates; then the state is rounded back once.  The
// step that decided to enter is taken here, so the call advances at least one
// step.  Returns true when the ray terminated.  Out of line: the FP32 step
// loop keeps its register budget.
template <class R, bool STATS, bool MIXED>
__device__ __noinline__ bool KerrRay<R, STATS, MIXED>::polar_passage_fp64(const TraceParams& P)
{
    if constexpr (MIXED && std::is_same<R, float>::value)
    {
        const CamFrame<double>& D = P.cd;
        KerrRay<double, STATS, false> d;
        const double E = k.E, Lz = k.Lz;
        d.k = KerrConsts<double>{E, Lz, D.a * E, E * D.a2 - D.a * Lz, 2.0 * E};
        d.r = r; d.th = th; d.ph = ph; d.pr = pr; d.pth = pth;
        sincos_theta(d.th, d.s, d.c);
        KerrEval<double> ev = kerr_rhs(D, d.k, d.r, d.s, d.c, d.pr, d.pth);
        d.d1 = ev.d;
        d.K1 = ev.K;
        d.tFlight = tFlight;
        if (!prevCart) { prevPos = cart((R)prevPos.x, prevPos.y, (R)prevPos.z); prevCart = true; }
        d.prevPos = prevPos; d.prevCart = true; d.accum = accum; d.trans = trans; d.maxHviol = maxHviol;
        d.step = step; d.horizon = horizon; d.escaped = escaped; d.useDeriv = useDeriv;
        if (STATS) { d.tally = tally; d.Q0 = Q0; }
        bool done = false;
        // bounded by the step budget: every iteration takes a step or terminates
        while (!(done = d.advance(P)))
            if (abs_p(d.s) >= (double)kPolarCap) break;
        r = (R)d.r; th = (R)d.th; ph = (R)d.ph; pr = (R)d.pr; pth = (R)d.pth;
        tFlight = (R)d.tFlight;
        prevPos = d.prevPos; prevCart = true; accum = d.accum; trans = d.trans; maxHviol = d.maxHviol;
        step = d.step; horizon = d.horizon; escaped = d.escaped; useDeriv = d.useDeriv;
        if (STATS) tally = d.tally;
        if (done && escaped && useDeriv && step >= P.maxSteps)
        {   // budget exhausted inside the passage: the last stage's derivative
            const double* dd = KerrRay<double, STATS, false>::last_deriv();
            R* dl = last_deriv();
            dl[0] = (R)dd[0]; dl[1] = (R)dd[1]; dl[2] = (R)dd[2];
        }
        if (done)
        {   // pack() reads the escape derivative from d1
            d1.r = (R)d.d1.r; d1.th = (R)d.d1.th; d1.ph = (R)d.d1.ph; d1.pr = (R)d.d1.pr; d1.pth = (R)d.d1.pth;
            K1 = (R)d.K1;
            sincos_theta(th, s, c);
            return true;
        }
        // back to FP32: the next step's first right-hand side from the rounded state
        sincos_theta(th, s, c);
        KerrEval<R> e32 = kerr_rhs(frame_of<R>(P), k, r, s, c, pr, pth);
        d1 = e32.d;
        K1 = e32.K;
        return false;
    }
    return false;
}
