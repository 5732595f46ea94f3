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
// MUFU reciprocal each; sin/cos of the polar angle at the start of a step come
// from the polynomial sincos_polar (relative accuracy at poles and equator)
// and are carried into the next step's first right-hand side, the slow-light
// term and the Cartesian chord; the three RK4 stage angles th + delta use the
// angle-addition formula from that anchored pair; the ever-growing azimuth
// uses sincos_fast.  The escape direction is rebuilt once per ray with the
// accurate library sincos.
// ---------------------------------------------------------------------------
#include "bh_shade.cuh"

enum { RAY_SKIP = 0, RAY_LIVE = 1, RAY_DONE = 2 };

// A finished ray as it waits for shading: outcome flags, the radiance gathered
// from the disk, and the six state values from which the escape direction is
// rebuilt at shading time (so the finishing lane only stores, and the
// trigonometry runs later with the whole warp converged).
constexpr unsigned kRayHorizon = 1u << 31, kRayEscaped = 1u << 30, kRayUseState = 1u << 29;
constexpr unsigned kRayKeyMask = kRayUseState - 1u;

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

// sin/cos of th + delta from the anchored pair (s, c) of th.  FP32: angle
// addition with the Taylor series of sin / cos delta to degree 7 / 6
// (truncation < 4e-10 for |delta| <= 0.3; the adaptive step keeps a stage's
// angular advance below 2.2 dPhi <= 0.22); larger deltas fall back to the
// full polynomial.  FP64: the library sincos.
BH_DEV void sincos_shift(float th, float s, float c, float delta, float& so, float& co)
{
    if (fabsf(delta) > 0.3f)
    {
        sincos_polar(th + delta, so, co);
        return;
    }
    float d2 = delta * delta;
    float ps = fmaf(d2, -1.98412698412698413e-4f, 8.33333333333333333e-3f);
    ps = fmaf(d2, ps, -1.66666666666666667e-1f);
    float sd = fmaf(delta * d2, ps, delta);
    float pc = fmaf(d2, -1.38888888888888889e-3f, 4.16666666666666667e-2f);
    pc = fmaf(d2, pc, -0.5f);
    float cd = fmaf(d2, pc, 1.f);
    so = fmaf(s, cd, c * sd);
    co = fmaf(c, cd, -(s * sd));
}
BH_DEV void sincos_shift(double th, double, double, double delta, double& so, double& co)
{
    sincos(th + delta, &so, &co);
}

// ===========================================================================
// Spherically symmetric metrics (Schwarzschild, Reissner-Nordstrom)
// ===========================================================================
template <class R, bool STATS>
struct SphRay
{
    using Real = R;
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
        const CamFrame<R>& F = frame_of<R>(P);
        const vec3<R> dir = widen<R>(dirf);
        horizon = escaped = haveDir = false;
        accum = v3(0.f, 0.f, 0.f);
        trans = 1.f;
        step = 0;
        tFlight = R(0);
        prevPos = tof3(P.camPos);
        if (STATS) { tally.samples = 0; tally.hitR = 0.f; tally.hitG = 0.f; I0 = 0.0; }

        // photon E, Lz (reference src/trace.cuh:213-247 with a = 0)
        R Eph = R(1), Lph = R(0);
        if (!F.camAtOrigin)
        {
            R dpc = xdot(F.ephS, dir);
            R ptUp = xsub(F.rsqS, xdiv(xmul(xmul(dpc, F.AS), F.gtpS), F.gttS));
            R pfUp = xmul(dpc, F.AS);
            Eph = -xadd(xmul(F.gttS, ptUp), xmul(F.gtpS, pfUp));
            Lph = xadd(xmul(F.gtpS, ptUp), xmul(F.gppS, pfUp));
            if (!(Eph > R(1e-6f)) || !finite_p(Eph)) { Eph = R(1); Lph = R(0); }
        }
        E = (float)Eph; Lz = (float)Lph;

        // orbital plane (reference src/trace.cuh:490-521)
        R ddr = xdot(F.e1, dir);
        R px = xsub(dir.x, xmul(F.e1[0], ddr));
        R py = xsub(dir.y, xmul(F.e1[1], ddr));
        R pz = xsub(dir.z, xmul(F.e1[2], ddr));
        R pl = xsqrt(xadd(xadd(xmul(px, px), xmul(py, py)), xmul(pz, pz)));
        if (pl < R(1e-6f))
        {   // exactly radial ray (reference src/trace.cuh:447-459, 500-505)
            const vec3<R> c = widen<R>(tof3(P.camPos));
            horizon = xadd(xadd(xmul(dir.x, c.x), xmul(dir.y, c.y)), xmul(dir.z, c.z)) < R(0);
            escaped = !horizon;
            return RAY_DONE;
        }
        R ipl = xdiv(R(1), pl);
        e2x = xmul(px, ipl); e2y = xmul(py, ipl); e2z = xmul(pz, ipl);
        R bImpact = max_p(xdiv(xmul(F.r0, pl), F.sf0), R(1e-6f));
        invB = rcp_p(bImpact);
        u = F.u0;
        du = xdiv(xmul(-F.sf0, ddr), xmul(F.r0, pl));
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
        const R M = (R)P.M, Q2 = (R)P.Q * (R)P.Q, dPhi = (R)P.dPhi;
        if (step >= P.maxSteps) { exhaust(P); return true; }

        const R invNineM = R(1) / (R(9) * M);
        R hMax = dPhi * min_p(max_p(invNineM * rcp_p(u), R(1)), R(6));
        R h = min_p(hMax, R(0.10f) * rcp_p(max_p(abs_p(du), R(1e-6f))));
        h = max_p(h, dPhi * R(0.03f));

        const R m3 = R(3) * M, q2 = R(2) * Q2;
        auto acc = [&](R x) { return (m3 * x - q2 * x * x) * x - x; };
        R hh = R(0.5f) * h;
        R k1v = acc(u);
        R u2 = u + hh * du, v2 = du + hh * k1v;
        R k2v = acc(u2);
        R u3 = u + hh * v2, v3_ = du + hh * k2v;
        R k3v = acc(u3);
        R u4 = u + h * v3_, v4 = du + h * k3v;
        R k4v = acc(u4);
        R h6 = h * R(1.0 / 6.0);
        u += h6 * (du + R(2) * v2 + R(2) * v3_ + v4);
        du += h6 * (k1v + R(2) * k2v + R(2) * k3v + k4v);
        phi += h;

        const R uHor = R(1) / max_p((R)capture_radius(P), R(1e-6f));
        if (!finite_p(u) || !finite_p(du)) { horizon = true; return true; }
        if (u >= uHor) { horizon = true; return true; }
        if (u < R(1e-4f)) { escaped = true; return true; }   // previous chord direction

        R r = rcp_p(u);
        ud = u; dud = du; phid = phi; haveDir = true;
        R fR = max_p(R(1) - R(2) * M * u + Q2 * u * u, R(1e-4f));
        tFlight += h * r * r * invB * rcp_p(fR);

        if (P.diskOn && trans > 0.01f)
        {
            const CamFrame<R>& F = frame_of<R>(P);
            R sp, cp;
            sincos_fast(phi, sp, cp);
            f3 pos = v3((float)((F.e1[0] * cp + e2x * sp) * r), (float)((F.e1[1] * cp + e2y * sp) * r),
                        (float)((F.e1[2] * cp + e2z * sp) * r));
            disk_segment<STATS>(P, E, Lz, prevPos, pos, (float)((R)P.diskTime - tFlight),
                                accum, trans, tally);
            prevPos = pos;
        }
        ++step;
        const R uEscape = R(1) / (R(120) * M);
        if (u < uEscape && du < R(0)) { escaped = true; return true; }
        return false;
    }

    BH_DEV void exhaust(const TraceParams& P)
    {   // budget spent: reference src/trace.cuh:603-609
        const R M = (R)P.M;
        if (u > R(1) / max_p(R(1.5f) * (R)P.rPhoton, R(3) * M)) horizon = true;
        else escaped = true;
    }

    BH_DEV void pack(const TraceParams& P, unsigned key, PackedRay<R>& q, PackedStats* st) const
    {
        const bool useState = escaped && haveDir;
        q.key = key | (horizon ? kRayHorizon : 0u) | (escaped ? kRayEscaped : 0u) | (useState ? kRayUseState : 0u);
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
template <class R>
BH_DEV KerrDeriv<R> kerr_rhs(R M, R a, R Q2, R E, R Lz, R r, R s, R c, R pr, R pth, R& K)
{
    s = max_p(s, R(1e-4f));                 // pole guard
    const R a2 = a * a, aE = a * E;
    R r2 = r * r;
    R Sig = r2 + a2 * c * c;
    R Del = max_p(r2 - R(2) * M * r + a2 + Q2, R(1e-6f));
    R Pp = E * (r2 + a2) - a * Lz;
    R is = rcp_p(s);
    R is2 = is * is;
    R B = Lz * is - aE * s;
    R iDel = rcp_p(Del);
    R PiD = Pp * iDel;
    R W = B * B - Pp * PiD;
    K = Del * pr * pr + pth * pth + W;
    R dDel = R(2) * r - R(2) * M;
    R dP = R(2) * r * E;
    R Wr = -PiD * (R(2) * dP - PiD * dDel);
    R Wth = R(2) * B * (-c * (Lz * is2 + aE));
    R iS = rcp_p(Sig);
    R iS2 = iS * iS;
    KerrDeriv<R> d;
    d.r = Del * pr * iS;
    d.th = pth * iS;
    d.ph = ((Lz * is2 - aE) + a * PiD) * iS;
    d.pr = R(-0.5f) * iS * (dDel * pr * pr + Wr) + r * iS2 * K;
    d.pth = R(-0.5f) * iS * Wth - a2 * s * c * iS2 * K;
    return d;
}

template <class R, bool STATS>
struct KerrRay
{
    using Real = R;
    R r, th, ph, pr, pth;   // Boyer-Lindquist state
    R s, c;                 // sin/cos of th, carried between steps
    R E, Lz, tFlight;
    R dr_, dth_, dph_;      // coordinate derivative that defines the escape direction
    f3 prevPos, accum;
    float trans, maxHviol;
    int step;
    bool horizon, escaped, useDeriv;
    DiskTally tally;
    double Q0;

    BH_DEV int init(const TraceParams& P, f3 dirf)
    {   // reference src/trace.cuh:703-739: the per-ray remainder of the tetrad map
        const CamFrame<R>& F = frame_of<R>(P);
        const vec3<R> dir = widen<R>(dirf);
        R drc = xdot(F.er, dir), dtc = xdot(F.eth, dir), dpc = xdot(F.eph, dir);
        R ptUp = xsub(F.rsq, xdiv(xmul(xmul(dpc, F.A), F.gtp), F.gtt));
        R pfUp = xmul(dpc, F.A);
        E = -xadd(xmul(F.gtt, ptUp), xmul(F.gtp, pfUp));
        Lz = xadd(xmul(F.gtp, ptUp), xmul(F.gpp, pfUp));
        r = F.r0; th = F.th0; ph = F.ph0;
        pr = xmul(drc, F.sqSD);
        pth = xmul(dtc, F.sqS);
        sincos_polar(th, s, c);

        tFlight = R(0);
        prevPos = tof3(P.camPos);
        accum = v3(0.f, 0.f, 0.f);
        trans = 1.f;
        maxHviol = 0.f;
        step = 0;
        horizon = escaped = useDeriv = false;
        dr_ = dth_ = dph_ = R(0);
        if (STATS)
        {
            tally.samples = 0; tally.hitR = 0.f; tally.hitG = 0.f;
            Q0 = carterQ(th, pth, (R)P.a, E, Lz);
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

    // One reference loop iteration (src/trace.cuh:752-868).  Returns true when
    // the ray has terminated.
    BH_DEV bool advance(const TraceParams& P)
    {
        if (step >= P.maxSteps) { exhaust(P); return true; }
        const R M = (R)P.M, a = (R)P.a, Q2 = (R)P.Q * (R)P.Q;
        const R dPhi = (R)P.dPhi;
        const R rCap = (R)capture_radius(P);
        const R rFloor = max_p((R)P.rPlus, rCap);

        R K1;
        KerrDeriv<R> d1 = kerr_rhs(M, a, Q2, E, Lz, r, s, c, pr, pth, K1);
        if (!finite_p(r) || !finite_p(pr) || !finite_p(pth) || !finite_p(d1.r) || !finite_p(d1.pr))
        { horizon = true; return true; }
        if (r <= rCap * R(1.002f) + R(1e-3f)) { horizon = true; return true; }
        if (STATS && r > rFloor * R(1.05f))
        {
            float viol = (float)(abs_p(K1) / (E * E * (r * r + a * a) + R(1e-12f)));
            maxHviol = fmaxf(maxHviol, viol);
        }
        if (r >= R(120) * M && d1.r > R(0))
        {
            dr_ = d1.r; dth_ = d1.th; dph_ = d1.ph;
            escaped = useDeriv = true;
            return true;
        }

        // adaptive affine step (reference src/trace.cuh:793-809)
        const R i8 = rcp_p(R(8.0f) * dPhi * max_p(r - rFloor, R(0.02f)));
        const R ang = abs_p(d1.th) + abs_p(d1.ph);
        R h = rcp_p(abs_p(d1.r) * i8 + ang * rcp_p(R(2.2f) * dPhi) + R(1e-5f));
        if (r < R(1.5f) * (R)P.rPhoton) h *= R(0.55f);
        R spd = abs_p(d1.r) + r * ang + R(1e-6f);
        R capLen;
        if (P.diskOn && r < (R)P.diskOuter * R(1.3f))
            capLen = (r * abs_p(c) < R(1.8f)) ? R(1.2f) : R(2.2f);
        else
            capLen = max_p(R(1.2f), R(0.22f) * r);
        h = min_p(h, capLen * rcp_p(spd));

        // classic RK4; stage angles th + delta via angle addition from (s, c)
        const R hh = R(0.5f) * h;
        R Kx, sx, cx;
        R yr = r + hh * d1.r, ypr = pr + hh * d1.pr, ypth = pth + hh * d1.pth;
        sincos_shift(th, s, c, hh * d1.th, sx, cx);
        KerrDeriv<R> d2 = kerr_rhs(M, a, Q2, E, Lz, yr, sx, cx, ypr, ypth, Kx);
        R sr = d1.r + R(2) * d2.r, sth = d1.th + R(2) * d2.th, sph = d1.ph + R(2) * d2.ph;
        R spr = d1.pr + R(2) * d2.pr, spth = d1.pth + R(2) * d2.pth;
        yr = r + hh * d2.r; ypr = pr + hh * d2.pr; ypth = pth + hh * d2.pth;
        sincos_shift(th, s, c, hh * d2.th, sx, cx);
        KerrDeriv<R> d3 = kerr_rhs(M, a, Q2, E, Lz, yr, sx, cx, ypr, ypth, Kx);
        sr += R(2) * d3.r; sth += R(2) * d3.th; sph += R(2) * d3.ph;
        spr += R(2) * d3.pr; spth += R(2) * d3.pth;
        yr = r + h * d3.r; ypr = pr + h * d3.pr; ypth = pth + h * d3.pth;
        sincos_shift(th, s, c, h * d3.th, sx, cx);
        KerrDeriv<R> d4 = kerr_rhs(M, a, Q2, E, Lz, yr, sx, cx, ypr, ypth, Kx);
        const R h6 = h * R(1.0 / 6.0);
        r += h6 * (sr + d4.r);
        th += h6 * (sth + d4.th);
        ph += h6 * (sph + d4.ph);
        pr += h6 * (spr + d4.pr);
        pth += h6 * (spth + d4.pth);

        // pole reflection guard
        if (th < R(1e-3f)) { th = R(1e-3f); pth = abs_p(pth); }
        else if (th > R(kPiF - 1e-3f)) { th = R(kPiF - 1e-3f); pth = -abs_p(pth); }
        dr_ = d4.r; dth_ = d4.th; dph_ = d4.ph;   // dLast of the reference
        sincos_polar(th, s, c);

        {   // slow light: Sigma dt/dl = a (Lz - a E sin^2) + (r^2 + a^2) P / Delta
            R sc = max_p(s, R(1e-4f));
            R r2a2 = r * r + a * a;
            R Sig = r * r + a * a * c * c;
            R Del = max_p(r * r - R(2) * M * r + a * a + Q2, R(1e-5f));
            R Pp = E * r2a2 - a * Lz;
            R dtdl = (a * (Lz - a * E * sc * sc) + r2a2 * Pp * rcp_p(Del)) * rcp_p(max_p(Sig, R(1e-8f)));
            tFlight += h * abs_p(dtdl);
        }
        if (P.diskOn)
        {
            R sp, cp;
            sincos_fast(ph, sp, cp);
            f3 pos = v3((float)(r * s * cp), (float)(r * c), (float)(-r * s * sp));
            if (trans > 0.01f)
                disk_segment<STATS>(P, (float)E, (float)Lz, prevPos, pos,
                                    (float)((R)P.diskTime - tFlight), accum, trans, tally);
            prevPos = pos;
        }
        ++step;
        return false;
    }

    BH_DEV void exhaust(const TraceParams& P)
    {   // budget spent: reference src/trace.cuh:871-888
        if (r < R(6) * (R)P.M) horizon = true;
        else { escaped = true; useDeriv = step > 0; }
    }

    BH_DEV void pack(const TraceParams& P, unsigned key, PackedRay<R>& q, PackedStats* st) const
    {
        const bool useState = escaped && useDeriv;
        q.key = key | (horizon ? kRayHorizon : 0u) | (escaped ? kRayEscaped : 0u) | (useState ? kRayUseState : 0u);
        q.acc[0] = accum.x; q.acc[1] = accum.y; q.acc[2] = accum.z;
        q.trans = trans;
        q.f[0] = r; q.f[1] = th; q.f[2] = ph; q.f[3] = dr_; q.f[4] = dth_; q.f[5] = dph_;
        if (STATS)
        {
            st->steps = step; st->samples = tally.samples; st->maxHviol = maxHviol;
            st->hitR = tally.hitR; st->hitG = tally.hitG;
            const R a = (R)P.a;
            double q1 = carterQ(th, pth, a, E, Lz);
            double scale = fabs(Q0) + (double)Lz * Lz + (double)a * a * (double)E * E;
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
