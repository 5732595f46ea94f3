#pragma once
// ---------------------------------------------------------------------------
// bh_integrate.cuh -- the two geodesic integrators as resumable ray objects.
//
// Each integrator is split into init() / step() / finish() so that a warp can
// hold 32 independent rays in registers and refill any lane whose ray ended
// (persistent-warp ray compaction, bh_trace.cu).  The arithmetic per step is
// the reference's method (Sqhh99/Black-hole):
//   SphRay   generalised Binet equation u'' = 3Mu^2 - 2Q^2u^3 - u, RK4 in the
//            orbital angle with the adaptive step of src/trace.cuh:466-611
//   KerrRay  Boyer-Lindquist Hamiltonian system (r, th, ph, p_r, p_th) with the
//            full dH derivatives (src/trace.cuh:620-659), static-observer
//            tetrad initial data (:704-739), adaptive affine step (:784-809),
//            RK4, pole guard, slow light and disk chords (:811-868)
// Termination tests and their order are the reference's, so step counts and
// outcomes agree ray by ray except where floating-point rounding decides.
//
// R is the integration precision (float: the product path; double: the GPU
// accuracy oracle).  Shading stays float in both.
//
// Arithmetic choices for R = float: divisions by state-dependent quantities
// use one MUFU reciprocal each (shared where a quantity divides twice);
// sin/cos of the polar angle use the polynomial sincos_polar (relative
// accuracy at the poles); the ever-growing azimuth uses sincos_fast.  The
// escape direction is rebuilt once per ray with the accurate library sincos.
// sin/cos of theta at the end of a step are carried into the next step's
// first right-hand side, the slow-light term and the Cartesian chord.
// ---------------------------------------------------------------------------
#include "bh_shade.cuh"

struct RayResult
{
    bool horizon, escaped;
    f3 escDir, accum;
    float trans, maxHviol, drift;
    int steps;
    DiskTally tally;
};

enum { RAY_SKIP = 0, RAY_LIVE = 1, RAY_DONE = 2 };

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

// Static-observer tetrad at the camera -> photon E, Lz (reference
// src/trace.cuh:213-247); accurate library functions.
template <class R>
BH_DEV void conserved_EL(vec3<R> o, vec3<R> dir, R M, R a, R Q, R& E, R& Lz)
{
    R r0 = sqrt_p(dot3(o, o));
    if (r0 < R(1e-4f)) { E = R(1); Lz = R(0); return; }
    R cth0 = min_p(max_p(o.y / r0, R(-1)), R(1));
    R th0 = acos(cth0);
    R ph0 = atan2(-o.z, o.x);
    R s = sin(th0);
    R sp, cp;
    sincos(ph0, &sp, &cp);
    R dpc = -dir.x * sp - dir.z * cp;
    R s0 = max_p(s, R(1e-4f));
    R s02 = s0 * s0;
    R Sig0 = r0 * r0 + a * a * cth0 * cth0;
    R m2r0 = R(2) * M * r0 - Q * Q;
    R gtt = -(R(1) - m2r0 / max_p(Sig0, R(1e-8f)));
    if (gtt > R(-1e-5f)) gtt = R(-1e-5f);
    R gtp = -a * m2r0 * s02 / Sig0;
    R gpp = (r0 * r0 + a * a + m2r0 * a * a * s02 / Sig0) * s02;
    R A = R(1) / sqrt_p(max_p(gpp - gtp * gtp / gtt, R(1e-8f)));
    R ptUp = R(1) / sqrt_p(-gtt) - dpc * A * gtp / gtt;
    R pfUp = dpc * A;
    E = -(gtt * ptUp + gtp * pfUp);
    Lz = gtp * ptUp + gpp * pfUp;
    if (!(E > R(1e-6f)) || !finite_p(E)) { E = R(1); Lz = R(0); }
}

// ===========================================================================
// Spherically symmetric metrics (Schwarzschild, Reissner-Nordstrom)
// ===========================================================================
template <class R, bool STATS>
struct SphRay
{
    R u, du, phi, tFlight, invB;
    R e1x, e1y, e1z, e2x, e2y, e2z;   // orbital-plane basis
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
        const R M = (R)P.M, Qc = (R)P.Q;
        vec3<R> c = widen<R>(tof3(P.camPos));
        vec3<R> dir = widen<R>(dirf);
        R Eph, Lph;
        conserved_EL(c, dir, M, R(0), Qc, Eph, Lph);
        E = (float)Eph; Lz = (float)Lph;

        horizon = escaped = haveDir = false;
        accum = v3(0.f, 0.f, 0.f);
        trans = 1.f;
        step = 0;
        tFlight = R(0);
        prevPos = tof3(P.camPos);
        if (STATS) { tally.samples = 0; tally.hitR = 0.f; tally.hitG = 0.f; }

        R r0 = sqrt_p(dot3(c, c));
        R ir0 = R(1) / r0;
        e1x = c.x * ir0; e1y = c.y * ir0; e1z = c.z * ir0;
        R ddr = dir.x * e1x + dir.y * e1y + dir.z * e1z;
        R px = dir.x - e1x * ddr, py = dir.y - e1y * ddr, pz = dir.z - e1z * ddr;
        R pl = sqrt_p(px * px + py * py + pz * pz);
        if (pl < R(1e-6f))
        {   // exactly radial ray (reference src/trace.cuh:447-459, 500-505)
            horizon = (dir.x * c.x + dir.y * c.y + dir.z * c.z) < R(0);
            escaped = !horizon;
            return RAY_DONE;
        }
        R ipl = R(1) / pl;
        e2x = px * ipl; e2y = py * ipl; e2z = pz * ipl;
        R f0 = max_p(R(1) - R(2) * M / r0 + Qc * Qc / (r0 * r0), R(1e-6f));
        R sf0 = sqrt_p(f0);
        invB = R(1) / max_p(r0 * pl / sf0, R(1e-6f));
        u = ir0;
        du = -sf0 * ddr / (r0 * pl);
        phi = R(0);
        if (STATS) I0 = binet(M, Qc * Qc, u, du);
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
            R sp, cp;
            sincos_fast(phi, sp, cp);
            f3 pos = v3((float)((e1x * cp + e2x * sp) * r), (float)((e1y * cp + e2y * sp) * r),
                        (float)((e1z * cp + e2z * sp) * r));
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

    BH_DEV void result(const TraceParams& P, f3 dir0, RayResult& o) const
    {
        o.horizon = horizon; o.escaped = escaped;
        o.accum = accum; o.trans = trans; o.steps = step;
        o.maxHviol = 0.f;
        o.escDir = dir0;
        if (escaped && haveDir)
        {   // chord direction of the last step, rebuilt with accurate trig
            R sp, cp;
            sincos(phid, &sp, &cp);
            R r = R(1) / ud;
            R drdphi = -dud / (ud * ud);
            R mx = e1x * cp + e2x * sp, my = e1y * cp + e2y * sp, mz = e1z * cp + e2z * sp;
            R qx = -e1x * sp + e2x * cp, qy = -e1y * sp + e2y * cp, qz = -e1z * sp + e2z * cp;
            o.escDir = normalize_x(v3((float)(mx * drdphi + qx * r), (float)(my * drdphi + qy * r),
                                      (float)(mz * drdphi + qz * r)));
        }
        if (STATS)
        {
            o.tally = tally;
            double I1 = binet((R)P.M, (R)P.Q * (R)P.Q, u, du);
            o.drift = (I0 > 0.0) ? (float)(fabs(I1 - I0) / I0) : 0.f;
        }
        else { o.drift = 0.f; o.tally.samples = 0; o.tally.hitR = 0.f; o.tally.hitG = 0.f; }
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
    {   // reference src/trace.cuh:703-739, accurate library functions
        const R M = (R)P.M, a = (R)P.a, Q = (R)P.Q;
        vec3<R> o = widen<R>(tof3(P.camPos));
        vec3<R> dir = widen<R>(dirf);
        R r0 = sqrt_p(dot3(o, o));
        R cth0 = min_p(max_p(o.y / r0, R(-1)), R(1));
        R th0 = acos(cth0);
        R ph0 = atan2(-o.z, o.x);
        R s0r, c0, sp, cp;
        sincos(th0, &s0r, &c0);
        sincos(ph0, &sp, &cp);
        R drc = dir.x * (s0r * cp) + dir.y * c0 + dir.z * (-s0r * sp);
        R dtc = dir.x * (c0 * cp) + dir.y * (-s0r) + dir.z * (-c0 * sp);
        R dpc = dir.x * (-sp) + dir.z * (-cp);
        R s0 = max_p(s0r, R(1e-4f));
        R s02 = s0 * s0;
        R Sig0 = r0 * r0 + a * a * cth0 * cth0;
        R Del0 = r0 * r0 - R(2) * M * r0 + a * a + Q * Q;
        R m2r0 = R(2) * M * r0 - Q * Q;
        R gtt = -(R(1) - m2r0 / Sig0);
        if (gtt > R(-1e-5f)) gtt = R(-1e-5f);
        R gtp = -a * m2r0 * s02 / Sig0;
        R gpp = (r0 * r0 + a * a + m2r0 * a * a * s02 / Sig0) * s02;
        R A = R(1) / sqrt_p(max_p(gpp - gtp * gtp / gtt, R(1e-8f)));
        R ptUp = R(1) / sqrt_p(-gtt) - dpc * A * gtp / gtt;
        R pfUp = dpc * A;
        E = -(gtt * ptUp + gtp * pfUp);
        Lz = gtp * ptUp + gpp * pfUp;

        r = r0; th = th0; ph = ph0;
        pr = drc * sqrt_p(Sig0 / max_p(Del0, R(1e-6f)));
        pth = dtc * sqrt_p(Sig0);
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
            Q0 = carterQ(th, pth, a, E, Lz);
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

        // classic RK4
        const R hh = R(0.5f) * h;
        R Kx, sx, cx;
        R yr = r + hh * d1.r, yth = th + hh * d1.th, ypr = pr + hh * d1.pr, ypth = pth + hh * d1.pth;
        sincos_polar(yth, sx, cx);
        KerrDeriv<R> d2 = kerr_rhs(M, a, Q2, E, Lz, yr, sx, cx, ypr, ypth, Kx);
        R sr = d1.r + R(2) * d2.r, sth = d1.th + R(2) * d2.th, sph = d1.ph + R(2) * d2.ph;
        R spr = d1.pr + R(2) * d2.pr, spth = d1.pth + R(2) * d2.pth;
        yr = r + hh * d2.r; yth = th + hh * d2.th; ypr = pr + hh * d2.pr; ypth = pth + hh * d2.pth;
        sincos_polar(yth, sx, cx);
        KerrDeriv<R> d3 = kerr_rhs(M, a, Q2, E, Lz, yr, sx, cx, ypr, ypth, Kx);
        sr += R(2) * d3.r; sth += R(2) * d3.th; sph += R(2) * d3.ph;
        spr += R(2) * d3.pr; spth += R(2) * d3.pth;
        yr = r + h * d3.r; yth = th + h * d3.th; ypr = pr + h * d3.pr; ypth = pth + h * d3.pth;
        sincos_polar(yth, sx, cx);
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

    BH_DEV void result(const TraceParams& P, f3 dir0, RayResult& o) const
    {
        o.horizon = horizon; o.escaped = escaped;
        o.accum = accum; o.trans = trans; o.steps = step;
        o.maxHviol = STATS ? maxHviol : 0.f;
        o.escDir = dir0;
        if (escaped && useDeriv)
        {   // kerrBasis(th, ph) applied to the coordinate derivative, accurate trig
            R sth, cth, sph, cph;
            sincos(th, &sth, &cth);
            sincos(ph, &sph, &cph);
            R vr = dr_, vt = r * dth_, vp = r * sth * dph_;
            f3 d = v3((float)(sth * cph * vr + cth * cph * vt - sph * vp),
                      (float)(cth * vr - sth * vt),
                      (float)(-sth * sph * vr - cth * sph * vt - cph * vp));
            o.escDir = normalize_x(d);
        }
        if (STATS)
        {
            o.tally = tally;
            const R a = (R)P.a;
            double q1 = carterQ(th, pth, a, E, Lz);
            double scale = fabs(Q0) + (double)Lz * Lz + (double)a * a * (double)E * E;
            o.drift = scale > 0.0 ? (float)(fabs(q1 - Q0) / scale) : 0.f;
        }
        else { o.drift = 0.f; o.tally.samples = 0; o.tally.hitR = 0.f; o.tally.hitG = 0.f; }
    }
};
