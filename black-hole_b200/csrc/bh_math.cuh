#pragma once
// ---------------------------------------------------------------------------
// bh_math.cuh -- device arithmetic shared by the tracer and post kernels.
//
// Three kinds of arithmetic are used on purpose:
//  * exact ("_x" helpers): IEEE round-to-nearest single operations with FMA
//    contraction blocked (__fadd_rn / __fmul_rn).  Used wherever the result
//    feeds a hash (the procedural star lattice, value noise, the dither), so
//    that a cell hash is bit-identical to the reference's host arithmetic; a
//    one-ulp change there would pick a different pseudo-random value.
//  * accurate: CUDA's full-precision library functions or the polynomial
//    sincos below, for quantities the geodesic state depends on.
//  * fast: MUFU-based intrinsics for shading weights, where a relative error
//    of ~1e-6 is far below the 1e-3 radiance tolerance.
// ---------------------------------------------------------------------------
#include <cuda_runtime.h>
#include <math_constants.h>

#define BH_DEV __device__ __forceinline__
// Large shading routines called from several places stay out of line: one
// copy in the kernel keeps the hot step loop's instruction footprint small.
#define BH_DEV_CALL static __device__ __noinline__

// ---- small vector type ------------------------------------------------------
template <class T> struct vec3 { T x, y, z; };
template <class T> BH_DEV vec3<T> v3(T x, T y, T z) { return vec3<T>{x, y, z}; }
template <class T> BH_DEV vec3<T> operator+(vec3<T> a, vec3<T> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> BH_DEV vec3<T> operator-(vec3<T> a, vec3<T> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> BH_DEV vec3<T> operator*(vec3<T> a, T s) { return v3(a.x * s, a.y * s, a.z * s); }
template <class T> BH_DEV T dot3(vec3<T> a, vec3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
typedef vec3<float> f3;
BH_DEV f3 tof3(float3 v) { return v3(v.x, v.y, v.z); }
template <class T> BH_DEV vec3<float> narrow(vec3<T> v) { return v3((float)v.x, (float)v.y, (float)v.z); }
template <class T> BH_DEV vec3<T> widen(f3 v) { return v3((T)v.x, (T)v.y, (T)v.z); }

// ---- exact single operations -------------------------------------------------
BH_DEV float add_x(float a, float b) { return __fadd_rn(a, b); }
BH_DEV float sub_x(float a, float b) { return __fsub_rn(a, b); }
BH_DEV float mul_x(float a, float b) { return __fmul_rn(a, b); }
BH_DEV float fract_x(float x) { return __fsub_rn(x, floorf(x)); }
// x * (1/sqrt(max(|v|^2, 1e-20))) with correctly rounded sqrt and divide:
// the reference host build evaluates normalize() this way.
BH_DEV f3 normalize_x(f3 a)
{
    float d = add_x(add_x(mul_x(a.x, a.x), mul_x(a.y, a.y)), mul_x(a.z, a.z));
    float k = __fdiv_rn(1.f, __fsqrt_rn(fmaxf(d, 1e-20f)));
    return v3(mul_x(a.x, k), mul_x(a.y, k), mul_x(a.z, k));
}

// ---- scalar helpers ----------------------------------------------------------
BH_DEV float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
BH_DEV double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }
BH_DEV float smoothstep_f(float e0, float e1, float x)
{
    float t = clampf(__fdividef(x - e0, e1 - e0), 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}
// fast reciprocal: one MUFU.RCP (relative error ~2^-23)
BH_DEV float rcp_f(float x) { float r; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
BH_DEV float rsqrt_f(float x) { float r; asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
// MUFU base-2 logarithm and exponential (absolute error ~2^-22 near 1, subnormals flushed)
BH_DEV float lg2_f(float x) { float r; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
BH_DEV float ex2_f(float x) { float r; asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
// fast square root (MUFU based, relative error ~2^-22, sqrt(0) = 0)
BH_DEV float sqrt_a(float x) { float r; asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }

// ---- sin/cos ---------------------------------------------------------------------
// Polynomial sincos for x in [0, pi] (the polar angle theta).  Reduce to
// v in [0, pi/4] by the reflections t = min(x, pi - x) and v = min(t, pi/2 - t)
// (pi and pi/2 split into a float head and tail; each difference is exact by
// Sterbenz's lemma where it is used), then evaluate the Taylor series of sin
// to degree 9 and cos to degree 10, whose truncation errors on [0, pi/4] are
// below 2e-9.  Both results keep relative accuracy at the poles (sin -> 0) and
// at the equator (cos -> 0), where a MUFU sine or cosine has only absolute
// accuracy (~4e-7).
BH_DEV void sincos_polar(float x, float& s, float& c)
{
    const float PI_HI = 3.14159274101257324f;       // float(pi)
    const float PI_LO = -8.74227765734758577e-8f;   // pi - float(pi)
    const float HPI_HI = 1.57079637050628662f;      // float(pi/2)
    const float HPI_LO = -4.37113882867379289e-8f;  // pi/2 - float(pi/2)
    float m = (PI_HI - x) + PI_LO;
    bool upper = m < x;
    float t = upper ? m : x;
    float u = (HPI_HI - t) + HPI_LO;
    bool swap = u < t;
    float v = swap ? u : t;
    float v2 = v * v;
    // sin v = v - v^3/3! + v^5/5! - v^7/7! + v^9/9!
    float ps = fmaf(v2, 2.75573192239858907e-6f, -1.98412698412698413e-4f);
    ps = fmaf(v2, ps, 8.33333333333333333e-3f);
    ps = fmaf(v2, ps, -1.66666666666666667e-1f);
    float sv = fmaf(v * v2, ps, v);
    // cos v = 1 - v^2/2! + v^4/4! - v^6/6! + v^8/8! - v^10/10!
    float pc = fmaf(v2, -2.75573192239858907e-7f, 2.48015873015873016e-5f);
    pc = fmaf(v2, pc, -1.38888888888888889e-3f);
    pc = fmaf(v2, pc, 4.16666666666666667e-2f);
    pc = fmaf(v2, pc, -0.5f);
    float cv = fmaf(v2, pc, 1.f);
    s = swap ? cv : sv;
    c = swap ? sv : cv;
    if (upper) c = -c;
}

// Fast sincos for an unbounded angle (an azimuth that keeps growing along the
// ray): Cody-Waite reduction by 2*pi with a two-part constant, then the MUFU
// sine/cosine on [-pi, pi] (absolute error ~4e-7).
BH_DEV void sincos_fast(float x, float& s, float& c)
{
    const float INV_2PI = 0.159154943091895336f;
    const float TWO_PI_HI = 6.28318548202514648f;   // float(2 pi)
    const float TWO_PI_LO = -1.74845553146951715e-7f;
    float k = rintf(x * INV_2PI);
    float r = fmaf(-k, TWO_PI_HI, x);
    r = fmaf(-k, TWO_PI_LO, r);
    __sincosf(r, &s, &c);
}

// Accurate versions for the double-precision integrator.
BH_DEV void sincos_polar(double x, double& s, double& c) { sincos(x, &s, &c); }

// sin/cos in double for angles near either pole: the Taylor series to degree
// 13 (sin) and 12 (cos) for |x| <= 0.2 (remainder below 1e-17 relative), and
// for |pi - x| <= 0.2 through sin(pi - t) = sin t, cos(pi - t) = -cos t with
// pi - x formed in two parts; the library sincos elsewhere.  Polar angles of
// the FP64 steps near the spin axis lie in that range, where this costs a
// dozen FMAs instead of a general argument reduction.
BH_DEV void sincos_cap(double x, double& s, double& c)
{
    const double PI_HI = 3.141592653589793116, PI_LO = 1.2246467991473532e-16;
    double t = x, sc = 1.0;
    if (fabs(x) > 0.2)
    {
        if (fabs(PI_HI - x) > 0.2) { sincos(x, &s, &c); return; }
        t = (PI_HI - x) + PI_LO;
        sc = -1.0;
    }
    const double t2 = t * t;
    double ps = -1.0 / 6227020800.0;                 // -1/13!
    ps = fma(ps, t2, 1.0 / 39916800.0);
    ps = fma(ps, t2, -1.0 / 362880.0);
    ps = fma(ps, t2, 1.0 / 5040.0);
    ps = fma(ps, t2, -1.0 / 120.0);
    ps = fma(ps, t2, 1.0 / 6.0);
    s = fma(-t * t2, ps, t);                         // t - t^3/3! + t^5/5! - ...
    double pc = 1.0 / 479001600.0;                   // 1/12!
    pc = fma(pc, t2, -1.0 / 3628800.0);
    pc = fma(pc, t2, 1.0 / 40320.0);
    pc = fma(pc, t2, -1.0 / 720.0);
    pc = fma(pc, t2, 1.0 / 24.0);
    pc = fma(pc, t2, -0.5);
    c = sc * fma(pc, t2, 1.0);                       // 1 - t^2/2! + t^4/4! - ...
}
BH_DEV void sincos_fast(double x, double& s, double& c) { sincos(x, &s, &c); }

// precision-generic elementary functions
BH_DEV float  rcp_p(float x)  { return rcp_f(x); }
BH_DEV double rcp_p(double x) { return 1.0 / x; }
BH_DEV float  rsqrt_p(float x)  { return rsqrt_f(x); }
BH_DEV double rsqrt_p(double x) { return rsqrt(x); }
BH_DEV float  sqrt_p(float x)  { return sqrtf(x); }
BH_DEV double sqrt_p(double x) { return sqrt(x); }
BH_DEV float  abs_p(float x)  { return fabsf(x); }
BH_DEV double abs_p(double x) { return fabs(x); }
BH_DEV float  min_p(float a, float b)   { return fminf(a, b); }
BH_DEV double min_p(double a, double b) { return fmin(a, b); }
BH_DEV float  max_p(float a, float b)   { return fmaxf(a, b); }
BH_DEV double max_p(double a, double b) { return fmax(a, b); }
// Two independent a * x_i + y_i sharing a: one packed FP32x2 FMA on sm_100
// (each component rounded exactly as a scalar FMA), two FMAs in FP64.
BH_DEV void fma2_p(float a, float x0, float x1, float y0, float y1, float& o0, float& o1)
{
    const float2 v = __ffma2_rn(make_float2(a, a), make_float2(x0, x1), make_float2(y0, y1));
    o0 = v.x;
    o1 = v.y;
}
BH_DEV void fma2_p(double a, double x0, double x1, double y0, double y1, double& o0, double& o1)
{
    o0 = fma(a, x0, y0);
    o1 = fma(a, x1, y1);
}
// Two independent sums / products (packed in FP32).
BH_DEV void add2_p(float x0, float x1, float y0, float y1, float& o0, float& o1)
{
    const float2 v = __fadd2_rn(make_float2(x0, x1), make_float2(y0, y1));
    o0 = v.x;
    o1 = v.y;
}
BH_DEV void add2_p(double x0, double x1, double y0, double y1, double& o0, double& o1)
{
    o0 = x0 + y0;
    o1 = x1 + y1;
}
BH_DEV void mul2_p(float x0, float x1, float y0, float y1, float& o0, float& o1)
{
    const float2 v = __fmul2_rn(make_float2(x0, x1), make_float2(y0, y1));
    o0 = v.x;
    o1 = v.y;
}
BH_DEV void mul2_p(double x0, double x1, double y0, double y1, double& o0, double& o1)
{
    o0 = x0 * y0;
    o1 = x1 * y1;
}
// ---- lane arithmetic: one ray (float / double) or two rays packed (float2) ----
// Explicit IEEE operations (no contraction decided by the compiler), so a
// computation written once gives the same bits for a single ray and for each
// half of a packed pair.
BH_DEV float  vfma(float a, float b, float c)    { return __fmaf_rn(a, b, c); }
BH_DEV double vfma(double a, double b, double c) { return fma(a, b, c); }
BH_DEV float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
BH_DEV float  vmul(float a, float b)    { return __fmul_rn(a, b); }
BH_DEV double vmul(double a, double b)  { return __dmul_rn(a, b); }
BH_DEV float2 vmul(float2 a, float2 b)  { return __fmul2_rn(a, b); }
BH_DEV float  vadd(float a, float b)    { return __fadd_rn(a, b); }
BH_DEV double vadd(double a, double b)  { return __dadd_rn(a, b); }
BH_DEV float2 vadd(float2 a, float2 b)  { return __fadd2_rn(a, b); }
BH_DEV float  vsub(float a, float b)    { return __fsub_rn(a, b); }
BH_DEV double vsub(double a, double b)  { return __dsub_rn(a, b); }
BH_DEV float2 vsub(float2 a, float2 b)  { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
BH_DEV float  vneg(float a)  { return -a; }
BH_DEV double vneg(double a) { return -a; }
BH_DEV float2 vneg(float2 a) { return make_float2(-a.x, -a.y); }
BH_DEV float  vmax(float a, float b)    { return fmaxf(a, b); }
BH_DEV double vmax(double a, double b)  { return fmax(a, b); }
BH_DEV float2 vmax(float2 a, float2 b)  { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
BH_DEV float  vrcp(float a)  { return rcp_f(a); }
BH_DEV double vrcp(double a) { return 1.0 / a; }
BH_DEV float2 vrcp(float2 a) { return make_float2(rcp_f(a.x), rcp_f(a.y)); }
// a per-frame scalar (float or double) in every lane of V
template <class V, class S> BH_DEV V lane(S x) { return (V)x; }
template <> BH_DEV float2 lane<float2, float>(float x) { return make_float2(x, x); }

BH_DEV bool   finite_p(float x)  { return isfinite(x); }
BH_DEV bool   finite_p(double x) { return isfinite(x); }

// ---- hashes and value noise (exact arithmetic; reference vec_math.cuh:56-98) ------
BH_DEV float hash12(float px, float py)
{
    float ax = fract_x(mul_x(px, 0.1031f));
    float ay = fract_x(mul_x(py, 0.1031f));
    float az = ax;  // the reference hashes p.x twice: fract(p.x * 0.1031)
    float d = add_x(add_x(mul_x(ax, add_x(ay, 33.33f)), mul_x(ay, add_x(az, 33.33f))),
                    mul_x(az, add_x(ax, 33.33f)));
    ax = add_x(ax, d); ay = add_x(ay, d); az = add_x(az, d);
    return fract_x(mul_x(add_x(ax, ay), az));
}

BH_DEV f3 hash33(f3 p)
{
    float x = fract_x(mul_x(p.x, 0.1031f));
    float y = fract_x(mul_x(p.y, 0.1030f));
    float z = fract_x(mul_x(p.z, 0.0973f));
    float d = add_x(add_x(mul_x(x, add_x(y, 33.33f)), mul_x(y, add_x(x, 33.33f))),
                    mul_x(z, add_x(z, 33.33f)));
    x = add_x(x, d); y = add_x(y, d); z = add_x(z, d);
    return v3(fract_x(mul_x(add_x(x, y), z)), fract_x(mul_x(add_x(x, z), y)),
              fract_x(mul_x(add_x(y, z), x)));
}

BH_DEV float lerp_x(float a, float b, float t) { return add_x(a, mul_x(sub_x(b, a), t)); }

BH_DEV float vnoise(float px, float py)
{
    float ix = floorf(px), iy = floorf(py);
    float fx = sub_x(px, ix), fy = sub_x(py, iy);
    float ux = mul_x(mul_x(fx, fx), sub_x(3.f, mul_x(2.f, fx)));
    float uy = mul_x(mul_x(fy, fy), sub_x(3.f, mul_x(2.f, fy)));
    float c00 = hash12(ix, iy);
    float c10 = hash12(add_x(ix, 1.f), add_x(iy, 0.f));
    float c01 = hash12(add_x(ix, 0.f), add_x(iy, 1.f));
    float c11 = hash12(add_x(ix, 1.f), add_x(iy, 1.f));
    return lerp_x(lerp_x(c00, c10, ux), lerp_x(c01, c11, ux), uy);
}

BH_DEV_CALL float fbm3(float px, float py)
{
    float v = 0.f, amp = 0.5f;
#pragma unroll
    for (int o = 0; o < 3; ++o)
    {
        v = add_x(v, mul_x(amp, vnoise(px, py)));
        float nx = add_x(mul_x(px, 2.03f), 11.7f);
        float ny = sub_x(mul_x(py, 2.01f), 5.2f);
        px = nx; py = ny;
        amp = mul_x(amp, 0.5f);
    }
    return v;
}
