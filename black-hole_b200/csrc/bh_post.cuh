#pragma once
// ---------------------------------------------------------------------------
// bh_post.cuh -- display pipeline arithmetic (reference src/post_process.cuh):
// ACES tone map, vibrance, gamma, triangular-pdf dither, 8-bit quantisation,
// accumulation blend and the bloom bright-pass / Gaussian weights.
//
// Everything here uses exact (uncontracted, correctly rounded) operations, so
// that, given the same HDR input, the 8-bit output equals the reference's host
// arithmetic except where a gamma power rounds differently (a one-LSB case).
// ---------------------------------------------------------------------------
#include "bh_math.cuh"
#include "bh_internal.h"

BH_DEV f3 aces_x(f3 x)
{
    const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
    auto one = [&](float v) {
        float num = mul_x(v, add_x(mul_x(v, A), B));
        float den = add_x(mul_x(v, add_x(mul_x(v, C), D)), E);
        return clampf(__fdiv_rn(num, den), 0.f, 1.f);
    };
    return v3(one(x.x), one(x.y), one(x.z));
}

// Gamma 1/2.2, dither and 8-bit quantisation of one channel x in [0, 1]:
// byte = trunc(clamp(x^(1/2.2) + dd, 0, 1) * 255 + 0.5), the power being the
// full-accuracy powf.  The MUFU form exp2(log2(x) / 2.2) (relative error
// below 1e-6, i.e. below 3e-4 in units of the unrounded byte value y) decides
// the byte wherever y lies more than 1e-3 from a truncation boundary; within
// that margin powf recomputes it.  The byte is therefore always the one powf
// gives, at a fraction of its cost (powf was a third of the tonemap's work).
BH_DEV unsigned char gamma_q8(float x, float dd)
{
    const float g = 1.0f / 2.2f;
    float y = add_x(mul_x(clampf(add_x(ex2_f(mul_x(lg2_f(x), g)), dd), 0.f, 1.f), 255.f), 0.5f);
    const float fr = sub_x(y, floorf(y));
    if (fr < 1e-3f || fr > 0.999f)
        y = add_x(mul_x(clampf(add_x(powf(x, g), dd), 0.f, 1.f), 255.f), 0.5f);
    return (unsigned char)__float2uint_rz(y);
}

// exposure -> bloom composite -> ACES -> vibrance 1.12 -> gamma 1/2.2 -> dither -> u8
BH_DEV uchar4 finalize_pixel(f3 hdr, f3 bloom, const PostConsts& pc, int px, int py)
{
    f3 c = v3(mul_x(hdr.x, pc.exposure), mul_x(hdr.y, pc.exposure), mul_x(hdr.z, pc.exposure));
    if (pc.bloomOn)
        c = v3(add_x(c.x, mul_x(bloom.x, pc.bloomStrength)), add_x(c.y, mul_x(bloom.y, pc.bloomStrength)),
               add_x(c.z, mul_x(bloom.z, pc.bloomStrength)));
    c = aces_x(c);
    float lum = add_x(add_x(mul_x(0.2126f, c.x), mul_x(0.7152f, c.y)), mul_x(0.0722f, c.z));
    c = v3(clampf(add_x(lum, mul_x(sub_x(c.x, lum), 1.12f)), 0.f, 1.f),
           clampf(add_x(lum, mul_x(sub_x(c.y, lum), 1.12f)), 0.f, 1.f),
           clampf(add_x(lum, mul_x(sub_x(c.z, lum), 1.12f)), 0.f, 1.f));
    float fx = (float)px, fy = (float)py;
    float d = sub_x(add_x(hash12(fx, fy), hash12(add_x(fx, 41.3f), add_x(fy, 17.7f))), 1.0f);
    float dd = mul_x(d, 1.0f / 255.0f);
    unsigned char r8 = gamma_q8(c.x, dd), g8 = gamma_q8(c.y, dd), b8 = gamma_q8(c.z, dd);
    return pc.swapRB ? make_uchar4(b8, g8, r8, 255) : make_uchar4(r8, g8, b8, 255);
}

// Blend a new HDR sample into the accumulation value (reference post_process.cuh:56-68).
BH_DEV f3 accum_blend(f3 prev, f3 cur, int mode, int idx)
{
    if (mode == 0 || idx <= 0) return cur;
    float w = (mode == 1) ? __fdiv_rn(1.0f, add_x((float)idx, 1.0f)) : 0.42f;
    return v3(add_x(prev.x, mul_x(sub_x(cur.x, prev.x), w)), add_x(prev.y, mul_x(sub_x(cur.y, prev.y), w)),
              add_x(prev.z, mul_x(sub_x(cur.z, prev.z), w)));
}

// Smooth bright-pass on the exposed colour (reference post_process.cuh:76-84).
BH_DEV f3 bright_pass(f3 c)
{
    float l = add_x(add_x(mul_x(0.2126f, c.x), mul_x(0.7152f, c.y)), mul_x(0.0722f, c.z));
    float t = clampf(__fdiv_rn(sub_x(l, 0.95f), sub_x(2.2f, 0.95f)), 0.f, 1.f);
    float w = mul_x(mul_x(t, t), sub_x(3.f, mul_x(2.f, t)));
    return v3(mul_x(c.x, w), mul_x(c.y, w), mul_x(c.z, w));
}

// normalised 9-tap Gaussian, sigma ~3 half-res pixels (reference post_process.cuh:88-93)
__constant__ static const float kGauss9[9] = {0.02907f, 0.06794f, 0.12458f, 0.17925f, 0.20236f,
                                              0.17925f, 0.12458f, 0.06794f, 0.02907f};
