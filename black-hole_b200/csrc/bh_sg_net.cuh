// ---------------------------------------------------------------------------
// bh_sg_net.cuh -- the lensing surrogate network, shared by the training
// kernels (bh_sg_train.cu) and the fused inference kernel (bh_sg_infer.cu).
//
// Inputs (7, each mapped to [-1, 1]): the ray direction in the camera basis
// (right, up, forward components), a*, q, log camera distance, inclination.
// Features (256): for every input x and band b = 0..15, sin(w_b x) and
// cos(w_b x) with w_b = pi 2^(b/2) (224), the 7 inputs themselves, 25 zeros.
// Network: 4 hidden layers 256 -> 256 with the tanh-form GELU, then a linear
// head 256 -> 16; BF16 weights and activations, FP32 accumulation.
// Head outputs: 0-2 class logits (escaped without touching the disk /
// captured without touching the disk / touched the disk); 3-5 correction to
// the camera-basis ray direction giving the escape direction; 6 disk-hit
// radius / 8; 7 log of the disk-hit redshift factor; 8 confidence logit.
// ---------------------------------------------------------------------------
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace bhsg {

constexpr int kIn = 7;          // network inputs
constexpr int kBands = 16;      // Fourier bands per input
constexpr int kWidth = 256;     // feature and hidden width
constexpr int kHidden = 4;      // hidden layers
constexpr int kOut = 16;        // head width
constexpr int kOutPad = 64;     // head width padded to one 64-column K block (backward)
constexpr int kLayers = kHidden + 1;

enum { kClsEscaped = 0, kClsCaptured = 1, kClsDisk = 2 };
enum { kOLogit0 = 0, kOEsc = 3, kODiskR = 6, kODiskG = 7, kOConf = 8 };

// input normalisation of the parameter box: a* in [-1, 1], q in [0, 0.6],
// camera distance r in [6, 60], inclination in [2, 88] degrees
struct SgNorm
{
    static __host__ __device__ float aStar(float a) { return a; }
    static __host__ __device__ float charge(float q) { return (q - 0.3f) * (1.f / 0.3f); }
    static __host__ __device__ float logR(float r)
    {
        return (logf(r) - 1.7917595f) * (2.f / 2.3025851f) - 1.f;   // ln 6, ln 10
    }
    static __host__ __device__ float incl(float deg) { return (deg - 45.f) * (1.f / 43.f); }
};

// 8 consecutive features (chunk j = 0..31) of the inputs x[0..6], packed BF16.
__device__ __forceinline__ uint4 sg_feature_chunk(const float* x, int j)
{
    float f[8];
    if (j < 28)
    {
        const int i = j >> 2, b0 = (j & 3) * 4;   // input i, bands b0 .. b0 + 3
        // bands b0 and b0 + 1 directly, b0 + 2 and b0 + 3 by angle doubling
        const float w0 = 3.14159265f * exp2f(0.5f * (float)b0);
        const float w1 = w0 * 1.41421356f;
        const float t0 = __fmul_rn(w0, x[i]), t1 = __fmul_rn(w1, x[i]);
        float s0, c0, s1, c1;   // reduced to [-pi, pi] first
        __sincosf(__fmaf_rn(-6.28318531f, rintf(__fmul_rn(t0, 0.159154943f)), t0), &s0, &c0);
        __sincosf(__fmaf_rn(-6.28318531f, rintf(__fmul_rn(t1, 0.159154943f)), t1), &s1, &c1);
        f[0] = s0; f[1] = c0; f[2] = s1; f[3] = c1;
        f[4] = 2.f * __fmul_rn(s0, c0); f[5] = __fmul_rn(c0 - s0, c0 + s0);
        f[6] = 2.f * __fmul_rn(s1, c1); f[7] = __fmul_rn(c1 - s1, c1 + s1);
    }
    else if (j == 28)
    {
#pragma unroll
        for (int k = 0; k < 7; ++k) f[k] = x[k];
        f[7] = 0.f;
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) f[k] = 0.f;
    }
    uint4 r;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(f[0], f[1]), p1 = __floats2bfloat162_rn(f[2], f[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(f[4], f[5]), p3 = __floats2bfloat162_rn(f[6], f[7]);
    r.x = *reinterpret_cast<uint32_t*>(&p0); r.y = *reinterpret_cast<uint32_t*>(&p1);
    r.z = *reinterpret_cast<uint32_t*>(&p2); r.w = *reinterpret_cast<uint32_t*>(&p3);
    return r;
}

// Band frequency of feature column k < 224 (for the CPU-side check).
__host__ __device__ inline float sg_band_w(int k)
{
    const int b = (k & 31) >> 1;
    return 3.14159265f * exp2f(0.5f * (float)b);
}

// GELU, tanh form, on two BF16 values: 0.5 x (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3))).
__device__ __forceinline__ __nv_bfloat162 gelu2(__nv_bfloat162 x)
{
    const __nv_bfloat162 c0 = __floats2bfloat162_rn(0.7978845608f, 0.7978845608f);
    const __nv_bfloat162 c1 = __floats2bfloat162_rn(0.0356774081f, 0.0356774081f);
    const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
    __nv_bfloat162 u = __hfma2(__hmul2(x, x), c1, c0);
    __nv_bfloat162 v = __hmul2(x, u);
    __nv_bfloat162 t;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(*reinterpret_cast<uint32_t*>(&t)) : "r"(*reinterpret_cast<uint32_t*>(&v)));
    __nv_bfloat162 h = __hmul2(x, half);
    return __hfma2(h, t, h);
}

// The same GELU from the halved input h = x / 2 (BF16): h + h tanh(h (2 c0 +
// 8 c1 h^2)).  Powers of two commute with BF16 rounding, so every
// intermediate is exactly twice or the same as gelu2's and the result is
// gelu2(2 h) bit for bit -- with one operation fewer per pair.
__device__ __forceinline__ __nv_bfloat162 gelu2_half(__nv_bfloat162 h)
{
    const __nv_bfloat162 k0 = __floats2bfloat162_rn(2.f * 0.7978845608f, 2.f * 0.7978845608f);
    const __nv_bfloat162 k1 = __floats2bfloat162_rn(8.f * 0.0356774081f, 8.f * 0.0356774081f);
    __nv_bfloat162 u = __hfma2(__hmul2(h, h), k1, k0);
    __nv_bfloat162 v = __hmul2(h, u);
    __nv_bfloat162 t;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(*reinterpret_cast<uint32_t*>(&t)) : "r"(*reinterpret_cast<uint32_t*>(&v)));
    return __hfma2(h, t, h);
}

// d gelu / dx of the same tanh form, in FP32, at x.
__device__ __forceinline__ float gelu_grad(float x)
{
    const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * 0.7978845608f * (1.f + 3.f * 0.044715f * x * x);
}

}  // namespace bhsg
