// ---------------------------------------------------------------------------
// bh_sg_train.cu -- training of the lensing surrogate on the GPU: the
// RK4-traced ray set, the forward and backward passes (tensor-core GEMMs of
// bh_gemm.cu plus the element-wise kernels below) and Adam.
//
// Batch of n rays, layer l = 0..3 hidden, 4 = head:
//   X0 = features(inputs)                          BF16 n x 256
//   Z_l = X_l W_l^T + b_l,  X_{l+1} = gelu(Z_l)     FP32 / BF16
//   Y = X4 Wh^T + bh                               FP32 n x 16
//   dY = d loss / dY (batch mean)                  BF16 n x 64 (cols >= 16 zero)
//   dW_l = dZ_l^T X_l,  db_l = sum_rows dZ_l,  dX_l = dZ_l W_l
//   dZ_l = dX_{l+1} * gelu'(Z_l)
// The GEMMs take K-major operands, so the weight-gradient products read the
// transposes of dZ_l and X_l (transpose kernels) and dX_l reads W_l^T (kept
// next to W_l after every update).
// No counterpart in the reference (it has no learned component).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_bf16.h>
#include "bh_integrate.cuh"
#include "bh_launch.h"
#include "bh_sg_net.cuh"
#include "bh_sg_train.h"
#include "bh_surrogate.h"

using namespace bhsg;

namespace {

// ---- element-wise kernels -------------------------------------------------------

__global__ void feat_kernel(const float* __restrict__ in, uint4* __restrict__ X, int n)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * 32) return;
    const long long row = t >> 5;
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[k] = __ldg(in + row * 8 + k);
    X[t] = sg_feature_chunk(x, (int)(t & 31));
}

__global__ void act_kernel(const float2* __restrict__ Z, __nv_bfloat162* __restrict__ X, long long pairs)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= pairs) return;
    const float2 z = Z[i];
    X[i] = gelu2_half(__floats2bfloat162_rn(0.5f * z.x, 0.5f * z.y));   // = gelu2 of bf16(z), exactly
}

// dZ = dX * gelu'(bf16(Z)) for 64 rows per block, thread = column; column sums -> db
__global__ void act_back_kernel(const float* __restrict__ Z, const float* __restrict__ dX,
                                __nv_bfloat16* __restrict__ dZ, float* __restrict__ db, int n)
{
    const int c = threadIdx.x;
    const int r0 = blockIdx.x * 64, r1 = min(r0 + 64, n);
    float s = 0.f;
    for (int r = r0; r < r1; ++r)
    {
        const size_t i = (size_t)r * kWidth + c;
        const float z = __bfloat162float(__float2bfloat16_rn(Z[i]));
        const float g = dX[i] * gelu_grad(z);
        dZ[i] = __float2bfloat16_rn(g);
        s += g;
    }
    atomicAdd(db + c, s);
}

// out[cols x rows] = in[rows x cols]^T, BF16, rows and cols multiples of 32
__global__ void transpose_kernel(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, int rows,
                                 int cols)
{
    __shared__ __nv_bfloat16 tile[32][34];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;   // bx: column block, by: row block
    const int tx = threadIdx.x, ty = threadIdx.y;           // 32 x 8
    for (int k = ty; k < 32; k += 8) tile[k][tx] = in[(size_t)(by + k) * cols + bx + tx];
    __syncthreads();
    for (int k = ty; k < 32; k += 8) out[(size_t)(bx + k) * rows + by + tx] = tile[tx][k];
}

struct LossWeights
{
    float esc, diskR, diskG, conf, escTol;
};

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per-ray loss terms and dY (scaled by 1/n); loss[0..4] += CE, escape, disk r,
// disk g, confidence (sums); dbh += column sums of dY.
__global__ void loss_kernel(const float* __restrict__ Y, const float* __restrict__ in, const float* __restrict__ tgt,
                            __nv_bfloat16* __restrict__ dY, float* __restrict__ dbh, float* __restrict__ loss, int n,
                            LossWeights w)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    float g[kOut], l[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < kOut; ++k) g[k] = 0.f;
    if (row < n)
    {
        float y[kOut];
#pragma unroll
        for (int k = 0; k < kOut; ++k) y[k] = Y[(size_t)row * kOut + k];
        const float* t = tgt + (size_t)row * 8;
        const int cls = (int)t[0];
        const float m = fmaxf(y[0], fmaxf(y[1], y[2]));
        const float e0 = expf(y[0] - m), e1 = expf(y[1] - m), e2 = expf(y[2] - m), se = e0 + e1 + e2;
        const float p[3] = {e0 / se, e1 / se, e2 / se};
        l[0] = -logf(fmaxf(p[cls], 1e-30f));
        for (int k = 0; k < 3; ++k) g[k] = p[k] - (k == cls ? 1.f : 0.f);
        float errE = 0.f;
        if (cls == kClsEscaped)
        {
            float r[3];
            for (int k = 0; k < 3; ++k) r[k] = in[(size_t)row * 8 + k] + y[kOEsc + k] - t[1 + k];
            errE = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            l[1] = w.esc * errE * errE;
            for (int k = 0; k < 3; ++k) g[kOEsc + k] = 2.f * w.esc * r[k];
        }
        if (t[6] > 0.5f)
        {
            const float dr = y[kODiskR] - t[4], dg = y[kODiskG] - t[5];
            l[2] = w.diskR * dr * dr;
            l[3] = w.diskG * dg * dg;
            g[kODiskR] = 2.f * w.diskR * dr;
            g[kODiskG] = 2.f * w.diskG * dg;
        }
        const int pred = (p[0] >= p[1] && p[0] >= p[2]) ? 0 : (p[1] >= p[2] ? 1 : 2);
        const float good = (pred == cls && (cls != kClsEscaped || errE < w.escTol)) ? 1.f : 0.f;
        const float s = 1.f / (1.f + expf(-y[kOConf]));
        l[4] = -w.conf * (good * logf(fmaxf(s, 1e-30f)) + (1.f - good) * logf(fmaxf(1.f - s, 1e-30f)));
        g[kOConf] = w.conf * (s - good);
        const float inv = 1.f / (float)n;
        __nv_bfloat16* d = dY + (size_t)row * kOutPad;
#pragma unroll
        for (int k = 0; k < kOut; ++k)
        {
            g[k] *= inv;
            d[k] = __float2bfloat16_rn(g[k]);
        }
        for (int k = kOut; k < kOutPad; ++k) d[k] = __float2bfloat16_rn(0.f);
    }
#pragma unroll
    for (int k = 0; k < kOut; ++k)
    {
        const float s = warp_sum(g[k]);
        if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(dbh + k, s);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k)
    {
        const float s = warp_sum(l[k]);
        if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(loss + k, s);
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int count, float lr, float b1, float b2, float eps, float c1,
                            float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// BF16 weights W_l (out x in) and their transposes (head transpose padded to 64 columns)
__global__ void pack_kernel(const float* __restrict__ params, __nv_bfloat16* __restrict__ W,
                            __nv_bfloat16* __restrict__ Wt, float* __restrict__ biasPacked)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int kHid = kHidden * kWidth * kWidth;
    if (i < kHid)
    {
        const int l = i / (kWidth * kWidth), r = (i / kWidth) % kWidth, c = i % kWidth;
        const float w = params[SgLayout::w(l) + r * kWidth + c];
        W[i] = __float2bfloat16_rn(w);
        Wt[(size_t)l * kWidth * kWidth + c * kWidth + r] = __float2bfloat16_rn(w);
    }
    else if (i < kHid + kWidth * kOutPad)
    {
        const int j = i - kHid, c = j / kOutPad, o = j % kOutPad;   // Wht: 256 x 64
        const float w = o < kOut ? params[SgLayout::w(kHidden) + o * kWidth + c] : 0.f;
        Wt[kHid + j] = __float2bfloat16_rn(w);
        if (o < kOut) W[kHid + o * kWidth + c] = __float2bfloat16_rn(w);
    }
    else if (i < kHid + kWidth * kOutPad + kHidden * kWidth + kOut)
    {   // biases of all layers, contiguous
        const int j = i - kHid - kWidth * kOutPad, l = j / kWidth;
        biasPacked[j] = params[SgLayout::b(l) + (l < kHidden ? j % kWidth : j - kHidden * kWidth)];
    }
}

// batch rows gathered from the ray set at hashed indices
__global__ void gather_kernel(const float4* __restrict__ dsIn, const float4* __restrict__ dsTgt, long long N,
                              unsigned seed, float4* __restrict__ in, float4* __restrict__ tgt, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    unsigned h = (unsigned)k * 0x9E3779B1u ^ seed;
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    unsigned h2 = h * 0x2C1B3C6Du + 0x297A2D39u;
    h2 ^= h2 >> 15;
    const long long idx = (long long)((((unsigned long long)h << 32) | h2) % (unsigned long long)N);
    in[2 * k] = dsIn[2 * idx]; in[2 * k + 1] = dsIn[2 * idx + 1];
    tgt[2 * k] = dsTgt[2 * idx]; tgt[2 * k + 1] = dsTgt[2 * idx + 1];
}

// ---- the RK4-traced ray set ----------------------------------------------------------
__device__ __forceinline__ unsigned hash_u32(unsigned x)
{
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

struct ViewInputs
{
    float aN, qN, rN, iN;
};

__global__ void rays_kernel(const __grid_constant__ TraceParams P, ViewInputs vi, unsigned seed, float3* __restrict__ dirs,
                            float* __restrict__ in, int R)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const unsigned h1 = hash_u32(seed ^ hash_u32((unsigned)k * 2u + 1u));
    const unsigned h2 = hash_u32(h1 + 0x9e3779b9u);
    const float fx = (float)(h1 >> 8) * (1.f / 16777216.f), fy = (float)(h2 >> 8) * (1.f / 16777216.f);
    const f3 d = camera_ray(P, fx, fy);
    dirs[k] = make_float3(d.x, d.y, d.z);
    float* x = in + (size_t)k * 8;
    x[0] = d.x * P.camRight.x + d.y * P.camRight.y + d.z * P.camRight.z;
    x[1] = d.x * P.camUp.x + d.y * P.camUp.y + d.z * P.camUp.z;
    x[2] = d.x * P.camFwd.x + d.y * P.camFwd.y + d.z * P.camFwd.z;
    x[3] = vi.aN; x[4] = vi.qN; x[5] = vi.rN; x[6] = vi.iN; x[7] = 0.f;
}

__global__ void targets_kernel(const BHProbe* __restrict__ rec, const __grid_constant__ TraceParams P,
                               float* __restrict__ tgt, int R)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const BHProbe& o = rec[k];
    const bool disk = (o.accum[0] + o.accum[1] + o.accum[2]) > 0.f || o.trans < 1.f;
    const int cls = disk ? kClsDisk : (o.outcome == 1 ? kClsEscaped : kClsCaptured);
    float* t = tgt + (size_t)k * 8;
    t[0] = (float)cls;
    const float ex = o.escDir[0], ey = o.escDir[1], ez = o.escDir[2];
    const float inv = rsqrtf(fmaxf(ex * ex + ey * ey + ez * ez, 1e-30f));
    t[1] = (ex * P.camRight.x + ey * P.camRight.y + ez * P.camRight.z) * inv;
    t[2] = (ex * P.camUp.x + ey * P.camUp.y + ez * P.camUp.z) * inv;
    t[3] = (ex * P.camFwd.x + ey * P.camFwd.y + ez * P.camFwd.z) * inv;
    const bool hit = o.diskR > 0.f;
    t[4] = hit ? o.diskR * 0.125f : 0.f;
    t[5] = hit ? logf(fmaxf(o.diskG, 1e-6f)) : 0.f;
    t[6] = hit ? 1.f : 0.f;
    t[7] = 0.f;
}

inline unsigned blocksFor(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
cudaError_t sg_features(const float* in, void* X0, int n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    feat_kernel<<<blocksFor((long long)n * 32, 256), 256, 0, s>>>(in, reinterpret_cast<uint4*>(X0), n);
    return cudaGetLastError();
}

cudaError_t sg_pack_weights(SgState& S, cudaStream_t s)
{
    const int count = kHidden * kWidth * kWidth + kWidth * kOutPad + kHidden * kWidth + kOut;
    pack_kernel<<<blocksFor(count, 256), 256, 0, s>>>(S.params, S.W, S.Wt, S.biasPacked);
    return cudaGetLastError();
}

cudaError_t sg_reserve(SgState& S, int n, cudaStream_t s)
{
    if (n <= S.cap) return cudaSuccess;
    sg_free_batch(S);
    const size_t nw = (size_t)n * kWidth;
    cudaError_t e = cudaSuccess;
    auto take = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(p), bytes); };
    for (int l = 0; l <= kHidden; ++l) take((void**)&S.X[l], nw * 2);
    for (int l = 0; l < kHidden; ++l) take((void**)&S.Z[l], nw * 4);
    take((void**)&S.Y, (size_t)n * kOut * 4);
    take((void**)&S.dY, (size_t)n * kOutPad * 2);
    take((void**)&S.dYt, (size_t)128 * n * 2);
    take((void**)&S.dX, nw * 4);
    take((void**)&S.dZ, nw * 2);
    take((void**)&S.T0, nw * 2);
    take((void**)&S.T1, nw * 2);
    take((void**)&S.headTmp, (size_t)128 * kWidth * 4);
    if (e == cudaSuccess) e = cudaMemsetAsync(S.dYt, 0, (size_t)128 * n * 2, s);   // ordered with its users
    if (e != cudaSuccess) { sg_free_batch(S); return e; }
    S.cap = n;
    return cudaSuccess;
}

void sg_free_batch(SgState& S)
{
    void* ps[] = {S.X[0], S.X[1], S.X[2], S.X[3], S.X[4], S.Z[0], S.Z[1], S.Z[2], S.Z[3], S.Y, S.dY, S.dYt, S.dX,
                  S.dZ, S.T0, S.T1, S.headTmp};
    for (void* p : ps)
        if (p) cudaFree(p);
    for (int l = 0; l <= kHidden; ++l) S.X[l] = nullptr;
    for (int l = 0; l < kHidden; ++l) S.Z[l] = nullptr;
    S.Y = nullptr; S.dY = nullptr; S.dYt = nullptr; S.dX = nullptr; S.dZ = nullptr;
    S.T0 = nullptr; S.T1 = nullptr; S.headTmp = nullptr;
    S.cap = 0;
}

static cudaError_t transpose(const void* in, void* out, int rows, int cols, cudaStream_t s)
{
    dim3 grid(cols / 32, rows / 32), block(32, 8);
    transpose_kernel<<<grid, block, 0, s>>>(reinterpret_cast<const __nv_bfloat16*>(in),
                                            reinterpret_cast<__nv_bfloat16*>(out), rows, cols);
    return cudaGetLastError();
}

// forward pass through the GEMM path (training form): Y = net(in)
cudaError_t sg_forward_train(SgState& S, const float* in, int n, cudaStream_t s)
{
    cudaError_t e = sg_reserve(S, n, s);
    if (e == cudaSuccess) e = sg_features(in, S.X[0], n, s);
    const size_t ww = (size_t)kWidth * kWidth;
    for (int l = 0; l < kHidden && e == cudaSuccess; ++l)
    {
        e = bh_gemm_bf16(S.X[l], kWidth, S.W + l * ww, kWidth, S.Z[l], kWidth, n, kWidth, kWidth, 1, false,
                         S.params + SgLayout::b(l), S.err, s);
        if (e == cudaSuccess)
        {
            const long long pairs = (long long)n * kWidth / 2;
            act_kernel<<<blocksFor(pairs, 256), 256, 0, s>>>(reinterpret_cast<const float2*>(S.Z[l]),
                                                             reinterpret_cast<__nv_bfloat162*>(S.X[l + 1]), pairs);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess)
        e = bh_gemm_bf16(S.X[kHidden], kWidth, S.W + kHidden * ww, kWidth, S.Y, kOut, n, kOut, kWidth, 1, false,
                         S.params + SgLayout::b(kHidden), S.err, s);
    return e;
}

// forward + loss + backward; gradients (batch mean) in S.grads, loss sums in S.loss
cudaError_t sg_gradients(SgState& S, const float* in, const float* tgt, int n, cudaStream_t s)
{
    if (n <= 0 || n % 128) return cudaErrorInvalidValue;
    cudaError_t e = sg_forward_train(S, in, n, s);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(S.grads, 0, SgLayout::count() * sizeof(float), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(S.loss, 0, 8 * sizeof(float), s)) != cudaSuccess) return e;
    LossWeights w{S.wEsc, S.wDiskR, S.wDiskG, S.wConf, S.escTol};
    loss_kernel<<<blocksFor(n, 128), 128, 0, s>>>(S.Y, in, tgt, reinterpret_cast<__nv_bfloat16*>(S.dY), S.grads + SgLayout::b(kHidden), S.loss, n, w);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    const int splits = std::max(1, std::min(64, n / 512));   // split-K over the batch for the weight gradients
    const int sp = ((n / 64) % splits == 0) ? splits : 1;
    const size_t ww = (size_t)kWidth * kWidth;
    // head: dWh = dY^T X4 (through a 128-row padded dY^T), dX4 = dY Wh
    if ((e = transpose(S.dY, S.dYt, n, kOutPad, s)) != cudaSuccess) return e;
    if ((e = transpose(S.X[kHidden], S.T1, n, kWidth, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(S.headTmp, 0, (size_t)128 * kWidth * 4, s)) != cudaSuccess) return e;
    if ((e = bh_gemm_bf16(S.dYt, n, S.T1, n, S.headTmp, kWidth, 128, kWidth, n, sp, true, nullptr, S.err, s)))
        return e;
    if ((e = cudaMemcpyAsync(S.grads + SgLayout::w(kHidden), S.headTmp, (size_t)kOut * kWidth * 4,
                             cudaMemcpyDeviceToDevice, s)))
        return e;
    if ((e = bh_gemm_bf16(S.dY, kOutPad, S.Wt + kHidden * ww, kOutPad, S.dX, kWidth, n, kWidth, kOutPad, 1, false,
                          nullptr, S.err, s)))
        return e;
    for (int l = kHidden - 1; l >= 0; --l)
    {
        act_back_kernel<<<blocksFor(n, 64), kWidth, 0, s>>>(S.Z[l], S.dX, reinterpret_cast<__nv_bfloat16*>(S.dZ),
                                                            S.grads + SgLayout::b(l), n);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = transpose(S.dZ, S.T0, n, kWidth, s)) != cudaSuccess) return e;
        if ((e = transpose(S.X[l], S.T1, n, kWidth, s)) != cudaSuccess) return e;
        if ((e = bh_gemm_bf16(S.T0, n, S.T1, n, S.grads + SgLayout::w(l), kWidth, kWidth, kWidth, n, sp, true,
                              nullptr, S.err, s)))
            return e;
        if (l > 0 && (e = bh_gemm_bf16(S.dZ, kWidth, S.Wt + l * ww, kWidth, S.dX, kWidth, n, kWidth, kWidth, 1,
                                       false, nullptr, S.err, s)))
            return e;
    }
    return cudaSuccess;
}

cudaError_t sg_adam(SgState& S, float lr, cudaStream_t s)
{
    ++S.step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)S.step)), c2 = 1.f / (1.f - std::pow(b2, (float)S.step));
    const int count = SgLayout::count();
    adam_kernel<<<blocksFor(count, 256), 256, 0, s>>>(S.params, S.grads, S.adamM, S.adamV, count, lr, b1, b2, 1e-8f,
                                                       c1, c2);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? sg_pack_weights(S, s) : e;
}

cudaError_t sg_make_rays(const TraceParams& P, float aN, float qN, float rN, float iN, unsigned seed, float3* dirs,
                         float* in, int R, cudaStream_t s)
{
    rays_kernel<<<blocksFor(R, 256), 256, 0, s>>>(P, ViewInputs{aN, qN, rN, iN}, seed, dirs, in, R);
    return cudaGetLastError();
}

cudaError_t sg_make_targets(const void* rec, const TraceParams& P, float* tgt, int R, cudaStream_t s)
{
    targets_kernel<<<blocksFor(R, 256), 256, 0, s>>>(reinterpret_cast<const BHProbe*>(rec), P, tgt, R);
    return cudaGetLastError();
}

cudaError_t sg_gather(const SgState& S, unsigned seed, float* in, float* tgt, int n, cudaStream_t s)
{
    if (S.dsN <= 0) return cudaErrorInvalidValue;
    gather_kernel<<<blocksFor(n, 256), 256, 0, s>>>(reinterpret_cast<const float4*>(S.dsIn),
                                                    reinterpret_cast<const float4*>(S.dsTgt), S.dsN, seed,
                                                    reinterpret_cast<float4*>(in), reinterpret_cast<float4*>(tgt), n);
    return cudaGetLastError();
}
