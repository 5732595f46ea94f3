// ---------------------------------------------------------------------------
// bh_post.cu -- bloom and tonemap as two HBM-streaming kernels.
//
// The reference runs four passes after tracing (downsample + bright pass,
// horizontal blur, vertical blur, composite; src/black_hole_kernel.cu:41-103),
// each a round trip through global memory.  Here:
//   bloom_h_kernel     reads the accumulation buffer once, forms the
//                      half-resolution bright pass in shared memory (with the
//                      4-pixel halo recomputed, not exchanged) and writes the
//                      horizontally blurred half-resolution image
//   composite_kernel   stages the horizontally blurred rows its tile needs in
//                      shared memory, blurs them vertically there, writes the
//                      tile's own vertically blurred half-res pixels to the
//                      caller's second bloom buffer (the reference leaves the
//                      finished bloom there), samples the result bilinearly
//                      and tonemaps the accumulation buffer to RGBA8
// Traffic per full-resolution pixel: 16 B accum read twice, 4 B half-res
// write + ~5 B half-res read, 4 B finished-bloom write, 4 B RGBA8 write
// (~49 B vs ~64 B for the reference's passes).  Clamp-to-edge addressing and the summation order of
// every tap are the reference's, in exact arithmetic.
// ---------------------------------------------------------------------------
#include "bh_post.cuh"
#include "bh_internal.h"

namespace {

constexpr int HB_TX = 128;            // half-res columns per bloom_h block
constexpr int CP_TX = 64;             // full-res tile of composite_kernel
constexpr int CP_TY = 16;
constexpr int CP_HC = CP_TX / 2 + 2;  // half-res columns the tile samples
constexpr int CP_HR = CP_TY / 2 + 2;  // half-res rows the tile samples
constexpr int CP_HH = CP_HR + 8;      // horizontally blurred rows the vertical blur reads

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// 2x2 box average of the accumulation buffer x exposure -> bright pass
// (reference black_hole_kernel.cu:41-62)
__device__ __forceinline__ f3 downsample(const float4* __restrict__ acc, int W, int H, int x, int y,
                                         float exposure)
{
    int x0 = x * 2, y0 = y * 2;
    int x1 = (x0 + 1 < W) ? x0 + 1 : x0;
    int y1 = (y0 + 1 < H) ? y0 + 1 : y0;
    float4 a = __ldg(acc + (size_t)y0 * W + x0);
    float4 b = __ldg(acc + (size_t)y0 * W + x1);
    float4 c = __ldg(acc + (size_t)y1 * W + x0);
    float4 d = __ldg(acc + (size_t)y1 * W + x1);
    f3 avg = v3(mul_x(add_x(add_x(add_x(a.x, b.x), c.x), d.x), 0.25f),
                mul_x(add_x(add_x(add_x(a.y, b.y), c.y), d.y), 0.25f),
                mul_x(add_x(add_x(add_x(a.z, b.z), c.z), d.z), 0.25f));
    return bright_pass(v3(mul_x(avg.x, exposure), mul_x(avg.y, exposure), mul_x(avg.z, exposure)));
}

__global__ void __launch_bounds__(HB_TX)
bloom_h_kernel(const float4* __restrict__ acc, float4* __restrict__ hblur, int W, int H, int bw, int bh,
               float exposure)
{
    __shared__ float s[3][HB_TX + 8];
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * HB_TX - 4;
    for (int i = threadIdx.x; i < HB_TX + 8; i += HB_TX)
    {
        f3 v = downsample(acc, W, H, clampi(x0 + i, 0, bw - 1), y, exposure);
        s[0][i] = v.x; s[1][i] = v.y; s[2][i] = v.z;
    }
    __syncthreads();
    const int x = blockIdx.x * HB_TX + threadIdx.x;
    if (x >= bw) return;
    float rx = 0.f, ry = 0.f, rz = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        const float w = kGauss9[k];
        rx = add_x(rx, mul_x(s[0][threadIdx.x + k], w));
        ry = add_x(ry, mul_x(s[1][threadIdx.x + k], w));
        rz = add_x(rz, mul_x(s[2][threadIdx.x + k], w));
    }
    hblur[(size_t)y * bw + x] = make_float4(rx, ry, rz, 1.f);
}

__global__ void __launch_bounds__(CP_TX * 4)
composite_kernel(uchar4* __restrict__ out, const float4* __restrict__ acc, const float4* __restrict__ hblur,
                 float4* __restrict__ vblur, int W, int H, int bw, int bh, PostConsts pc)
{
    __shared__ float hs[3][CP_HH][CP_HC];
    __shared__ float vs[3][CP_HR][CP_HC];
    const int X0 = blockIdx.x * CP_TX, Y0 = blockIdx.y * CP_TY;
    const int hc0 = X0 / 2 - 1, hr0 = Y0 / 2 - 1;
    const int tid = threadIdx.x;

    if (pc.bloomOn)
    {
        for (int i = tid; i < CP_HH * CP_HC; i += CP_TX * 4)
        {
            int rr = i / CP_HC, cc = i % CP_HC;
            int row = clampi(hr0 - 4 + rr, 0, bh - 1), col = clampi(hc0 + cc, 0, bw - 1);
            float4 v = __ldg(hblur + (size_t)row * bw + col);
            hs[0][rr][cc] = v.x; hs[1][rr][cc] = v.y; hs[2][rr][cc] = v.z;
        }
        __syncthreads();
        for (int i = tid; i < CP_HR * CP_HC; i += CP_TX * 4)
        {
            int rr = i / CP_HC, cc = i % CP_HC;
            int r = hr0 + rr;
            int shift = clampi(r, 0, bh - 1) - r;        // vertical blur centred on the clamped row
            int base = rr + shift;                       // hs row of tap k = -4
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
            for (int k = 0; k < 9; ++k)
            {
                const float w = kGauss9[k];
                sx = add_x(sx, mul_x(hs[0][base + k][cc], w));
                sy = add_x(sy, mul_x(hs[1][base + k][cc], w));
                sz = add_x(sz, mul_x(hs[2][base + k][cc], w));
            }
            vs[0][rr][cc] = sx; vs[1][rr][cc] = sy; vs[2][rr][cc] = sz;
            // rows 1..CP_HR-2 and columns 1..CP_HC-2 are this tile's own half-res pixels
            // (each half-res pixel belongs to exactly one tile): the reference's vertical
            // blur output, black_hole_kernel.cu:75-84
            const int c = hc0 + cc;
            if (vblur && rr >= 1 && rr <= CP_HR - 2 && cc >= 1 && cc <= CP_HC - 2 && r < bh && c < bw)
                vblur[(size_t)r * bw + c] = make_float4(sx, sy, sz, 1.f);
        }
        __syncthreads();
    }

    const int tx = tid % CP_TX;
    const int px = X0 + tx;
    if (px >= W) return;
    for (int ty = tid / CP_TX; ty < CP_TY; ty += 4)
    {
        const int py = Y0 + ty;
        if (py >= H) break;
        float4 av = __ldg(acc + (size_t)py * W + px);
        f3 bloom = v3(0.f, 0.f, 0.f);
        if (pc.bloomOn)
        {   // bilinear sample of the half-res bloom (reference post_process.cuh:106-117)
            float x = sub_x(mul_x(add_x((float)px, 0.5f), 0.5f), 0.5f);
            float y = sub_x(mul_x(add_x((float)py, 0.5f), 0.5f), 0.5f);
            int ix = (int)floorf(x), iy = (int)floorf(y);
            float fx = sub_x(x, (float)ix), fy = sub_x(y, (float)iy);
            int j = ix - hc0, i = iy - hr0;
            float r[3];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch)
            {
                float c00 = vs[ch][i][j], c10 = vs[ch][i][j + 1];
                float c01 = vs[ch][i + 1][j], c11 = vs[ch][i + 1][j + 1];
                float top = add_x(c00, mul_x(sub_x(c10, c00), fx));
                float bot = add_x(c01, mul_x(sub_x(c11, c01), fx));
                r[ch] = add_x(top, mul_x(sub_x(bot, top), fy));
            }
            bloom = v3(r[0], r[1], r[2]);
        }
        out[(size_t)py * W + px] = finalize_pixel(v3(av.x, av.y, av.z), bloom, pc, px, py);
    }
}

}  // namespace

cudaError_t bh_launch_post(uchar4* out, const float4* accum, float4* hblur, float4* vblur, int W, int H,
                           const PostConsts& pc, cudaStream_t stream)
{
    const int bw = (W + 1) / 2, bh = (H + 1) / 2;
    if (pc.bloomOn)
    {
        dim3 g((bw + HB_TX - 1) / HB_TX, bh);
        bloom_h_kernel<<<g, HB_TX, 0, stream>>>(accum, hblur, W, H, bw, bh, pc.exposure);
    }
    dim3 g2((W + CP_TX - 1) / CP_TX, (H + CP_TY - 1) / CP_TY);
    composite_kernel<<<g2, CP_TX * 4, 0, stream>>>(out, accum, hblur, pc.bloomOn ? vblur : nullptr, W, H, bw,
                                                    bh, pc);
    return cudaGetLastError();
}
