// ---------------------------------------------------------------------------
// bh_peak.cu -- measured FP32 FMA throughput of the current GPU.
//
// The tracer is FP32-bound, and no FP32 peak is published for this machine's
// clocks, so the roofline denominator is measured: every thread runs eight
// independent FMA chains (enough ILP to cover the FMA latency at full
// occupancy), the grid fills every SM, and the launch is timed with CUDA
// events after a warm-up.  FLOPs counted as 2 per FMA.  The tracer issues
// both scalar FMAs and packed FP32x2 FMAs (sm_100), so both forms are timed
// and the higher rate is the peak.
// ---------------------------------------------------------------------------
#include <cuda_runtime.h>
#include "bh_internal.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) fma_kernel(float* out, float a, float b)
{
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (float)(threadIdx.x + c) * 1e-3f;
#pragma unroll 4
    for (int i = 0; i < kIters; ++i)
    {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1234.5678f) out[blockIdx.x] = s;   // keeps the chains live
}

// the same work as packed FP32x2 FMAs (two lanes' worth of FMAs per instruction)
__global__ void __launch_bounds__(256) fma2_kernel(float* out, float a, float b)
{
    float2 x[kChains / 2];
#pragma unroll
    for (int c = 0; c < kChains / 2; ++c)
        x[c] = make_float2((float)(threadIdx.x + 2 * c) * 1e-3f, (float)(threadIdx.x + 2 * c + 1) * 1e-3f);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll 4
    for (int i = 0; i < kIters; ++i)
    {
#pragma unroll
        for (int c = 0; c < kChains / 2; ++c) x[c] = __ffma2_rn(x[c], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains / 2; ++c) s += x[c].x + x[c].y;
    if (s == 1234.5678f) out[blockIdx.x] = s;
}

template <class K>
float best_ms(K kernel, float* out, int blocks)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; ++w) kernel<<<blocks, 256>>>(out, 0.999f, 1e-4f);
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep)
    {
        cudaEventRecord(e0);
        kernel<<<blocks, 256>>>(out, 0.999f, 1e-4f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

double bh_measure_fp32_peak()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0.0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0.0;
    float* out = nullptr;
    const int blocks = sms * 8;
    if (bh_device_alloc(reinterpret_cast<void**>(&out), blocks * sizeof(float)) != cudaSuccess) return 0.0;
    const float best = fminf(best_ms(fma_kernel, out, blocks), best_ms(fma2_kernel, out, blocks));
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return 0.0;
    const double flops = 2.0 * kChains * (double)kIters * 256.0 * blocks;
    return flops / (best * 1e-3) / 1e12;
}
