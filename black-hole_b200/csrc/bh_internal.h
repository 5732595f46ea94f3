#pragma once
// ---------------------------------------------------------------------------
// bh_internal.h -- declarations shared by the host C++ and the CUDA sources
// of libbh.so (not part of the public C-ABI in include/).
// ---------------------------------------------------------------------------
#include <cuda_runtime_api.h>
#include <vector_types.h>
#include "bh_trace_params.h"

// Tracing CTAs: 128 threads, except the FP32 Kerr-family render kernels (160
// threads, 5 CTAs of 80 registers = 25 warps per SM, where 128-thread CTAs fit
// only 6 x 4 = 24); BH_TRACE_BLOCK_MAX sizes per-thread shared arrays.
#define BH_TRACE_BLOCK 128
#define BH_TRACE_BLOCK_KERR 160
#define BH_TRACE_BLOCK_MAX 160
// resident CTAs per SM the spherical FP32 tracing kernels are register-budgeted for
// (65536 / (128 * 7) -> 72 registers per thread, 28 warps per SM)
#ifndef BH_TRACE_MIN_BLOCKS
#define BH_TRACE_MIN_BLOCKS 7
#endif

struct PostConsts
{
    float exposure, bloomStrength;
    int bloomOn, swapRB;
};

// tracing: zero the ray counter, then one persistent launch (bh_trace.cu)
cudaError_t bh_launch_trace(const TraceParams& P, int precision, bool stats, int blocksPerSm,
                            cudaStream_t stream);

// batched views of one metric family (`kerr`: Kerr / Kerr-Newman, else the
// spherical metrics): zero the counter, then one persistent launch over all
// the views' tiles (bh_trace.cu); `views` and `tileBase` (n + 1 prefix sums of
// tiles) are device tables
cudaError_t bh_launch_batch(bool kerr, const TraceParams* views, const unsigned* tileBase, int n,
                            unsigned totalTiles, unsigned* counter, int blocksPerSm, cudaStream_t stream);

// resident CTAs per SM of the FP32 tracing kernel of a model's family
cudaError_t bh_trace_max_blocks(int model, int* out);

// cudaMalloc, counted per device for bhLibraryDeviceBytes (bh_api.cpp)
cudaError_t bh_device_alloc(void** p, size_t bytes);

// bloom + tonemap of an accumulation buffer (bh_post.cu); `hblur` receives the
// horizontally blurred half-resolution image ((W+1)/2 x (H+1)/2 float4) and,
// when not null, `vblur` the finished (vertically blurred) bloom of the same size
cudaError_t bh_launch_post(uchar4* out, const float4* accum, float4* hblur, float4* vblur, int W, int H,
                           const PostConsts& pc, cudaStream_t stream);

// frame constants of a sanitised view for the given output (bh_api.cpp), and
// the CTAs per SM the view's metric family is tuned for
struct RenderParams;
TraceParams bh_frame_params(const RenderParams& P, int outMode, void* out);
int bh_family_blocks(const RenderParams& P);
// the library's per-device work counter (allocated on first use)
cudaError_t bh_device_counter(unsigned** out);

// camera-frame constants of t.camPos / t.M / t.a / t.Q in FP32 and FP64 (bh_camera.cpp)
void bh_fill_camera_frames(TraceParams& t);

// FP32 FMA throughput probe (bh_peak.cu)
double bh_measure_fp32_peak();
