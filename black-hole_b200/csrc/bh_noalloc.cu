// ---------------------------------------------------------------------------
// bh_noalloc.cu -- the full frame pipeline without any device allocation.
//
// launchRenderPipeline needs two pieces of scratch memory besides the caller's
// buffers: the work counter the persistent tracing kernel draws rays from, and
// a tile-order table, both allocated by the library on first use.  Some
// callers cannot let a library allocate: a plugin whose host framework owns
// every byte of device memory and hands out only the buffers it manages, or a
// real-time frame loop that must never stall on the allocator (cudaMalloc can
// synchronise the device).  For them
// this file holds all the scratch in one file-scope __device__ array of fixed
// size, loaded with the module; the entry point below allocates nothing.
//
// Limits and sharing (also stated in include/bh_launch.h):
//   * scratch = 256 bytes (work counter) + BH_NOALLOC_MAX_HALF_PIXELS float4
//     for the horizontally blurred half-resolution bloom image, so with bloom
//     on, frames up to (W+1)/2 * (H+1)/2 <= 524288 half-res pixels (1920x1080,
//     2048x1024) are accepted and larger ones rejected;
//   * every call on a device uses the same array, which keeps the previous
//     call's contents (the counter is cleared on the stream before each
//     trace), so calls that overlap on the GPU race: serialise them;
//   * the array belongs to this library's module: under lazy module loading
//     (the CUDA default) the module, and with it the array, is loaded on a
//     device at the first call there; later calls allocate nothing;
//   * tiles are traced in row-major order (no order table); the image is the
//     same as launchRenderPipeline's.
// ---------------------------------------------------------------------------
#include <cuda_runtime.h>
#include "bh_launch.h"
#include "bh_internal.h"

namespace {

constexpr size_t kHeaderBytes = 256;
constexpr size_t kScratchBytes = kHeaderBytes + (size_t)BH_NOALLOC_MAX_HALF_PIXELS * sizeof(float4);

// Every GPU that loads libbh.so holds this array until the process exits.
static __device__ __align__(256) unsigned char gNoAllocScratch[kScratchBytes];

// Device address of the array in the current device's context (host code
// cannot use the symbol itself: on the host it names a stand-in, not device
// memory).  Looked up on every call, so a device reset or another context
// never leaves a stale address; the lookup allocates nothing once the module
// is loaded.
cudaError_t scratch_address(unsigned char** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, gNoAllocScratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

}  // namespace

extern "C" cudaError_t bhRenderPipelineNoAlloc(uchar4* out, float4* accum, const RenderParams& p,
                                               cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    if (!out || !accum) return cudaErrorInvalidValue;
    const size_t half = (size_t)((P.width + 1) / 2) * (size_t)((P.height + 1) / 2);
    if (P.bloomEnabled && half > (size_t)BH_NOALLOC_MAX_HALF_PIXELS) return cudaErrorInvalidValue;

    unsigned char* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) return e;

    TraceParams t = bh_frame_params(P, BH_OUT_ACCUM, accum);
    t.counter = reinterpret_cast<unsigned*>(base);
    t.tileOrder = nullptr;
    e = bh_launch_trace(t, BH_PREC_FP32, false, bh_family_blocks(P), stream);
    if (e != cudaSuccess) return e;
    PostConsts pc{P.exposure, P.bloomStrength, P.bloomEnabled ? 1 : 0, P.swapRB};
    return bh_launch_post(out, accum, reinterpret_cast<float4*>(base + kHeaderBytes), nullptr, P.width, P.height, pc,
                          stream);
}
