// ---------------------------------------------------------------------------
// bh_sg_infer.h -- launch interface of the fused surrogate inference kernel
// (bh_sg_infer.cu) and of the per-frame held-out comparison.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_runtime.h>
#include "bh_surrogate.h"
#include "bh_trace_params.h"

constexpr int kCritBins = 512;

// Frame mode: pixel k of the W x H frame is ray k.  Surrogate-resolved pixels
// are written to the accumulation buffer (tp.out); RK4 pixels (disk class,
// low probability or confidence, within critBand of the critical curve, and
// the held-out sample) are appended to `list`.
struct SgFrame
{
    TraceParams tp;
    float aN, qN, rN, iN;           // normalised scene inputs
    float crit[kCritBins];          // critical screen radius (tan units) per polar angle bin
    float critBand;                 // relative half-width of the RK4 band around it
    float minProb, minConf;         // class probability / confidence needed to keep a pixel
    unsigned* list;                 // RK4 pixel list, in 32-entry groups (BH_PIX_SKIP pads a group)
    unsigned* listCount;            // entries of the list (padding included)
    unsigned* traced;               // pixels on the list
    unsigned* heldPix;              // held-out sample: pixel and surrogate HDR
    float4* heldPred;
    unsigned* heldCount;
    unsigned heldCap;
    int heldStride;                 // 1 in heldStride surrogate pixels is held out (0: none)
    unsigned frameSeed;
    // cell-gate mode (anchored frames): ray k is pixel evalPix[k]; instead of deciding the
    // pixel, the kernel writes the probabilities of "escaped without the disk" and of
    // "captured without the disk" to gateOut[k]
    const unsigned* evalPix;
    float2* gateOut;
};

struct SgInferArgs
{
    const void* Whidden;            // BF16 4 x 256 x 256 (out x in), stacked
    const void* Whead;              // BF16 16 x 256
    const float* bias;              // 4 x 256 + 16 (packed)
    const float* rawIn;             // raw mode: n x 8 inputs
    float* rawOut;                  // raw mode: n x 16 head outputs
    unsigned n;                     // rays
    unsigned* err;                  // device error word
};

// frame == nullptr: raw mode (rawIn -> rawOut)
cudaError_t sg_infer_launch(const SgInferArgs& a, const SgFrame* frame, cudaStream_t s);

// Anchored surrogate frame (bh_sg_anchor.cu).  The anchors are the pixels
// (S ax, S ay), ax < nx = (W - 1) / S + 1, ay < ny = (H - 1) / S + 1, traced
// by RK4 into `anchors` (BH_OUT_ANCHOR records, row-major).  The resolve
// pass writes every anchor's HDR and every pixel it can interpolate to the
// accumulation buffer (tp.out), appends the pixels to trace to `list` in
// whole 8x4 tiles, and records the held-out sample in heldPix.  Pixels whose
// sky needs the sampled flatness test (a star may lie within reach of the
// bound) are deferred to a compact buffer and tested by a second pass with
// full warps, which resolves them or appends them to the list one by one.
struct SgAnchorFrame
{
    TraceParams tp;
    const BHAnchor* anchors;        // row-major: anchor (ax, ay) at ay * nx + ax
    const unsigned* blockOrder;     // null, or resolve block k -> 32 x 8 pixel block (row-major index)
    int S, nx, ny;
    const float2* cellGate;         // null, or per cell (nx - 1) x (ny - 1): (P(sky), P(shadow))
    float minProb;                  // cell gate: probability of the cell's class needed at its centre
    float epsMax;                   // largest interpolation error bound (rad) a pixel may have
    float maxStep;                  // sensitivity bar: display-value change (byte units) within the bound
    unsigned* list;
    unsigned* listCount;
    unsigned* heldPix;
    float4* heldPred;
    unsigned* heldCount;
    unsigned heldCap;
    int heldStride;
    unsigned frameSeed;
    float4* sampleDir;              // deferred pixels: (interpolated direction, error bound)
    unsigned* samplePix;
    unsigned* sampleCount;          // deferred pixels claimed (beyond sampleCap, which the host sizes
                                    // to the whole frame: traced instead)
    unsigned sampleCap;
    unsigned* stats;                // [0] interpolated, [1] rejected by the anchors / cell gate,
                                    // [2] by the error bound, [3] by the sky sensitivity,
                                    // [4] pixels on the list (the list itself is padded to tiles;
                                    // held-out pixels are not on it), [7] incomplete anchors
};

cudaError_t sg_anchor_resolve(const SgAnchorFrame& F, cudaStream_t s);

// Appends the held-out sample (heldPix[0, min(*heldCount, heldCap))) to the RK4
// list after its *listCount entries and writes the total length to *total, so
// one tracer launch traces both: the sampled pixels fill the end of the launch
// instead of each claiming a tracing warp in its own tile.
cudaError_t sg_append_held(unsigned* list, const unsigned* listCount, const unsigned* heldPix,
                           const unsigned* heldCount, unsigned heldCap, unsigned* total, cudaStream_t s);

// Held-out comparison after the RK4 pass: stats[0] += pixels compared,
// stats[1] += pixels whose RGBA8 (exposure, no bloom) differs by more than
// 1 LSB, stats[2] = max |HDR difference| (float bits), stats[3] += pixels whose
// HDR differs by more than 1e-3 relative (floor 1e-3).
cudaError_t sg_held_compare(const float4* accum, const unsigned* heldPix, const float4* heldPred,
                            const unsigned* heldCount, unsigned heldCap, const TraceParams& tp, unsigned* stats,
                            cudaStream_t s);
