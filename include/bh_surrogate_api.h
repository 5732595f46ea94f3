#pragma once
/*
 * bh_surrogate_api.h -- C-ABI of the learned lensing surrogate in libbh.so
 * (an extension: the reference renderer has no learned component).
 *
 * A small MLP predicts, per pixel, the outcome class of the ray (escaped
 * without touching the disk / captured without touching the disk / touched
 * the disk), its escape direction and its disk-hit radius and redshift.  Its
 * dense layers run on the B200 tensor cores (tcgen05, BF16 operands, FP32
 * accumulation in tensor memory); it is trained on the GPU, on rays the RK4
 * tracer of this library generates, by the library's own forward and backward
 * kernels.  Pixels the network is not sure of, pixels near the critical curve
 * and disk pixels are traced by the RK4 tracer.
 *
 * Conventions as in bh_launch.h: device buffers, asynchronous on `stream`
 * unless stated, the return value is the launch status.
 */
#include <cuda_runtime_api.h>
#include "bh_render_params.h"

#ifdef __cplusplus
extern "C" {
#endif

/* C (=|+=) A . B^T (+ bias): A is M x K, B is N x K, both row-major BF16
 * (leading dimensions lda / ldb elements, multiples of 8, 16-byte-aligned
 * bases); C is M x N row-major FP32 (ldc).  K must be a multiple of 64 and
 * `splits` must divide K / 64: with splits > 1 (split-K) or accumulate != 0
 * the tile results are added to C with atomics, otherwise stored; `bias`
 * (N floats, may be null) is added once.  One 128 x min(N, 256) tile per CTA,
 * TMA-fed, tcgen05.mma into tensor memory.  Internal waits are bounded: a
 * time-out sets a flag read by bhTcErrorFlags. */
cudaError_t bhTcGemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
                     int splits, int accumulate, const float* bias, cudaStream_t stream);

/* Reads and clears the tensor-core kernels' error flags (blocking): bit 0 =
 * a bounded wait inside a kernel timed out (its results are invalid). */
cudaError_t bhTcErrorFlags(unsigned* flags);

/* Self-check of that error path: one kernel waits (bounded, limitUs
 * microseconds, 1 .. 1e6) on a barrier phase that nothing completes, so the
 * wait gives up, sets bit 0 of the flags and the kernel returns; the next
 * bhTcErrorFlags reports it.  The device stays usable. */
cudaError_t bhTcWaitProbe(int limitUs, cudaStream_t stream);

/* ---- the network -------------------------------------------------------------
 * Inputs, one row of 8 floats per ray: the unit ray direction in the camera
 * basis (right, up, forward components), a* in [-1, 1], (q - 0.3) / 0.3,
 * (ln r - ln 6) * 2 / ln 10 - 1 for camera distance r (code units), and
 * (inclination - 45 deg) / 43 deg; the 8th float is ignored.
 * Features: sin and cos of pi 2^(b/2) x for every input x and b = 0..15,
 * plus the 7 inputs, zero-padded to 256 (BF16).
 * Layers: 4 x (256 -> 256, tanh-form GELU), head 256 -> 16, BF16 weights and
 * activations, FP32 accumulation.
 * Head outputs (16 floats per ray): 0-2 class logits (0 escaped without
 * touching the disk, 1 captured without touching the disk, 2 touched the
 * disk); 3-5 added to the input direction give the camera-basis escape
 * direction; 6 disk-hit radius / 8; 7 ln of the disk-hit redshift factor;
 * 8 confidence logit; 9-15 unused.
 * Targets, one row of 8 floats per ray: class, camera-basis unit escape
 * direction (3), disk-hit radius / 8, ln redshift factor, 1 if the ray hit
 * the disk plane inside the disk else 0, unused.
 * Parameters: one FP32 vector of bhSurrogateParamCount() floats: for hidden
 * layer l = 0..3 the 256 x 256 weight (row = output unit) then 256 biases,
 * then the 16 x 256 head weight and 16 biases. */
typedef struct BHSurrogate BHSurrogate;

int bhSurrogateParamCount(void);

/* New network on the current device, Xavier-uniform weights from `seed`,
 * zero biases (blocking). */
cudaError_t bhSurrogateCreate(BHSurrogate** s, unsigned seed);
void bhSurrogateDestroy(BHSurrogate* s);

/* A second handle with the same parameters and frame settings (form, gate,
 * anchor stride and budget), its own scratch and statistics and no ray set
 * (blocking): with the source on one stream and the clone on another, two
 * frames are rendered at once (frames in flight).  Destroy it on its own. */
cudaError_t bhSurrogateClone(BHSurrogate* src, BHSurrogate** out);

/* Copy the FP32 parameter vector to / from host memory (blocking); setting
 * parameters resets the optimiser state. */
cudaError_t bhSurrogateGetParams(BHSurrogate* s, float* host);
cudaError_t bhSurrogateSetParams(BHSurrogate* s, const float* host);

/* The BF16 feature matrix (n x 256, row-major) of n input rows. */
cudaError_t bhSurrogateFeatures(const float* in, void* features, int n, cudaStream_t stream);

/* Head outputs (n x 16 floats) of n input rows.  fused != 0: the fused
 * persistent tensor-core kernel used for rendering; fused == 0: the training
 * path (one tensor-core GEMM per layer plus element-wise kernels). */
cudaError_t bhSurrogateForward(BHSurrogate* s, const float* in, float* out, int n, int fused, cudaStream_t stream);

/* Forward, loss and backward on n rays (n a multiple of 128; device inputs
 * and targets); copies the gradient of the batch-mean loss (ParamCount
 * floats) and the five batch-mean loss terms (class cross-entropy, escape
 * direction, disk radius, disk redshift, confidence) to host memory
 * (blocking; the call first waits for all work on the device, so the inputs
 * may come from any stream).  Loss weights: 100 |escape error|^2 on escaped rays, 1 on the
 * disk terms of disk-hit rays, 0.1 on the confidence cross-entropy whose
 * target is 1 when the predicted class is right and, for escaped rays, the
 * escape error is below 1e-3. */
cudaError_t bhSurrogateGradients(BHSurrogate* s, const float* in, const float* tgt, int n, float* gradsHost,
                                 float* lossHost);

/* Trace `rays` rays with the FP32 RK4 tracer of this library over `views`
 * random views of the parameter box (model uniform over the four families;
 * a* U(-0.998, 0.998) and q U(0, 0.6) with a*^2 + q^2 <= 0.98 by rejection,
 * zeroed where the family has no spin / charge; camera distance U(6, 60);
 * inclination U(2, 88) deg; azimuth U(0, 360) deg; vertical FOV U(30, 90)
 * deg, 16:9; disk on; balanced preset), directions uniform over each view's
 * screen, all from `seed`; the ray set (inputs and targets) stays in device
 * memory (blocking). */
cudaError_t bhSurrogateGenerate(BHSurrogate* s, long long rays, int views, unsigned seed);

/* Device pointers to the current ray set (rows of 8 floats) and its size. */
cudaError_t bhSurrogateDataset(BHSurrogate* s, const float** in, const float** tgt, long long* n);

/* Copy rows first .. first + count - 1 of the ray set to host memory (either
 * pointer may be null; blocking). */
cudaError_t bhSurrogateDatasetCopy(BHSurrogate* s, float* in, float* tgt, long long first, long long count);

/* `steps` Adam steps (beta 0.9 / 0.999) on batches of `batch` rays (a
 * multiple of 128) drawn from the ray set by a hash of (seed, step); the
 * learning rate decays from lr to lr / 20 on a cosine.  lossHistory (may be
 * null) receives 5 batch-mean loss terms per step (blocking). */
cudaError_t bhSurrogateTrain(BHSurrogate* s, int steps, int batch, float lr, unsigned seed, float* lossHistory);

/* Render one frame with the surrogate: same buffers and result layout as
 * launchRenderPipeline.  Wherever the network is evaluated (the network
 * form, the anchored form's cell gate) it requires an orbit camera (looking at
 * the hole, no roll: camRight.y == 0); the anchored form without the cell gate
 * takes any camera.  The network form requires accumMode 0; the anchored form
 * also accumulates (modes 1 and 2 blend each pixel's sample as the tracer
 * does, with the same sub-pixel jitter; the held-out sample is then off).
 * Two forms (bhSurrogateSetAnchors):
 *  - anchored (the default, anchor stride 8): the FP32 RK4 tracer traces one
 *    pixel in stride x stride (the anchors); a pixel between anchors takes the
 *    bicubic interpolation of the 4 x 4 surrounding anchors' escape directions
 *    when all 16 escaped without touching the disk, the network gives its cell
 *    centre a probability >= minProb of escaping without the disk, the
 *    interpolation error bound is <= epsMax and the sky is flat within that
 *    bound (display values within maxStep of a byte step, below the bloom
 *    threshold); a pixel whose 16 anchors were all captured without the disk
 *    (and whose cell centre the network calls captured) is black; every other
 *    pixel is traced.  The anchors are traced with a step budget
 *    (bhSurrogateSetAnchorSteps); an anchor that spends it is traced in full
 *    with the rest, and no pixel interpolates from it;
 *  - network (stride 0): the fused kernel resolves the pixels it is sure of
 *    from its own escape direction (escaped or captured without the disk,
 *    class probability and confidence >= 0.95, farther than 2 % from the
 *    critical curve, which is found by RK4 bisection once per metric, camera
 *    distance, inclination and field of view and cached -- that first call
 *    blocks); the rest go through the RK4 tracer.
 * In both forms a held-out sample of 1 in 256 of the resolved pixels is also
 * traced and compared, then bloom and tonemap run.  The first anchored frame
 * of a handle at a size and stride builds its tables (a blocking upload that
 * waits for all work on the device).  A handle's scratch is its own: two
 * handles may render on two streams at once (two frames in flight); one
 * handle must not render on two streams at once. */
cudaError_t bhSurrogateRender(BHSurrogate* s, uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                              const RenderParams* p, cudaStream_t stream);

/* Acceptance gate of bhSurrogateRender (defaults 0.95, 0.95, 0.02, 256): a
 * pixel is resolved by the network only if its class probability is at least
 * minProb, its confidence at least minConf and it lies farther than
 * critBand (relative) from the critical curve; 1 in heldStride resolved
 * pixels is also traced by RK4 and compared (0: none).  Lower thresholds trade
 * accuracy for speed; heldStride 1 compares every resolved pixel. */
cudaError_t bhSurrogateSetGate(BHSurrogate* s, float minProb, float minConf, float critBand, int heldStride);

/* Form of bhSurrogateRender (defaults 8, 1, 1e-4, 0.5): anchor stride (0:
 * the network form; else 2..64), whether the network's cell gate applies,
 * the largest escape-direction error bound (rad) an interpolated pixel may
 * have, and the largest display-value change (in byte steps) allowed within
 * that bound. */
cudaError_t bhSurrogateSetAnchors(BHSurrogate* s, int stride, int useNetwork, float epsMax, float maxStep);

/* Step budget of the anchored form's anchor pass (default 600; 0: the frame's
 * maxSteps).  The pass lasts as long as its longest ray, and the few rays that
 * graze the photon sphere take several times the median step count; an anchor
 * that spends the budget is traced again in full with the other RK4 pixels,
 * so the frame does not depend on it. */
cudaError_t bhSurrogateSetAnchorSteps(BHSurrogate* s, int maxSteps);

/* Statistics of the last rendered frame (blocking). */
typedef struct BHSurrogateStats
{
    unsigned pixels;          /* W * H */
    unsigned rk4Pixels;       /* pixels traced by RK4 (fallback + held-out) */
    unsigned heldOut;         /* held-out pixels compared */
    unsigned heldOutOver1Lsb; /* held-out pixels whose RGBA8 differs by > 1 LSB */
    unsigned heldOutOverTol;  /* held-out pixels with HDR error > 1e-3 relative */
    float heldOutMaxAbs;      /* largest HDR difference on the held-out sample */
    unsigned anchors;         /* anchored form: anchor pixels (counted in rk4Pixels) */
    unsigned interpolated;    /* anchored form: pixels built from the anchors */
    unsigned rejectAnchors;   /* traced: an anchor not sky-only, or the cell gate, or the frame border */
    unsigned rejectBound;     /* traced: interpolation error bound above epsMax */
    unsigned rejectSky;       /* traced: sky not flat within the bound */
    unsigned skySampled;      /* anchored form: pixels whose sky flatness needed the sampled test */
    unsigned anchorsIncomplete; /* anchored form: anchors that spent the anchor step budget (traced
                                   again in full, counted in rk4Pixels twice and in rejectAnchors) */
} BHSurrogateStats;
cudaError_t bhSurrogateFrameStats(BHSurrogate* s, BHSurrogateStats* stats);

#ifdef __cplusplus
}
#endif
