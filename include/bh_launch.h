#pragma once
/*
 * bh_launch.h -- C-ABI of libbh.so, the B200 (sm_100a) null-geodesic tracer.
 *
 * The first two entry points are the drop-in boundary: same names, argument
 * order, ownership and error behaviour as the reference launchers in
 * src/black_hole_kernel.cu of Sqhh99/Black-hole.  Everything after them is
 * an additive extension (probing, precision modes, batching, measurement).
 *
 * Conventions shared by every entry point
 *  - All buffers are device pointers owned by the caller.
 *  - Work is enqueued on `stream` and the call returns without
 *    synchronising; the return value is the launch status
 *    (cudaGetLastError after the enqueue), as in the reference.
 *  - The caller's RenderParams is never modified: it is copied and the copy
 *    is sanitised (bhSanitizeRenderParams) before use.
 *  - Tracing kernels draw rays from a work counter.  The library allocates a
 *    small scratch block (4 KiB: a ring of 32 counters) once per device, on
 *    the first call made on that device; every launch takes the next counter
 *    of the ring and resets it on `stream`, so launches on different streams
 *    may overlap on the GPU, up to 32 at a time per device.  Make the first
 *    call before any CUDA-graph capture begins.
 */
#include <cuda_runtime_api.h>
#include <stdint.h>
#include "bh_render_params.h"

#ifdef __cplusplus
#define BH_PARAMS_IN const RenderParams&
extern "C" {
#else
#define BH_PARAMS_IN const RenderParams*
#endif

/* Metric families (reference metric.cuh:32-38). */
enum { BH_SCHWARZSCHILD = 0, BH_REISSNER_NORDSTROM = 1, BH_KERR = 2, BH_KERR_NEWMAN = 3 };

/* Arithmetic of the geodesic integration.
 *  BH_PREC_FP32  : everything in FP32 (the reference's arithmetic).
 *  BH_PREC_MIXED : FP32 stepping; FP64 for the conserved-quantity set-up at
 *                  the camera, for every passage of the Kerr-family polar cap
 *                  (|sin th| < 1/64, state carried in FP64), for the
 *                  spherical family's turning-point steps, and for bisection
 *                  of equatorial disk crossings.
 *  BH_PREC_FP64  : the whole integration in FP64 (GPU oracle). */
enum { BH_PREC_FP32 = 0, BH_PREC_MIXED = 1, BH_PREC_FP64 = 2 };

/* Derived black-hole quantities (reference metric.cuh:204-215; the two bool
 * flags are ints here so the struct is plain C). */
typedef struct BHDerived
{
    float a, Q;          /* code units: a = a* M (signed), Q = q M */
    float rPlus, rMinus; /* horizons (0 when naked) */
    float rPhoton;       /* photon sphere / co-rotating photon orbit */
    float rErgo;         /* equatorial ergosphere radius */
    float rIsco;         /* numeric innermost stable circular orbit */
    int   clamped;       /* inputs had to be modified */
    int   naked;         /* a*^2 + q^2 > 1 */
} BHDerived;

/* Per-ray record written by the probe entry points.  Field meanings follow
 * the reference TraceResult (src/trace.cuh:418-428) and its test probe
 * (tests/test_main.cu:63-69); the last group is added by this library. */
typedef struct BHProbe
{
    int   outcome;      /* 0 captured (horizon), 1 escaped -- reference Probe.outcome */
    int   cls;          /* 0 captured, 1 disk hit (trans < 0.5), 2 escaped */
    int   steps;        /* integration steps taken (reference TraceResult.steps) */
    int   diskSamples;  /* disk sub-samples that contributed emission */
    float escDir[3];    /* deflected escape direction (unit) */
    float trans;        /* remaining transmittance */
    float accum[3];     /* disk radiance accumulated along the ray */
    float maxHviol;     /* max |K| / (E^2 (r^2 + a^2)) along a rotating-metric ray */
    float hdr[3];       /* linear HDR sample (accum + sky * trans) */
    float diskR;        /* cylindrical radius where trans first fell below 0.5 (0 if never) */
    float diskG;        /* emitter redshift factor g at that sub-sample */
    float drift;        /* relative drift of the conserved quantity (Carter Q or Binet integral) */
} BHProbe;

/* ---- drop-in boundary (reference src/black_hole_kernel.cu) ------------- */

/* Full-quality frame: one geodesic sample per pixel blended into `accum`
 * (W*H float4, persistent across frames), half-resolution bloom through
 * `bloomA` / `bloomB` (ceil(W/2)*ceil(H/2) float4 each; unused when bloom is
 * off), then exposure, ACES, gamma and dither into `out` (W*H uchar4).
 * With bloom on, the call leaves the horizontally blurred bright pass in
 * `bloomB` and the finished (vertically blurred) bloom in `bloomA`, as the
 * reference's passes do.
 * Replaces launchRenderPipeline, reference src/black_hole_kernel.cu:108-134. */
cudaError_t launchRenderPipeline(uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                                 BH_PARAMS_IN p, cudaStream_t stream);

/* Single pass: one centred sample per pixel straight to `out`; no
 * accumulation, bloom forced off.
 * Replaces launchRenderKernel, reference src/black_hole_kernel.cu:151-163. */
cudaError_t launchRenderKernel(uchar4* out, BH_PARAMS_IN p, cudaStream_t stream);

/* ---- host-side parameter handling (reference src/metric.cuh) ----------- */

/* Clamp every field to a renderable value; returns 1 if anything changed.
 * Replaces sanitizeRenderParams, reference src/metric.cuh:344-419. */
int bhSanitizeRenderParams(RenderParams* p);

/* Validate (clamp) M, a*, q for `model` in place and derive horizons,
 * photon orbit, ergosphere and numeric ISCO into *out.
 * Replaces bhValidateAndDerive, reference src/metric.cuh:257-329. */
void bhValidateAndDerive(int model, float* M, float* aStar, float* q, int allowNaked,
                         BHDerived* out);

/* One black hole to derive on the device (the arguments of bhValidateAndDerive). */
typedef struct BHDeriveRequest
{
    int model;
    float M, aStar, q;
    int allowNaked;
} BHDeriveRequest;

/* bhValidateAndDerive for n black holes on the GPU (device arrays): out[i]
 * receives the derived quantities and requests[i].M / aStar / q are
 * overwritten with the validated values, exactly as the host function
 * updates its arguments.  Same results as the host function (and so as the
 * reference's host code, metric.cuh:224-329) bit for bit, except rPhoton of
 * Kerr / Kerr-Newman, whose acos and cos are rounded correctly here: one ulp
 * of difference from the host libm's acos grows to a few ulps (within 1e-6
 * relative); the numeric ISCO scan runs as one CTA per request.  No counterpart in the reference, which
 * derives on the host per view. */
cudaError_t bhDeriveBatch(BHDeriveRequest* requests, BHDerived* out, int n, cudaStream_t stream);

/* ---- extensions ------------------------------------------------------- */

/* Trace the nx*ny grid of pixel-centre rays of the camera in `p` and write
 * one BHProbe per ray (row-major).  The analogue of the reference's test
 * probe kernel (tests/test_main.cu:71-89), with constraint monitoring on. */
cudaError_t bhProbeGrid(BHProbe* out, BH_PARAMS_IN p, int nx, int ny, int precision,
                        cudaStream_t stream);

/* Trace `n` arbitrary unit directions (float3, device memory) from the
 * camera position (reference tests/test_main.cu:91-98, batched). */
cudaError_t bhProbeRays(BHProbe* out, const float3* dirs, int n, BH_PARAMS_IN p,
                        int precision, cudaStream_t stream);

/* Linear-HDR frame: one sample per pixel (the same jitter rule as the
 * pipeline) into `hdr` (W*H float4, alpha = 1), no blending, no
 * post-processing.  The sample of reference renderSampleHDR
 * (src/trace.cuh:908-926) for every pixel. */
cudaError_t bhRenderHDR(float4* hdr, BH_PARAMS_IN p, int precision, cudaStream_t stream);

/* Pipeline with a selectable integration precision (BH_PREC_*).  With
 * BH_PREC_FP32 it is launchRenderPipeline. */
cudaError_t bhRenderPipelinePrec(uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                                 BH_PARAMS_IN p, int precision, cudaStream_t stream);

/* The tracing half of the pipeline: one sample per pixel blended into
 * `accum` exactly as launchRenderPipeline does, without post-processing.
 * launchRenderPipeline == bhRenderAccum + bhPostProcess on the same stream. */
cudaError_t bhRenderAccum(float4* accum, BH_PARAMS_IN p, int precision, cudaStream_t stream);

/* Post-processing alone (bloom + tonemap of an existing accumulation
 * buffer; bloomA / bloomB filled as by launchRenderPipeline):
 * reference src/black_hole_kernel.cu:41-103. */
cudaError_t bhPostProcess(uchar4* out, const float4* accum, float4* bloomA, float4* bloomB,
                          BH_PARAMS_IN p, cudaStream_t stream);

/* Work-distribution tuning of a metric family (0: Schwarzschild / RN,
 * 1: Kerr / Kerr-Newman): a warp refills its idle lanes once at least
 * `refillMin` (1..32) are idle; `blocksPerSm` CTAs (160 threads for the
 * rotating family, 128 for the spherical one) stay
 * resident per SM (0: as many as occupancy allows).  With refillMin = 32 (the
 * default) FP32 renders run the tile-synchronous kernel (a warp traces one
 * 8x4 tile to its last ray, then takes the next); below 32 they run the
 * refill-queue kernel.  Returns 1 when applied, 0 when a value is out of
 * range.  Process-wide; set by the autotuner. */
int bhSetTuning(int family, int refillMin, int blocksPerSm);
void bhGetTuning(int family, int* refillMin, int* blocksPerSm);

/* Order in which the 8x4-pixel tiles of a frame are traced: 0 row-major,
 * 1 centre-out (default; the shadow and photon ring first, so the frame ends on
 * short escaping rays).  The table is built once per device and resolution on
 * the first call at that resolution (a blocking upload that first waits for
 * all work on the device, since frames of the previous resolution may still
 * read the table: make that first call outside any stream capture).  Returns
 * 1 when applied, 0 when out of range. */
int bhSetTileOrder(int mode);
int bhGetTileOrder(void);

/* ---- batches of views (no counterpart in the reference) ----------------- */

/* One view of a batch: its parameters and the buffers launchRenderPipeline
 * would take for it (bloomA / bloomB may be null when bloom is off). */
typedef struct BHView
{
    RenderParams params;
    uchar4* out;
    float4* accum;
    float4* bloomA;
    float4* bloomB;
} BHView;

/* Render n views: the same images as n launchRenderPipeline calls, traced by
 * one persistent launch per metric family (Kerr / Kerr-Newman, then
 * Schwarzschild / Reissner-Nordstrom) that draws 8x4-pixel tiles of all the
 * family's views, any mix of resolutions, from a single device work queue,
 * followed by each view's bloom and tonemap.  Within a family views are queued
 * largest first.  FP32; CTAs per SM from bhSetTuning of each family.  The
 * library keeps per-device tables of the views' frame constants, grown on
 * demand (an allocation on the first call and when n grows; make those calls
 * outside stream capture).  Immediate-mode batches on one device share those
 * tables, so two bhRenderBatch calls must not overlap on the GPU; the graph
 * form below owns its own. */
cudaError_t bhRenderBatch(const BHView* views, int n, cudaStream_t stream);

/* The batch as a CUDA graph: created once for fixed views (buffers,
 * resolutions, bloom on/off, exposure, bloom strength and metric family),
 * then launched every frame; bhBatchGraphUpdate replaces the other parameters
 * (camera, spin, charge, disk time, ...) before the next launch (it waits for
 * the previous launch to have read them) and refuses changes to the fixed
 * ones with cudaErrorInvalidValue.  The graph owns its tables and counter. */
typedef struct BHBatchGraph BHBatchGraph;
cudaError_t bhBatchGraphCreate(BHBatchGraph** graph, const BHView* views, int n);
cudaError_t bhBatchGraphUpdate(BHBatchGraph* graph, const BHView* views, int n);
cudaError_t bhBatchGraphLaunch(BHBatchGraph* graph, cudaStream_t stream);
void bhBatchGraphDestroy(BHBatchGraph* graph);

/* Autotuner: times the FP32 tracing kernel of p's metric family on p's view
 * (blocking, with a temporary HDR buffer) over the resident CTAs per SM, the
 * warp refill threshold and the tile order, applies the fastest setting
 * (bhSetTuning / bhSetTileOrder) and reports it. */
cudaError_t bhAutotune(BH_PARAMS_IN p, int* refillMin, int* blocksPerSm, int* tileOrder, float* bestMs);

/* Batch autotuner: for each metric family present in the views, times
 * bhRenderBatch on that family's views (blocking) over the resident CTAs per
 * SM, applies the fastest (bhSetTuning; the refill threshold is kept) and
 * reports it (blocksKerr / blocksSph are left unchanged for an absent family).
 * bestMs = the two families' best times added. */
cudaError_t bhAutotuneBatch(const BHView* views, int n, int* blocksKerr, int* blocksSph, float* bestMs);

/* ---- allocation-free pipeline (no counterpart in the reference) --------- */

/* Largest half-resolution image ((W+1)/2 * (H+1)/2 pixels) the allocation-free
 * pipeline accepts with bloom on: 1920x1080 and 2048x1024 fit. */
#define BH_NOALLOC_MAX_HALF_PIXELS 524288

/* launchRenderPipeline for callers that cannot let a library allocate device
 * memory -- a plugin whose host application owns all device memory and hands
 * out only its own buffers; a real-time frame loop that must never stall on
 * the allocator (cudaMalloc can synchronise the device).  No counterpart in
 * the reference.  The caller still passes the
 * output (W*H uchar4) and the accumulation buffer (W*H float4, persistent);
 * the bloom intermediate and the work counter live in one fixed array inside
 * the library (256 B + BH_NOALLOC_MAX_HALF_PIXELS * 16 B = 8 MiB), which every
 * GPU that loads libbh.so holds until exit.  The call allocates nothing: it
 * makes no cudaMalloc or cudaFree and calls no allocating library routine.
 *  - Frames whose half-resolution image exceeds BH_NOALLOC_MAX_HALF_PIXELS
 *    are rejected with cudaErrorInvalidValue when bloom is on (nothing is
 *    launched); with bloom off any size is accepted.
 *  - The array belongs to the library's module.  Under lazy module loading
 *    (the CUDA default) the first call on a device loads that module, which
 *    places the 8 MiB array on the device; later calls allocate nothing.
 *    Make that first call before any stream capture begins.
 *  - Every call looks up the array's device address in the current context
 *    (cudaGetSymbolAddress, which allocates nothing).
 *  - All calls on a device share the array and it keeps the last call's
 *    contents; calls that overlap on the GPU race, so serialise them (one
 *    stream, or events between streams).
 *  - Tiles are traced in row-major order; the image is launchRenderPipeline's. */
cudaError_t bhRenderPipelineNoAlloc(uchar4* out, float4* accum, BH_PARAMS_IN p, cudaStream_t stream);

/* Measured FP32 FMA throughput of the current device, in TFLOP/s: the higher
 * of a scalar-FMA and a packed FP32x2-FMA kernel (independent chains, every
 * SM filled), timed with CUDA events (blocking). */
double bhMeasureFp32Peak(void);

/* Bytes of device memory libbh.so has allocated on `device` since it was
 * loaded, cumulative (work-counter ring, tile-order and batch tables, graph
 * and surrogate workspaces).  An accounting aid: a process whose only libbh
 * calls are bhRenderPipelineNoAlloc reads 0. */
unsigned long long bhLibraryDeviceBytes(int device);

/* Library version / build string. */
const char* bhVersion(void);

#ifdef __cplusplus
}
#endif
#undef BH_PARAMS_IN
