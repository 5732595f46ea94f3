// ---------------------------------------------------------------------------
// bh_api.cpp -- the C-ABI of libbh.so (declared in include/bh_launch.h).
//
// Host work per frame: copy and sanitise the caller's RenderParams, compute
// the frame constants once (camera energy factor, jitter), then enqueue the
// persistent tracing kernel and, for the pipeline, the two post-processing
// kernels on the caller's stream.  Nothing synchronises; the return value is
// the launch status, as in the reference launchers
// (src/black_hole_kernel.cu:108-163 of Sqhh99/Black-hole).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <atomic>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "bh_launch.h"
#include "bh_internal.h"

namespace {
constexpr int kMaxDevices = 64;
std::atomic<unsigned long long> gAllocBytes[kMaxDevices];
}  // namespace

// Every device allocation the library makes (caches, tables, workspaces of
// handles) goes through here, so bhLibraryDeviceBytes can account for it.
cudaError_t bh_device_alloc(void** p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes);
    int dev = 0;
    if (e == cudaSuccess && cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices)
        gAllocBytes[dev].fetch_add(bytes);
    return e;
}

namespace {

// ---- per-device scratch: the ray counter of the work queue --------------------
constexpr size_t kScratchBytes = 4096;
std::mutex gScratchLock;
unsigned* gScratch[kMaxDevices] = {};

// Work counters: the scratch block holds a ring of kCounterSlots counters, 128 B
// apart; every tracing launch takes the next one, so launches on different
// streams may overlap (up to kCounterSlots in flight on a device).
constexpr unsigned kCounterSlots = 32;
std::atomic<unsigned> gSlot[kMaxDevices];

cudaError_t deviceScratch(unsigned** out);

cudaError_t launchCounter(unsigned** out)
{
    unsigned* base = nullptr;
    cudaError_t e = deviceScratch(&base);
    if (e != cudaSuccess) return e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    *out = base + (gSlot[dev].fetch_add(1u) % kCounterSlots) * 32u;
    return cudaSuccess;
}

cudaError_t deviceScratch(unsigned** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(gScratchLock);
    if (!gScratch[dev])
    {
        void* p = nullptr;
        e = bh_device_alloc(&p, kScratchBytes);
        if (e != cudaSuccess) return e;
        gScratch[dev] = static_cast<unsigned*>(p);
    }
    *out = gScratch[dev];
    return cudaSuccess;
}

// ---- trace order of the 8x4 tiles ---------------------------------------------------
// Mode 1 (centre-out) traces tiles in order of distance from the image centre:
// with the hole at the centre of the view, the shadow and photon ring -- the
// longest rays -- go first and the frame's last tiles are short escaping rays,
// which shortens the tail where SMs run out of work.  The table depends only on
// the resolution; it is built and uploaded once per device and resolution.
struct OrderCache
{
    int W = 0, H = 0;
    unsigned* dev = nullptr;
    size_t cap = 0;
};
OrderCache gOrder[kMaxDevices];
int gTileOrderMode = 1;

cudaError_t tileOrder(int W, int H, const unsigned** out)
{
    *out = nullptr;
    if (gTileOrderMode == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(gScratchLock);
    OrderCache& c = gOrder[dev];
    if (c.W != W || c.H != H || !c.dev)
    {
        const int tx = (W + 7) / 8, ty = (H + 3) / 4;
        const size_t n = (size_t)tx * ty;
        std::vector<unsigned> order(n);
        std::vector<float> key(n);
        const float cx = 0.5f * W, cy = 0.5f * H;
        for (size_t i = 0; i < n; ++i)
        {
            order[i] = (unsigned)i;
            const float dx = ((float)(i % tx) * 8.f + 4.f) - cx, dy = ((float)(i / tx) * 4.f + 2.f) - cy;
            key[i] = dx * dx + dy * dy;
        }
        std::stable_sort(order.begin(), order.end(), [&](unsigned a, unsigned b) { return key[a] < key[b]; });
        if (c.cap < n)
        {
            if (c.dev) cudaFree(c.dev);
            c.dev = nullptr;
            c.cap = 0;
            void* p = nullptr;
            e = bh_device_alloc(&p, n * sizeof(unsigned));
            if (e != cudaSuccess) return e;
            c.dev = static_cast<unsigned*>(p);
            c.cap = n;
        }
        // the table is shared by every stream: no frame may still read the old one, and the
        // upload (a pageable copy, whose transfer can outlast the call) must be complete before
        // a kernel on any stream reads it
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
        e = cudaMemcpy(c.dev, order.data(), n * sizeof(unsigned), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return e;
        c.W = W;
        c.H = H;
    }
    *out = c.dev;
    return cudaSuccess;
}

// ---- tuning (set by bhSetTuning / the autotuner) ------------------------------
struct Tuning
{
    int refillMin = 32;     // refill a warp when this many lanes are idle
    int blocksPerSm = 0;    // 0: as many as occupancy allows
};
Tuning gTune[2];            // [0] spherical family, [1] rotating family

// ---- frame constants ------------------------------------------------------------
inline float clampF(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }

// static-observer energy factor of the sky at the camera (reference trace.cuh:81-96)
float cameraEnergy(const RenderParams& P)
{
    const float3 c = P.camPos;
    const float r = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
    if (r < 1e-4f) return 1.f;
    if (P.model == BH_KERR || P.model == BH_KERR_NEWMAN)
    {
        float cth = clampF(c.y / r, -1.f, 1.f);
        float Sig = r * r + P.aSpin * P.aSpin * cth * cth;
        float m2r = 2.f * P.M * r - P.Qc * P.Qc;
        float gtt = -(1.f - m2r / std::fmax(Sig, 1e-8f));
        float alpha = std::sqrt(std::fmax(-gtt, 1e-6f));
        return clampF(1.f / alpha, 0.5f, 4.f);
    }
    float f = 1.f - 2.f * P.M / r + P.Qc * P.Qc / (r * r);
    return clampF(1.f / std::sqrt(std::fmax(f, 1e-6f)), 0.5f, 4.f);
}

// R2 low-discrepancy sub-pixel offset (reference post_process.cuh:47-53)
void jitter(int mode, int idx, float& jx, float& jy)
{
    if (mode == 0 || idx <= 0) { jx = jy = 0.5f; return; }
    float n = (float)idx;
    float a = 0.7548776662f * n + 0.5f, b = 0.5698402909f * n + 0.5f;
    jx = a - std::floor(a);
    jy = b - std::floor(b);
}

TraceParams frameParams(const RenderParams& P, int outMode, void* out)
{
    TraceParams t{};
    t.W = P.width;
    t.H = P.height;
    t.tilesX = (P.width + 7) / 8;
    const long long tilesY = (P.height + 3) / 4;
    t.nRays = (unsigned)((long long)t.tilesX * tilesY * 32);
    jitter(P.accumMode, P.sampleIndex, t.jx, t.jy);
    t.dirs = nullptr;
    t.camPos = P.camPos; t.camFwd = P.camForward; t.camRight = P.camRight; t.camUp = P.camUp;
    t.tanHalfFov = P.tanHalfFov;
    t.aspect = P.aspect;
    t.gCam = cameraEnergy(P);
    t.model = P.model;
    t.M = P.M; t.a = P.aSpin; t.Q = P.Qc;
    t.rPlus = P.rPlus; t.rPhoton = P.rPhoton;
    t.rCap = (P.rPlus > 1e-6f) ? P.rPlus : 0.05f * P.M;
    t.dPhi = P.dPhi;
    t.maxSteps = P.maxSteps;
    t.diskOn = P.diskEnabled ? 1 : 0;
    t.diskInner = P.diskInner; t.diskOuter = P.diskOuter; t.diskTime = P.diskTime;
    t.emisK = P.diskEmisScale; t.absK = P.diskAbsScale;
    t.spotsOn = P.hotSpotsEnabled ? 1 : 0;
    t.spotStrength = P.hotSpotStrength;
    t.outMode = outMode;
    t.out = out;
    t.accumMode = P.accumMode;
    t.sampleIndex = P.sampleIndex;
    t.exposure = P.exposure;
    t.swapRB = P.swapRB;
    const Tuning& tu = gTune[(P.model == BH_KERR || P.model == BH_KERR_NEWMAN) ? 1 : 0];
    t.refillMin = tu.refillMin;
    bh_fill_camera_frames(t);
    return t;
}

int familyBlocks(const RenderParams& P)
{
    return gTune[(P.model == BH_KERR || P.model == BH_KERR_NEWMAN) ? 1 : 0].blocksPerSm;
}

cudaError_t trace(TraceParams t, const RenderParams& P, int precision, bool stats, cudaStream_t s)
{
    if (precision < BH_PREC_FP32 || precision > BH_PREC_FP64) return cudaErrorInvalidValue;
    if (!t.out) return cudaErrorInvalidValue;
    cudaError_t e = launchCounter(&t.counter);
    if (e != cudaSuccess) return e;
    if (!t.dirs)
    {
        e = tileOrder(t.W, t.H, &t.tileOrder);
        if (e != cudaSuccess) return e;
    }
    return bh_launch_trace(t, precision, stats, familyBlocks(P), s);
}

PostConsts postConsts(const RenderParams& P)
{
    return PostConsts{P.exposure, P.bloomStrength, P.bloomEnabled ? 1 : 0, P.swapRB};
}

cudaError_t pipeline(uchar4* out, float4* accum, float4* bloomA, float4* bloomB, const RenderParams& p,
                     int precision, cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    if (!out || !accum || (P.bloomEnabled && (!bloomA || !bloomB))) return cudaErrorInvalidValue;
    cudaError_t e = trace(frameParams(P, BH_OUT_ACCUM, accum), P, precision, false, stream);
    if (e != cudaSuccess) return e;
    return bh_launch_post(out, accum, bloomB, bloomA, P.width, P.height, postConsts(P), stream);
}

}  // namespace

TraceParams bh_frame_params(const RenderParams& P, int outMode, void* out)
{
    return frameParams(P, outMode, out);
}

int bh_family_blocks(const RenderParams& P) { return familyBlocks(P); }

cudaError_t bh_device_counter(unsigned** out) { return launchCounter(out); }

extern "C" {

cudaError_t launchRenderPipeline(uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                                 const RenderParams& p, cudaStream_t stream)
{
    return pipeline(out, accum, bloomA, bloomB, p, BH_PREC_FP32, stream);
}

cudaError_t launchRenderKernel(uchar4* out, const RenderParams& p, cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    P.bloomEnabled = 0;
    TraceParams t = frameParams(P, BH_OUT_RGBA, out);
    t.jx = t.jy = 0.5f;   // the single-pass kernel always samples pixel centres
    return trace(t, P, BH_PREC_FP32, false, stream);
}

cudaError_t bhRenderPipelinePrec(uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                                 const RenderParams& p, int precision, cudaStream_t stream)
{
    return pipeline(out, accum, bloomA, bloomB, p, precision, stream);
}

cudaError_t bhRenderAccum(float4* accum, const RenderParams& p, int precision, cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    return trace(frameParams(P, BH_OUT_ACCUM, accum), P, precision, false, stream);
}

cudaError_t bhRenderHDR(float4* hdr, const RenderParams& p, int precision, cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    return trace(frameParams(P, BH_OUT_HDR, hdr), P, precision, false, stream);
}

cudaError_t bhPostProcess(uchar4* out, const float4* accum, float4* bloomA, float4* bloomB,
                          const RenderParams& p, cudaStream_t stream)
{
    RenderParams P = p;
    bhSanitizeRenderParams(&P);
    if (!out || !accum || (P.bloomEnabled && !bloomB)) return cudaErrorInvalidValue;
    return bh_launch_post(out, accum, bloomB, bloomA, P.width, P.height, postConsts(P), stream);
}

cudaError_t bhProbeGrid(BHProbe* out, const RenderParams& p, int nx, int ny, int precision,
                        cudaStream_t stream)
{
    if (nx < 1 || ny < 1) return cudaErrorInvalidValue;
    RenderParams P = p;   // as the reference probe: parameters used as given
    P.width = nx;
    P.height = ny;
    TraceParams t = frameParams(P, BH_OUT_PROBE, out);
    t.jx = t.jy = 0.5f;
    return trace(t, P, precision, true, stream);
}

cudaError_t bhProbeRays(BHProbe* out, const float3* dirs, int n, const RenderParams& p, int precision,
                        cudaStream_t stream)
{
    if (n < 0 || !dirs) return cudaErrorInvalidValue;
    RenderParams P = p;
    TraceParams t = frameParams(P, BH_OUT_PROBE, out);
    t.dirs = dirs;
    t.nRays = (unsigned)n;
    return trace(t, P, precision, true, stream);
}

int bhSetTuning(int family, int refillMin, int blocksPerSm)
{
    if (family < 0 || family > 1 || refillMin < 1 || refillMin > 32 || blocksPerSm < 0) return 0;
    gTune[family].refillMin = refillMin;
    gTune[family].blocksPerSm = blocksPerSm;
    return 1;
}

int bhSetTileOrder(int mode)
{
    if (mode < 0 || mode > 1) return 0;
    gTileOrderMode = mode;
    return 1;
}

int bhGetTileOrder(void) { return gTileOrderMode; }

void bhGetTuning(int family, int* refillMin, int* blocksPerSm)
{
    const Tuning& t = gTune[(family == 1) ? 1 : 0];
    if (refillMin) *refillMin = t.refillMin;
    if (blocksPerSm) *blocksPerSm = t.blocksPerSm;
}

double bhMeasureFp32Peak(void) { return bh_measure_fp32_peak(); }

unsigned long long bhLibraryDeviceBytes(int device)
{
    return (device >= 0 && device < kMaxDevices) ? gAllocBytes[device].load() : 0ull;
}

const char* bhVersion(void) { return "libbh 0.1 (sm_100a)"; }

}  // extern "C"
