// ---------------------------------------------------------------------------
// bh_sg_api.cpp -- C-ABI of the lensing surrogate (include/bh_surrogate_api.h):
// the network object, the RK4-traced ray set, the training loop, and the
// surrogate frame (fused inference -> RK4 for the rest -> held-out check ->
// bloom and tonemap).
// No counterpart in the reference (it has no learned component); the frames
// it renders use the reference's camera, sky and post-processing exactly as
// launchRenderPipeline does.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <cuda_runtime.h>
#include "bh_internal.h"
#include "bh_launch.h"
#include "bh_sg_infer.h"
#include "bh_sg_train.h"
#include "bh_surrogate.h"
#include "bh_surrogate_api.h"

namespace {

constexpr int kHidW = 256 * 256;           // one hidden weight matrix
constexpr int kWCount = 4 * kHidW + 256 * 64;
constexpr int kBiasCount = 4 * 256 + 16;
constexpr int kHeldStride = 256;
constexpr int kAnchorSteps = 600;
constexpr float kPi = 3.14159265358979f;

// uniform float in [lo, hi) from a 32-bit generator (portable, unlike std distributions)
float uni(std::mt19937& g, float lo, float hi)
{
    return lo + (hi - lo) * (float)((double)g() * (1.0 / 4294967296.0));
}

struct CritKey
{
    int model = -1, maxSteps = 0;
    float M = 0, a = 0, Q = 0, dist = 0, cosIncl = 0, tanHalfFov = 0, dPhi = 0;
    bool operator==(const CritKey& o) const
    {
        return model == o.model && maxSteps == o.maxSteps && M == o.M && a == o.a && Q == o.Q && dist == o.dist &&
               cosIncl == o.cosIncl && tanHalfFov == o.tanHalfFov && dPhi == o.dPhi;
    }
};

float length3(const float3& v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// The orbit camera of the reference application (src/main.cpp:186-228): camera
// at distance d, elevation el, azimuth az about the +Y spin axis, looking at
// the hole, no body rotation.
void orbitCamera(RenderParams& P, float az, float el, float d, float fovDeg)
{
    const float ca = std::cos(az), sa = std::sin(az), ce = std::cos(el), se = std::sin(el);
    float3 p{d * ce * ca, d * se, d * ce * sa};
    const float fl = length3(p);
    float3 f{-p.x / fl, -p.y / fl, -p.z / fl};
    float3 r{-f.z, 0.f, f.x};
    float rl = std::sqrt(r.x * r.x + r.z * r.z);
    if (rl < 1e-6f) { r = float3{1.f, 0.f, 0.f}; rl = 1.f; }
    r = float3{r.x / rl, 0.f, r.z / rl};
    float3 u{r.y * f.z - r.z * f.y, r.z * f.x - r.x * f.z, r.x * f.y - r.y * f.x};
    const float ul = length3(u);
    u = float3{u.x / ul, u.y / ul, u.z / ul};
    P.camPos = p; P.camForward = f; P.camRight = r; P.camUp = u;
    P.tanHalfFov = std::tan(fovDeg * kPi / 180.f * 0.5f);
    P.aspect = (float)P.width / (float)P.height;
}

// applyBlackHole (src/main.cpp:97-134): derive, disk inner edge at the ISCO.
void applyHole(RenderParams& P, int model, float aStar, float q)
{
    float M = 0.5f, a = aStar, qq = q;
    BHDerived d;
    bhValidateAndDerive(model, &M, &a, &qq, 0, &d);
    P.model = model;
    P.M = M;
    P.aSpin = d.a; P.Qc = d.Q;
    P.rPlus = d.rPlus; P.rPhoton = d.rPhoton; P.rErgo = d.rErgo;
    P.allowNaked = 0;
    P.diskInner = d.rIsco;
    P.diskOuter = 8.f;
}

// normalised scene inputs of a sanitised orbit-camera frame
void sceneInputs(const RenderParams& P, float& aN, float& qN, float& rN, float& iN)
{
    const float r = length3(P.camPos);
    const float incl = std::acos(std::fmax(-1.f, std::fmin(1.f, P.camPos.y / r))) * 180.f / kPi;
    aN = P.aSpin / P.M;
    qN = (P.Qc / P.M - 0.3f) * (1.f / 0.3f);
    rN = (std::log(r) - 1.7917595f) * (2.f / 2.3025851f) - 1.f;
    iN = (incl - 45.f) * (1.f / 43.f);
}

}  // namespace

struct BHSurrogate
{
    SgState S;
    cudaStream_t stream = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr;   // anchored frames: the cell gate beside the anchor pass
    // frame scratch
    unsigned* list = nullptr;
    size_t listCap = 0;
    unsigned* counters = nullptr;     // [0] RK4 list groups x 32, [1] held-out count, [4..7] held-out statistics,
                                      // [8..11] anchored tallies, [12] listed pixels, [13] list + held-out length,
                                      // [14] pixels deferred to the sampled sky test, [15] incomplete anchors
    unsigned* heldPix = nullptr;
    float4* heldPred = nullptr;
    unsigned heldCap = 0;
    float4* sampleDir = nullptr;      // anchored form: pixels deferred to the sampled sky test
    unsigned* samplePix = nullptr;
    unsigned sampleCap = 0;
    unsigned frames = 0;
    // acceptance gate of the surrogate frame
    float minProb = 0.95f, minConf = 0.95f, critBand = 0.02f;
    int heldStride = kHeldStride;
    unsigned lastPixels = 0;
    // critical curve cache
    bool critValid = false;
    CritKey critKey;
    float crit[kCritBins];
    // batch buffers of the training loop
    float* bIn = nullptr;
    float* bTgt = nullptr;
    int bCap = 0;
    // anchored frames: RK4 anchors every anchorStride pixels (0: the network's own directions)
    int anchorStride = 8;
    bool anchorNet = true;
    int anchorSteps = kAnchorSteps;   // step budget of the anchor pass (0: the frame's maxSteps)
    float epsMax = 1e-4f, maxStep = 0.5f;
    int aW = 0, aH = 0, aS = 0, aNx = 0, aNy = 0;
    unsigned* anchorPix = nullptr;    // anchor pixels in trace order
    unsigned* anchorRecIdx = nullptr; // trace position k -> the row-major record of anchorPix[k]
    unsigned* blockOrder = nullptr;   // resolve pass: 32 x 8 pixel blocks, nearest the screen centre first
    size_t bCapOrder = 0;
    BHAnchor* anchorRec = nullptr;
    unsigned* cellPix = nullptr;      // cell-centre pixels
    float2* cellGate = nullptr;
    size_t aCap = 0, cCap = 0;
    unsigned lastAnchors = 0;
};

namespace {

void freeAll(BHSurrogate* s)
{
    SgState& S = s->S;
    sg_free_batch(S);
    void* ps[] = {S.params, S.grads, S.adamM, S.adamV, S.W, S.Wt, S.biasPacked, S.loss, S.dsIn, S.dsTgt, s->list,
                  s->counters, s->heldPix, s->heldPred, s->bIn, s->bTgt, s->anchorPix, s->anchorRecIdx, s->anchorRec,
                  s->cellPix, s->cellGate, s->sampleDir, s->samplePix, s->blockOrder};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (s->evFork) cudaEventDestroy(s->evFork);
    if (s->evJoin) cudaEventDestroy(s->evJoin);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

cudaError_t checkErrWord(BHSurrogate* s)
{
    unsigned flags = 0;
    cudaError_t e = cudaMemcpy(&flags, s->S.err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    if (flags)
    {
        unsigned zero = 0;
        cudaMemcpy(s->S.err, &zero, sizeof(unsigned), cudaMemcpyHostToDevice);
        return cudaErrorTimeout;
    }
    return cudaSuccess;
}

// Critical screen radius (tan units) per polar angle: bisection between a ray
// aimed at the hole (captured) and one far outside (escaped), FP32 RK4 without
// the disk, all angle bins in one probe launch per step.
cudaError_t criticalCurve(BHSurrogate* s, const RenderParams& P0, float* crit)
{
    RenderParams P = P0;
    P.diskEnabled = 0;
    P.hotSpotsEnabled = 0;
    const int n = kCritBins;
    std::vector<float> lo(n, 0.f), hi(n, 4.f);
    std::vector<float3> dirs(n);
    std::vector<BHProbe> rec(n);
    float3* dDirs = nullptr;
    BHProbe* dRec = nullptr;
    cudaError_t e = bh_device_alloc(reinterpret_cast<void**>(&dDirs), n * sizeof(float3));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&dRec), n * sizeof(BHProbe));
    auto dirFor = [&](int k, float rho) {
        const float psi = 2.f * kPi * (float)k / (float)n;
        const float sx = rho * std::cos(psi), sy = rho * std::sin(psi);
        float3 d{P.camForward.x + P.camRight.x * sx + P.camUp.x * sy,
                 P.camForward.y + P.camRight.y * sx + P.camUp.y * sy,
                 P.camForward.z + P.camRight.z * sx + P.camUp.z * sy};
        const float l = length3(d);
        return float3{d.x / l, d.y / l, d.z / l};
    };
    for (int it = 0; it < 22 && e == cudaSuccess; ++it)
    {
        for (int k = 0; k < n; ++k) dirs[k] = dirFor(k, 0.5f * (lo[k] + hi[k]));
        e = cudaMemcpyAsync(dDirs, dirs.data(), n * sizeof(float3), cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = bhProbeRays(dRec, dDirs, n, P, BH_PREC_FP32, s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(rec.data(), dRec, n * sizeof(BHProbe), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        for (int k = 0; k < n && e == cudaSuccess; ++k)
        {
            const float mid = 0.5f * (lo[k] + hi[k]);
            if (rec[k].outcome == 1) hi[k] = mid; else lo[k] = mid;
        }
    }
    for (int k = 0; k < n; ++k) crit[k] = 0.5f * (lo[k] + hi[k]);
    if (dDirs) cudaFree(dDirs);
    if (dRec) cudaFree(dRec);
    return e;
}

// Frame scratch of a W x H frame.  The RK4 list holds whole 32-entry groups
// (8x4 tiles in the anchored form, 32 consecutive pixels in the network form),
// bounded by the frame padded to whole tiles or whole groups; then, in the
// anchored form, the deferred pixels the sampled sky test rejects; then the
// held-out sample (at most heldCap pixels).  The deferral buffer holds every
// pixel of the frame (20 bytes each), so which pixels are deferred, and hence
// the frame, never depends on the order of the resolve pass's atomics.
cudaError_t ensureFrame(BHSurrogate* s, int W, int H)
{
    const size_t pixels = (size_t)W * H;
    const size_t stride = s->heldStride > 0 ? (size_t)s->heldStride : pixels + 1;
    const size_t want = std::min(pixels, pixels / stride * 2 + 4096);
    const size_t sampleCap = pixels;
    const size_t listLen =
        std::max((size_t)((W + 7) / 8 * 8) * (size_t)((H + 3) / 4 * 4), (pixels + 31) / 32 * 32) + sampleCap + want;
    if (listLen <= s->listCap && want <= s->heldCap && sampleCap <= s->sampleCap) return cudaSuccess;
    void* old[] = {s->list, s->heldPix, s->heldPred, s->sampleDir, s->samplePix};
    for (void* p : old)
        if (p) cudaFree(p);
    s->list = nullptr; s->heldPix = nullptr; s->heldPred = nullptr; s->sampleDir = nullptr; s->samplePix = nullptr;
    s->listCap = 0; s->heldCap = 0; s->sampleCap = 0;
    const unsigned cap = (unsigned)want;
    cudaError_t e = bh_device_alloc(reinterpret_cast<void**>(&s->list), listLen * sizeof(unsigned));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&s->heldPix), cap * sizeof(unsigned));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&s->heldPred), cap * sizeof(float4));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&s->sampleDir), sampleCap * sizeof(float4));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&s->samplePix), sampleCap * sizeof(unsigned));
    if (e != cudaSuccess) return e;
    s->listCap = listLen;
    s->heldCap = cap;
    s->sampleCap = (unsigned)sampleCap;
    return cudaSuccess;
}

// Anchor lattice of a W x H frame: pixels (S ax, S ay), and the centres of the
// (nx - 1) x (ny - 1) cells between them; built once per size and stride
// (blocking upload).  The anchors are traced in 8x4 groups of neighbouring
// anchors (one tracing warp each), groups nearest the screen centre first as
// in the plain frame's tile order, so the long rays near the shadow start early.
cudaError_t ensureAnchors(BHSurrogate* s, int W, int H, int S)
{
    if (s->aW == W && s->aH == H && s->aS == S && s->anchorPix) return cudaSuccess;
    const int nx = (W - 1) / S + 1, ny = (H - 1) / S + 1;
    const size_t nA = (size_t)nx * ny, nC = (size_t)std::max(nx - 1, 1) * std::max(ny - 1, 1);
    cudaError_t e = cudaSuccess;
    if (nA > s->aCap)
    {
        if (s->anchorPix) cudaFree(s->anchorPix);
        if (s->anchorRecIdx) cudaFree(s->anchorRecIdx);
        if (s->anchorRec) cudaFree(s->anchorRec);
        s->anchorPix = nullptr; s->anchorRecIdx = nullptr; s->anchorRec = nullptr; s->aCap = 0;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->anchorPix), nA * sizeof(unsigned)))) return e;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->anchorRecIdx), nA * sizeof(unsigned)))) return e;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->anchorRec), nA * sizeof(BHAnchor)))) return e;
        s->aCap = nA;
    }
    if (nC > s->cCap)
    {
        if (s->cellPix) cudaFree(s->cellPix);
        if (s->cellGate) cudaFree(s->cellGate);
        s->cellPix = nullptr; s->cellGate = nullptr; s->cCap = 0;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->cellPix), nC * sizeof(unsigned)))) return e;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->cellGate), nC * sizeof(float2)))) return e;
        s->cCap = nC;
    }
    const int gx = (nx + 7) / 8, gy = (ny + 3) / 4;
    std::vector<unsigned> groups((size_t)gx * gy);
    std::vector<float> key(groups.size());
    for (size_t g = 0; g < groups.size(); ++g)
    {
        groups[g] = (unsigned)g;
        const float dx = ((float)(g % gx) * 8.f + 3.5f) * S - 0.5f * W, dy = ((float)(g / gx) * 4.f + 1.5f) * S - 0.5f * H;
        key[g] = dx * dx + dy * dy;
    }
    std::stable_sort(groups.begin(), groups.end(), [&](unsigned p, unsigned q) { return key[p] < key[q]; });
    std::vector<unsigned> a, recIdx, c(nC, 0u);
    recIdx.reserve(nA);
    a.reserve(nA);
    for (unsigned g : groups)
        for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 8; ++i)
            {
                const int x = (int)(g % gx) * 8 + i, y = (int)(g / gx) * 4 + j;
                if (x >= nx || y >= ny) continue;
                recIdx.push_back((unsigned)(y * nx + x));
                a.push_back((unsigned)(y * S) * (unsigned)W + (unsigned)(x * S));
            }
    for (int y = 0; y + 1 < ny; ++y)
        for (int x = 0; x + 1 < nx; ++x)
            c[(size_t)y * (nx - 1) + x] = (unsigned)(y * S + S / 2) * (unsigned)W + (unsigned)(x * S + S / 2);
    // blocking upload: no earlier frame of this handle may still read the tables, and the
    // pageable copies must have landed before a kernel on any stream reads them
    if ((e = cudaDeviceSynchronize())) return e;
    if ((e = cudaMemcpy(s->anchorPix, a.data(), nA * sizeof(unsigned), cudaMemcpyHostToDevice))) return e;
    if ((e = cudaMemcpy(s->anchorRecIdx, recIdx.data(), nA * sizeof(unsigned), cudaMemcpyHostToDevice))) return e;
    // resolve blocks (32 x 8 pixels) nearest the screen centre first
    const int rbx = (W + 31) / 32, rby = (H + 7) / 8;
    const size_t nB = (size_t)rbx * rby;
    std::vector<unsigned> blocks(nB);
    std::vector<float> bkey(nB);
    for (size_t b = 0; b < nB; ++b)
    {
        blocks[b] = (unsigned)b;
        const float dx = (float)(b % rbx) * 32.f + 16.f - 0.5f * W, dy = (float)(b / rbx) * 8.f + 4.f - 0.5f * H;
        bkey[b] = dx * dx + dy * dy;
    }
    std::stable_sort(blocks.begin(), blocks.end(), [&](unsigned p, unsigned q) { return bkey[p] < bkey[q]; });
    if (nB > s->bCapOrder)
    {
        if (s->blockOrder) cudaFree(s->blockOrder);
        s->blockOrder = nullptr; s->bCapOrder = 0;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->blockOrder), nB * sizeof(unsigned)))) return e;
        s->bCapOrder = nB;
    }
    if ((e = cudaMemcpy(s->blockOrder, blocks.data(), nB * sizeof(unsigned), cudaMemcpyHostToDevice))) return e;
    if ((e = cudaMemcpy(s->cellPix, c.data(), nC * sizeof(unsigned), cudaMemcpyHostToDevice))) return e;
    if ((e = cudaDeviceSynchronize())) return e;
    s->aW = W; s->aH = H; s->aS = S; s->aNx = nx; s->aNy = ny;
    return cudaSuccess;
}

// The anchored frame: cell gate (network), RK4 anchors, resolve pass; the RK4
// list, held-out comparison and post-processing follow in bhSurrogateRender.
cudaError_t anchoredFrame(BHSurrogate* s, const RenderParams& P, float4* accum, cudaStream_t stream)
{
    const int S = s->anchorStride;
    cudaError_t e = ensureAnchors(s, P.width, P.height, S);
    if (e != cudaSuccess) return e;
    const unsigned nA = (unsigned)(s->aNx * s->aNy);
    const unsigned nC = (unsigned)((s->aNx - 1) * (s->aNy - 1));
    const bool gate = s->anchorNet && s->aNx > 1 && s->aNy > 1;
    // the cell gate (network at the cell centres) needs nothing of the anchor pass: it runs on
    // the surrogate's own stream beside it and takes the SMs the anchor pass's tail frees
    if (gate && (e = cudaEventRecord(s->evFork, stream)) != cudaSuccess) return e;
    TraceParams t = bh_frame_params(P, BH_OUT_ANCHOR, s->anchorRec);
    if (s->anchorSteps > 0 && s->anchorSteps < t.maxSteps) t.maxSteps = s->anchorSteps;
    t.pixList = s->anchorPix;
    t.outIndex = s->anchorRecIdx;     // records land row-major for the resolve pass
    t.nRays = nA;
    if ((e = bh_device_counter(&t.counter)) != cudaSuccess) return e;
    if ((e = bh_launch_trace(t, BH_PREC_FP32, false, bh_family_blocks(P), stream)) != cudaSuccess) return e;
    if (gate)
    {
        SgState& S_ = s->S;
        SgFrame F{};
        F.tp = bh_frame_params(P, BH_OUT_ACCUM, accum);
        sceneInputs(P, F.aN, F.qN, F.rN, F.iN);
        F.evalPix = s->cellPix;
        F.gateOut = s->cellGate;
        SgInferArgs a{S_.W, S_.W + 4 * kHidW, S_.biasPacked, nullptr, nullptr, nC, S_.err};
        if ((e = cudaStreamWaitEvent(s->stream, s->evFork, 0)) != cudaSuccess) return e;
        if ((e = sg_infer_launch(a, &F, s->stream)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(s->evJoin, s->stream)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(stream, s->evJoin, 0)) != cudaSuccess) return e;
    }
    SgAnchorFrame A{};
    A.tp = bh_frame_params(P, BH_OUT_ACCUM, accum);
    A.anchors = s->anchorRec;
    A.blockOrder = s->blockOrder;
    A.S = S; A.nx = s->aNx; A.ny = s->aNy;
    A.cellGate = s->anchorNet ? s->cellGate : nullptr;
    A.minProb = s->minProb;
    A.epsMax = s->epsMax;
    A.maxStep = s->maxStep;
    A.list = s->list;
    A.listCount = s->counters;
    A.heldPix = s->heldPix;
    A.heldPred = s->heldPred;
    A.heldCount = s->counters + 1;
    A.heldCap = s->heldCap;
    // under progressive accumulation the buffer holds the blend, not this frame's sample, so the
    // held-out comparison (RK4 sample against the interpolated one) is off
    A.heldStride = P.accumMode != 0 ? 0 : s->heldStride;
    A.frameSeed = ++s->frames;
    A.sampleDir = s->sampleDir;
    A.samplePix = s->samplePix;
    A.sampleCount = s->counters + 14;
    A.sampleCap = s->sampleCap;
    A.stats = s->counters + 8;      // [8..11] tallies, [12] pixels on the list
    s->lastAnchors = nA;
    return sg_anchor_resolve(A, stream);
}

// RK4 for the listed pixels and, after them, the held-out sample (the tracer
// reads the list and its device-side length), the held-out comparison, then
// bloom and tonemap.
cudaError_t traceListAndPost(BHSurrogate* s, const RenderParams& P, uchar4* out, float4* accum, float4* bloomA,
                             float4* bloomB, cudaStream_t stream)
{
    cudaError_t e = sg_append_held(s->list, s->counters, s->heldPix, s->counters + 1, s->heldCap, s->counters + 13,
                                   stream);
    if (e != cudaSuccess) return e;
    TraceParams t = bh_frame_params(P, BH_OUT_ACCUM, accum);
    t.pixList = s->list;
    t.nRaysDev = s->counters + 13;
    t.nRays = (unsigned)s->listCap;
    if ((e = bh_device_counter(&t.counter)) != cudaSuccess) return e;
    if ((e = bh_launch_trace(t, BH_PREC_FP32, false, bh_family_blocks(P), stream)) != cudaSuccess) return e;
    if ((e = sg_held_compare(accum, s->heldPix, s->heldPred, s->counters + 1, s->heldCap, t, s->counters + 4,
                             stream)) != cudaSuccess)
        return e;
    PostConsts pc{P.exposure, P.bloomStrength, P.bloomEnabled ? 1 : 0, P.swapRB};
    return bh_launch_post(out, accum, bloomB, bloomA, P.width, P.height, pc, stream);
}

}  // namespace

extern "C" {

int bhSurrogateParamCount(void) { return SgLayout::count(); }

cudaError_t bhSurrogateCreate(BHSurrogate** out, unsigned seed)
{
    if (!out) return cudaErrorInvalidValue;
    *out = nullptr;
    BHSurrogate* s = new BHSurrogate();
    SgState& S = s->S;
    const size_t pc = (size_t)SgLayout::count() * sizeof(float);
    cudaError_t e = cudaGetDevice(&S.device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->evFork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->evJoin, cudaEventDisableTiming);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.params), pc);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.grads), pc);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.adamM), pc);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.adamV), pc);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.W), kWCount * 2);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.Wt), kWCount * 2);
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.biasPacked), kBiasCount * sizeof(float));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.loss), 8 * sizeof(float));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&s->counters), 64);
    if (e == cudaSuccess) e = bh_tc_error_word(&S.err);
    // every set-up write goes on the network's stream, ordered with the kernels that follow
    if (e == cudaSuccess) e = cudaMemsetAsync(S.W, 0, kWCount * 2, s->stream);
    if (e != cudaSuccess) { freeAll(s); return e; }
    // Xavier-uniform weights, zero biases
    std::vector<float> p(SgLayout::count(), 0.f);
    std::mt19937 g(seed);
    for (int l = 0; l < 4; ++l)
    {
        const float lim = std::sqrt(6.f / 512.f);
        for (int i = 0; i < kHidW; ++i) p[SgLayout::w(l) + i] = uni(g, -lim, lim);
    }
    const float limH = std::sqrt(6.f / (256.f + 16.f));
    for (int i = 0; i < 16 * 256; ++i) p[SgLayout::w(4) + i] = uni(g, -limH, limH);
    *out = s;
    e = bhSurrogateSetParams(s, p.data());
    if (e != cudaSuccess) { freeAll(s); *out = nullptr; }
    return e;
}

void bhSurrogateDestroy(BHSurrogate* s)
{
    if (!s) return;
    cudaStreamSynchronize(s->stream);
    freeAll(s);
}

cudaError_t bhSurrogateGetParams(BHSurrogate* s, float* host)
{
    if (!s || !host) return cudaErrorInvalidValue;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(host, s->S.params, SgLayout::count() * sizeof(float), cudaMemcpyDeviceToHost);
}

cudaError_t bhSurrogateClone(BHSurrogate* src, BHSurrogate** out)
{
    if (!src || !out) return cudaErrorInvalidValue;
    *out = nullptr;
    std::vector<float> p((size_t)SgLayout::count());
    cudaError_t e = bhSurrogateGetParams(src, p.data());
    if (e != cudaSuccess) return e;
    BHSurrogate* c = nullptr;
    if ((e = bhSurrogateCreate(&c, 1u)) != cudaSuccess) return e;
    if ((e = bhSurrogateSetParams(c, p.data())) != cudaSuccess)
    {
        bhSurrogateDestroy(c);
        return e;
    }
    // the frame settings; scratch, statistics and the ray set stay the clone's own
    c->minProb = src->minProb; c->minConf = src->minConf; c->critBand = src->critBand;
    c->heldStride = src->heldStride;
    c->anchorStride = src->anchorStride; c->anchorNet = src->anchorNet;
    c->epsMax = src->epsMax; c->maxStep = src->maxStep; c->anchorSteps = src->anchorSteps;
    *out = c;
    return cudaSuccess;
}

cudaError_t bhSurrogateSetParams(BHSurrogate* s, const float* host)
{
    if (!s || !host) return cudaErrorInvalidValue;
    SgState& S = s->S;
    const size_t pc = (size_t)SgLayout::count() * sizeof(float);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.params, host, pc, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(S.adamM, 0, pc, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(S.adamV, 0, pc, s->stream);
    if (e == cudaSuccess) e = sg_pack_weights(S, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    S.step = 0;
    return e;
}

cudaError_t bhSurrogateFeatures(const float* in, void* features, int n, cudaStream_t stream)
{
    if (n < 0 || (n > 0 && (!in || !features))) return cudaErrorInvalidValue;
    return sg_features(in, features, n, stream);
}

cudaError_t bhSurrogateForward(BHSurrogate* s, const float* in, float* out, int n, int fused, cudaStream_t stream)
{
    if (!s || n < 0 || (n > 0 && (!in || !out))) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    SgState& S = s->S;
    if (fused)
    {
        SgInferArgs a{S.W, S.W + 4 * kHidW, S.biasPacked, in, out, (unsigned)n, S.err};
        return sg_infer_launch(a, nullptr, stream);
    }
    cudaError_t e = sg_forward_train(S, in, n, stream);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(out, S.Y, (size_t)n * 16 * sizeof(float), cudaMemcpyDeviceToDevice, stream);
}

cudaError_t bhSurrogateGradients(BHSurrogate* s, const float* in, const float* tgt, int n, float* gradsHost,
                                 float* lossHost)
{
    if (!s || !in || !tgt || n <= 0 || n % 128) return cudaErrorInvalidValue;
    SgState& S = s->S;
    // the caller's inputs may come from any stream: wait for all prior work
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = sg_gradients(S, in, tgt, n, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = checkErrWord(s);
    if (e == cudaSuccess && gradsHost)
        e = cudaMemcpy(gradsHost, S.grads, SgLayout::count() * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && lossHost)
    {
        float l[8];
        e = cudaMemcpy(l, S.loss, sizeof(l), cudaMemcpyDeviceToHost);
        for (int k = 0; k < 5; ++k) lossHost[k] = l[k] / (float)n;
    }
    return e;
}

cudaError_t bhSurrogateGenerate(BHSurrogate* s, long long rays, int views, unsigned seed)
{
    if (!s || rays <= 0 || views <= 0 || rays % views) return cudaErrorInvalidValue;
    SgState& S = s->S;
    const long long R = rays / views;
    if (R > (1 << 26)) return cudaErrorInvalidValue;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (S.dsN != rays)
    {
        if (S.dsIn) cudaFree(S.dsIn);
        if (S.dsTgt) cudaFree(S.dsTgt);
        S.dsIn = S.dsTgt = nullptr;
        S.dsN = 0;
        if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.dsIn), (size_t)rays * 8 * sizeof(float));
        if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&S.dsTgt), (size_t)rays * 8 * sizeof(float));
        if (e != cudaSuccess) return e;
    }
    float3* dirs = nullptr;
    BHProbe* rec = nullptr;
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&dirs), (size_t)R * sizeof(float3));
    if (e == cudaSuccess) e = bh_device_alloc(reinterpret_cast<void**>(&rec), (size_t)R * sizeof(BHProbe));
    std::mt19937 g(seed);
    for (int v = 0; v < views && e == cudaSuccess; ++v)
    {
        const int model = (int)(g() % 4u);
        float a = 0.f, q = 0.f;
        do { a = uni(g, -0.998f, 0.998f); q = uni(g, 0.f, 0.6f); } while (a * a + q * q > 0.98f);
        if (model == BH_SCHWARZSCHILD || model == BH_REISSNER_NORDSTROM) a = 0.f;
        if (model == BH_SCHWARZSCHILD || model == BH_KERR) q = 0.f;
        const float r = uni(g, 6.f, 60.f), incl = uni(g, 2.f, 88.f), az = uni(g, 0.f, 2.f * kPi);
        const float fov = uni(g, 30.f, 90.f);
        RenderParams P;
        P.width = 1920; P.height = 1080;
        applyHole(P, model, a, q);
        orbitCamera(P, az, (90.f - incl) * kPi / 180.f, r, fov);
        P.diskEnabled = 1; P.hotSpotsEnabled = (g() & 1u) ? 1 : 0;
        P.dPhi = 0.012f; P.maxSteps = 2000;
        P.accumMode = 0; P.sampleIndex = 0;
        bhSanitizeRenderParams(&P);
        float aN, qN, rN, iN;
        sceneInputs(P, aN, qN, rN, iN);
        const TraceParams tp = bh_frame_params(P, BH_OUT_PROBE, nullptr);
        float* in = S.dsIn + (size_t)v * R * 8;
        float* tgt = S.dsTgt + (size_t)v * R * 8;
        e = sg_make_rays(tp, aN, qN, rN, iN, seed * 0x9E3779B1u + (unsigned)v * 0x85EBCA77u, dirs, in, (int)R,
                         s->stream);
        if (e == cudaSuccess) e = bhProbeRays(rec, dirs, (int)R, P, BH_PREC_FP32, s->stream);
        if (e == cudaSuccess) e = sg_make_targets(rec, tp, tgt, (int)R, s->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (dirs) cudaFree(dirs);
    if (rec) cudaFree(rec);
    if (e == cudaSuccess) S.dsN = rays;
    return e;
}

cudaError_t bhSurrogateDataset(BHSurrogate* s, const float** in, const float** tgt, long long* n)
{
    if (!s) return cudaErrorInvalidValue;
    if (in) *in = s->S.dsIn;
    if (tgt) *tgt = s->S.dsTgt;
    if (n) *n = s->S.dsN;
    return cudaSuccess;
}

cudaError_t bhSurrogateTrain(BHSurrogate* s, int steps, int batch, float lr, unsigned seed, float* lossHistory)
{
    if (!s || steps < 0 || batch <= 0 || batch % 128 || !(lr > 0.f)) return cudaErrorInvalidValue;
    SgState& S = s->S;
    if (S.dsN <= 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaSuccess;
    if (batch > s->bCap)
    {
        if (s->bIn) cudaFree(s->bIn);
        if (s->bTgt) cudaFree(s->bTgt);
        s->bIn = s->bTgt = nullptr;
        s->bCap = 0;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->bIn), (size_t)batch * 8 * sizeof(float))) != cudaSuccess) return e;
        if ((e = bh_device_alloc(reinterpret_cast<void**>(&s->bTgt), (size_t)batch * 8 * sizeof(float))) != cudaSuccess) return e;
        s->bCap = batch;
    }
    float* hist = nullptr;
    if (steps > 0 && (e = bh_device_alloc(reinterpret_cast<void**>(&hist), (size_t)steps * 8 * sizeof(float))) != cudaSuccess) return e;
    for (int it = 0; it < steps && e == cudaSuccess; ++it)
    {
        const float t = steps > 1 ? (float)it / (float)(steps - 1) : 0.f;
        const float lrT = lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos(kPi * t)));
        e = sg_gather(S, seed * 0x9E3779B1u + (unsigned)it * 0x632BE5ABu, s->bIn, s->bTgt, batch, s->stream);
        if (e == cudaSuccess) e = sg_gradients(S, s->bIn, s->bTgt, batch, s->stream);
        if (e == cudaSuccess) e = sg_adam(S, lrT, s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hist + (size_t)it * 8, S.loss, 8 * sizeof(float), cudaMemcpyDeviceToDevice, s->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = checkErrWord(s);
    if (e == cudaSuccess && lossHistory && steps > 0)
    {
        std::vector<float> h((size_t)steps * 8);
        e = cudaMemcpy(h.data(), hist, h.size() * sizeof(float), cudaMemcpyDeviceToHost);
        for (int it = 0; it < steps; ++it)
            for (int k = 0; k < 5; ++k) lossHistory[it * 5 + k] = h[(size_t)it * 8 + k] / (float)batch;
    }
    if (hist) cudaFree(hist);
    return e;
}

cudaError_t bhSurrogateRender(BHSurrogate* s, uchar4* out, float4* accum, float4* bloomA, float4* bloomB,
                              const RenderParams* p, cudaStream_t stream)
{
    if (!s || !p) return cudaErrorInvalidValue;
    RenderParams P = *p;
    bhSanitizeRenderParams(&P);
    if (!out || !accum || (P.bloomEnabled && (!bloomA || !bloomB))) return cudaErrorInvalidValue;
    // the network's inputs assume an orbit camera; the anchored form without its cell
    // gate works in screen space and takes any camera
    const bool network = s->anchorStride < 2 || s->anchorNet;
    if (network && std::fabs(P.camRight.y) > 1e-4f) return cudaErrorInvalidValue;
    if (s->anchorStride < 2 && P.accumMode != 0) return cudaErrorInvalidValue;
    const size_t pixels = (size_t)P.width * P.height;
    cudaError_t e = ensureFrame(s, P.width, P.height);
    if (e != cudaSuccess) return e;
    s->lastPixels = (unsigned)pixels;
    if (s->anchorStride >= 2)
    {
        if ((e = cudaMemsetAsync(s->counters, 0, 64, stream)) != cudaSuccess) return e;
        if ((e = anchoredFrame(s, P, accum, stream)) != cudaSuccess) return e;
        return traceListAndPost(s, P, out, accum, bloomA, bloomB, stream);
    }
    s->lastAnchors = 0;
    CritKey key;
    key.model = P.model; key.maxSteps = P.maxSteps; key.M = P.M; key.a = P.aSpin; key.Q = P.Qc;
    key.dist = length3(P.camPos); key.cosIncl = P.camPos.y / key.dist; key.tanHalfFov = P.tanHalfFov;
    key.dPhi = P.dPhi;
    if (!s->critValid || !(key == s->critKey))
    {
        if ((e = criticalCurve(s, P, s->crit)) != cudaSuccess) return e;
        s->critKey = key;
        s->critValid = true;
    }
    SgState& S = s->S;
    SgFrame F{};
    F.tp = bh_frame_params(P, BH_OUT_ACCUM, accum);
    sceneInputs(P, F.aN, F.qN, F.rN, F.iN);
    std::memcpy(F.crit, s->crit, sizeof(F.crit));
    F.critBand = s->critBand;
    F.minProb = s->minProb;
    F.minConf = s->minConf;
    F.list = s->list;
    F.listCount = s->counters;
    F.traced = s->counters + 12;
    F.heldPix = s->heldPix;
    F.heldPred = s->heldPred;
    F.heldCount = s->counters + 1;
    F.heldCap = s->heldCap;
    F.heldStride = s->heldStride;
    F.frameSeed = ++s->frames;
    if ((e = cudaMemsetAsync(s->counters, 0, 64, stream)) != cudaSuccess) return e;
    SgInferArgs a{S.W, S.W + 4 * kHidW, S.biasPacked, nullptr, nullptr, (unsigned)pixels, S.err};
    if ((e = sg_infer_launch(a, &F, stream)) != cudaSuccess) return e;
    return traceListAndPost(s, P, out, accum, bloomA, bloomB, stream);
}

cudaError_t bhSurrogateFrameStats(BHSurrogate* s, BHSurrogateStats* st)
{
    if (!s || !st) return cudaErrorInvalidValue;
    unsigned c[16];
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(c, s->counters, sizeof(c), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = checkErrWord(s);
    if (e != cudaSuccess) return e;
    st->pixels = s->lastPixels;
    st->heldOut = c[4];
    st->heldOutOver1Lsb = c[5];
    float mx;
    std::memcpy(&mx, &c[6], sizeof(float));
    st->heldOutMaxAbs = mx;
    st->heldOutOverTol = c[7];
    st->anchors = s->lastAnchors;
    st->rk4Pixels = c[12] + std::min(c[1], s->heldCap) + s->lastAnchors;   // listed + held-out + anchors
    st->interpolated = c[8];
    st->rejectAnchors = c[9];
    st->rejectBound = c[10];
    st->rejectSky = c[11];
    st->skySampled = s->lastAnchors ? std::min(c[14], s->sampleCap) : 0u;
    st->anchorsIncomplete = s->lastAnchors ? c[15] : 0u;
    return cudaSuccess;
}

}  // extern "C"

extern "C" cudaError_t bhSurrogateDatasetCopy(BHSurrogate* s, float* in, float* tgt, long long first, long long count)
{
    if (!s || first < 0 || count < 0 || first + count > s->S.dsN) return cudaErrorInvalidValue;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess && in)
        e = cudaMemcpy(in, s->S.dsIn + first * 8, (size_t)count * 8 * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && tgt)
        e = cudaMemcpy(tgt, s->S.dsTgt + first * 8, (size_t)count * 8 * sizeof(float), cudaMemcpyDeviceToHost);
    return e;
}

extern "C" cudaError_t bhSurrogateSetAnchors(BHSurrogate* s, int stride, int useNetwork, float epsMax,
                                             float maxStep)
{
    if (!s || stride < 0 || stride == 1 || stride > 64 || !(epsMax > 0.f) || !(maxStep > 0.f && maxStep <= 1.f))
        return cudaErrorInvalidValue;
    s->anchorStride = stride;
    s->anchorNet = useNetwork != 0;
    s->epsMax = epsMax;
    s->maxStep = maxStep;
    return cudaSuccess;
}

extern "C" cudaError_t bhSurrogateSetAnchorSteps(BHSurrogate* s, int maxSteps)
{
    if (!s || maxSteps < 0) return cudaErrorInvalidValue;
    s->anchorSteps = maxSteps;
    return cudaSuccess;
}

extern "C" cudaError_t bhSurrogateSetGate(BHSurrogate* s, float minProb, float minConf, float critBand, int heldStride)
{
    if (!s || !(minProb >= 0.f && minProb <= 1.f) || !(minConf >= 0.f && minConf <= 1.f) ||
        !(critBand >= 0.f && critBand < 1.f) || heldStride < 0)
        return cudaErrorInvalidValue;
    s->minProb = minProb;
    s->minConf = minConf;
    s->critBand = critBand;
    s->heldStride = heldStride;
    return cudaSuccess;
}
