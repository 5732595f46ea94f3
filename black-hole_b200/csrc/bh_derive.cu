// ---------------------------------------------------------------------------
// bh_derive.cu -- bhValidateAndDerive on the GPU for many black holes at once
// (one CTA per request), so batched views can be derived without a host round
// trip.
//
// Restates the reference's host derivation (src/metric.cuh:257-329, numeric
// ISCO metric.cuh:224-248) exactly as bh_params.cpp does: every operation is
// an IEEE single operation with contraction blocked (__fadd_rn, __fmul_rn,
// __fdiv_rn, __fsqrt_rn), in the same order, so the results are bit-identical
// to the host build.  acos and cos of the Kerr photon orbit are evaluated in
// double and rounded to float (correctly rounded; the host libm's float acos
// differs from that by one ulp on some inputs, a few ulps of rPhoton).
//
// The ISCO scan visits r = rStart, rStart + dr, ... as a running float sum --
// a sequential recurrence whose rounding fixes the visited radii.  Thread 0
// generates the exact sequence into shared memory 1024 values at a time; the
// CTA evaluates the circular-orbit energies of a chunk in parallel and keeps,
// per thread, the first minimum in visiting order; a final reduction picks
// the smallest energy, ties to the earliest radius, which is what the
// sequential strict "E < bestE" loop selects.
// ---------------------------------------------------------------------------
#include <cmath>
#include <cuda_runtime.h>
#include "bh_launch.h"

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 1024;
constexpr float kExtremal = 0.995f;
constexpr float kNakedCap = 2.25f;
constexpr float kSingCut = 0.05f;

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fq(float a) { return __fsqrt_rn(a); }

__device__ bool spinning(int m) { return m == BH_KERR || m == BH_KERR_NEWMAN; }
__device__ bool charged(int m) { return m == BH_REISSNER_NORDSTROM || m == BH_KERR_NEWMAN; }

__device__ float outerHorizon(float M, float a, float Q)
{
    const float d = fs(fs(fm(M, M), fm(a, a)), fm(Q, Q));
    return fa(M, fq(d < 0.f ? 0.f : d));
}

__device__ float innerHorizon(float M, float a, float Q)
{
    const float d = fs(fs(fm(M, M), fm(a, a)), fm(Q, Q));
    return fs(M, fq(d < 0.f ? 0.f : d));
}

__device__ float photonSphere(float M, float Q)
{
    const float d = fs(fm(fm(9.f, M), M), fm(fm(8.f, Q), Q));
    return fm(0.5f, fa(fm(3.f, M), fq(d < 0.f ? 0.f : d)));
}

__device__ float photonOrbitKerr(float M, float aStar)
{
    const float x = aStar > 1.f ? 1.f : (aStar < -1.f ? -1.f : aStar);
    const float ac = (float)acos((double)(-x));
    const float c = (float)cos((double)fm(2.f / 3.f, ac));
    return fm(fm(2.f, M), fa(1.f, c));
}

__device__ float photonOrbitKN(float M, float aStar, float q)
{
    const float rK = photonOrbitKerr(M, aStar);
    const float rS = photonSphere(M, fm(q, M));
    if (fabsf(aStar) < 1e-5f) return rS;
    float w = fm(q, q);
    w = w < 0.f ? 0.f : (w > 1.f ? 1.f : w);
    return fa(fm(fs(1.f, fm(0.35f, w)), rK), fm(fm(0.35f, w), rS));
}

__device__ float ergoRadius(float M, float Q)
{
    const float d = fs(fm(M, M), fm(Q, Q));
    return fa(M, fq(d < 0.f ? 0.f : d));
}

// specific energy of the circular orbit at r (metric.cuh:145-199 via bh_params.cpp)
__device__ bool orbitEnergy(float r, float M, float a, float Q, float& E)
{
    const float w2 = fs(fm(M, r), fm(Q, Q));
    if (w2 <= 0.f) return false;
    const float sw = fq(w2);
    const float Om = fd(sw, fa(fm(r, r), fm(a, sw)));
    if (Om <= 0.f) return false;
    const float r2 = fm(r, r);
    const float m2r = fs(fm(fm(2.f, M), r), fm(Q, Q));
    const float gtt = -fs(1.f, fd(m2r, r2));
    const float gtp = fd(fm(-a, m2r), r2);
    const float gpp = fa(fa(r2, fm(a, a)), fd(fm(fm(m2r, a), a), r2));
    const float den = -fa(fa(gtt, fm(fm(2.f, Om), gtp)), fm(fm(Om, Om), gpp));
    if (den <= 1e-6f) return false;
    E = fd(-fa(gtt, fm(Om, gtp)), fq(den));
    return true;
}

__global__ void __launch_bounds__(kThreads)
derive_kernel(BHDeriveRequest* __restrict__ req, BHDerived* __restrict__ out, int n)
{
    __shared__ float rs[kChunk];
    __shared__ float redE[kThreads];
    __shared__ int redK[kThreads];
    __shared__ int sCount;
    __shared__ float sNext;
    __shared__ BHDerived sD;
    __shared__ float sM, sA, sQ, sRp;
    const int i = blockIdx.x;
    if (i >= n) return;

    if (threadIdx.x == 0)
    {
        BHDeriveRequest R = req[i];
        float M = R.M, aStar = R.aStar, q = R.q;
        BHDerived d{0.f, 0.f, 1.f, 0.f, 1.5f, 1.f, 3.f, 0, 0};
        if (!(M > 0.f) || !isfinite(M)) { M = 0.5f; d.clamped = 1; }
        if (!isfinite(aStar)) { aStar = 0.f; d.clamped = 1; }
        if (!isfinite(q)) { q = 0.f; d.clamped = 1; }
        const float knob = R.allowNaked ? 1.5f : kExtremal;   // sqrt(2.25) = 1.5 exactly
        if (aStar < -knob) { aStar = -knob; d.clamped = 1; }
        if (aStar > knob) { aStar = knob; d.clamped = 1; }
        if (q < 0.f) { q = 0.f; d.clamped = 1; }
        if (q > knob) { q = knob; d.clamped = 1; }
        float aEff = spinning(R.model) ? aStar : 0.f;
        float qEff = charged(R.model) ? q : 0.f;
        const float bound = R.allowNaked ? kNakedCap : kExtremal;
        const float s2 = fa(fm(aEff, aEff), fm(qEff, qEff));
        if (s2 > bound)
        {
            const float k = fq(fd(bound, s2));
            aEff = fm(aEff, k);
            qEff = fm(qEff, k);
            if (spinning(R.model)) aStar = aEff;
            if (charged(R.model)) q = qEff;
            d.clamped = 1;
        }
        d.a = fm(aEff, M);
        d.Q = fm(qEff, M);
        if (fs(fs(fm(M, M), fm(d.a, d.a)), fm(d.Q, d.Q)) < 0.f) { d.naked = 1; d.rPlus = 0.f; d.rMinus = 0.f; }
        else { d.rPlus = outerHorizon(M, d.a, d.Q); d.rMinus = innerHorizon(M, d.a, d.Q); }
        d.rErgo = d.naked ? 0.f : ergoRadius(M, d.Q);
        if (spinning(R.model))
        {
            d.rPhoton = (R.model == BH_KERR_NEWMAN) ? photonOrbitKN(M, aEff, qEff) : photonOrbitKerr(M, aEff);
            if (d.rPlus > 0.f) { if (d.rPhoton < fm(d.rPlus, 1.02f)) d.rPhoton = fm(d.rPlus, 1.02f); }
            else if (d.rPhoton < fm(fm(kSingCut, M), 2.f)) d.rPhoton = fm(3.f, M);
        }
        else
        {
            d.rPhoton = photonSphere(M, d.Q);
            if (d.naked && !(d.rPhoton > 0.f)) d.rPhoton = fm(3.f, M);
        }
        // ISCO scan set-up (iscoRadius)
        const bool horizon = fs(fs(fm(M, M), fm(d.a, d.a)), fm(d.Q, d.Q)) >= 0.f;
        const float rp = horizon ? outerHorizon(M, d.a, d.Q) : fm(kSingCut, M);
        sRp = rp;
        sNext = rp > 1e-6f ? fm(rp, 1.02f) : fm(0.5f, M);
        sD = d;
        sM = M; sA = aStar; sQ = q;
        req[i].M = M; req[i].aStar = aStar; req[i].q = q;
    }
    __syncthreads();
    const float M = sM, a = sD.a, Q = sD.Q;
    const float rEnd = fm(12.f, M), dr = fm(0.001f, M);
    float bestE = 1e30f;
    int bestK = 0x7fffffff;
    int base = 0;
    while (true)
    {
        if (threadIdx.x == 0)
        {   // the exact visiting sequence of `for (r = rStart; r <= rEnd; r += dr)`
            float r = sNext;
            int c = 0;
            while (c < kChunk && r <= rEnd) { rs[c++] = r; r = fa(r, dr); }
            sCount = c;
            sNext = r;
        }
        __syncthreads();
        const int c = sCount;
        for (int k = threadIdx.x; k < c; k += kThreads)
        {
            float E;
            if (orbitEnergy(rs[k], M, a, Q, E) && E < bestE) { bestE = E; bestK = base + k; }
        }
        base += c;
        __syncthreads();
        if (c < kChunk) break;
    }
    redE[threadIdx.x] = bestE;
    redK[threadIdx.x] = bestK;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
        {
            const float e2 = redE[threadIdx.x + s];
            const int k2 = redK[threadIdx.x + s];
            if (e2 < redE[threadIdx.x] || (e2 == redE[threadIdx.x] && k2 < redK[threadIdx.x]))
            {
                redE[threadIdx.x] = e2;
                redK[threadIdx.x] = k2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        const float rp = sRp;
        float best;
        if (redK[0] != 0x7fffffff)
        {   // radius of the winning index: replay the same running sum
            float r = rp > 1e-6f ? fm(rp, 1.02f) : fm(0.5f, M);
            for (int k = 0; k < redK[0]; ++k) r = fa(r, dr);
            best = r;
        }
        else
        {
            best = (fm(6.f, M) > fm(rp, 1.5f)) ? fm(6.f, M) : fm(rp, 1.5f);
        }
        const float floorR = rp > 1e-6f ? fm(rp, 1.15f) : fm(0.5f, M);
        BHDerived d = sD;
        d.rIsco = best > floorR ? best : floorR;
        out[i] = d;
    }
}

}  // namespace

extern "C" cudaError_t bhDeriveBatch(BHDeriveRequest* requests, BHDerived* out, int n, cudaStream_t stream)
{
    if (n < 0 || (n > 0 && (!requests || !out))) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    derive_kernel<<<n, kThreads, 0, stream>>>(requests, out, n);
    return cudaGetLastError();
}
