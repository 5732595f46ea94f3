// ---------------------------------------------------------------------------
// bh_sg_infer.cu -- fused, persistent inference of the lensing surrogate on
// the tensor cores: Fourier features -> 4 x (256 x 256 GEMM + GELU) -> head,
// one launch, activations never leave shared memory.
//
// CTA pairs (clusters of 2, tcgen05 cta_group::2): a pair computes 256-row
// tiles, 128 rows in each CTA, with M = 256 MMAs issued by the leader (cluster
// rank 0); each CTA streams only its half of every weight chunk (128 of the
// 256 output rows), so the per-SM weight stream is half that of a single-SM
// 128-row tile.  Each CTA = 18 warps, one CTA per SM (~202 KB shared memory,
// all 512 TMEM columns, allocated for the pair):
//   warps 0-7   epilogue group 0: this CTA's 128 rows of tile pair A0; warp w
//               reads TMEM lane quarter w % 4 and column half w / 4
//   warps 8-15  epilogue group 1: the same for A1
//   warp 16     TMA producer: this CTA's 128 x 64 weight chunk (16 KB) into a
//               5-stage ring, completing on the leader's barrier
//   warp 17     MMA issuer (leader only): tcgen05.mma M=256 N=256 K=16,
//               accumulators in both CTAs' TMEM (group g owns columns 256g ..)
// The two groups ping-pong: while group 0 turns layer l's accumulator into
// layer l+1's BF16 operand (bias, GELU, 128-byte-swizzled stores), the tensor
// core runs group 1's layer l, and the other way round.  Producers and the
// issuer walk the same chunk sequence per tile pair:
//   for l in 0..3: for g in 0..1: for kb in 0..3: W_l[rank half of rows, kb cols]
//   then for g in 0..1: for kb in 0..3: W_head (32 rows, 16 per CTA, the upper 16 zero)
// Barriers: full[s] (leader: both CTAs' chunk bytes), empty[s] and accFull[g]
// (multicast MMA commits to both CTAs), aReady[g] (leader: 512 epilogue
// arrivals from both CTAs -- the operand of the next layer is in shared memory
// and the accumulator is free).  All waits are bounded (bh_tc.cuh).
// ---------------------------------------------------------------------------
#include <cuda.h>
#include <cuda_bf16.h>
#include "bh_integrate.cuh"
#include "bh_post.cuh"
#include "bh_sg_infer.h"
#include "bh_sg_net.cuh"
#include "bh_tc.cuh"

using namespace bhtc;
using namespace bhsg;

namespace {

constexpr int kRing = 5;
constexpr uint32_t kTileBytes = 128u * 256u * 2u;       // one group's operand: 128 rows x 256 BF16
constexpr uint32_t kChunkBytes = 128u * 128u;           // 128 weight rows x 64 BF16
constexpr uint32_t kHeadChunkBytes = 16u * 128u;        // 16 head rows x 64 BF16
constexpr int kThreads = 576;
constexpr int kProducerWarp = 16, kMmaWarp = 17;
constexpr uint32_t kSmemBytes = 2 * kTileBytes + kRing * kChunkBytes + 1024;

struct Bars
{
    uint64_t full[kRing], empty[kRing], aReady[2], accFull[2], done;
    uint32_t tmem;
};

// 8 packed BF16 values -> the operand row `row`, columns col .. col + 7
__device__ __forceinline__ void st_chunk(uint8_t* tile, uint32_t row, uint32_t col, uint4 v)
{
    *reinterpret_cast<uint4*>(tile + sw128_offset(row, col, 128)) = v;
}

// (acc + bias) / 2 in one packed FP32 FMA (bias2 = bias / 2; exact halving),
// BF16 rounding, GELU from the halved input (bit-identical to gelu2)
__device__ __forceinline__ uint32_t pack_gelu(float a, float b, float ba2, float bb2)
{
    const float2 z = __ffma2_rn(make_float2(a, b), make_float2(0.5f, 0.5f), make_float2(ba2, bb2));
    __nv_bfloat162 h = gelu2_half(__floats2bfloat162_rn(z.x, z.y));
    return *reinterpret_cast<uint32_t*>(&h);
}

// Network inputs of one ray.
struct RayIn
{
    float x[kIn];
    f3 dirW;          // world direction (frame mode)
};

__device__ __forceinline__ void frame_inputs(const SgFrame& F, unsigned pix, RayIn& r)
{
    const TraceParams& P = F.tp;
    const int py = (int)(pix / (unsigned)P.W), px = (int)(pix - (unsigned)py * (unsigned)P.W);
    const float fx = __fdiv_rn(add_x((float)px, P.jx), (float)P.W);
    const float fy = __fdiv_rn(add_x((float)py, P.jy), (float)P.H);
    const f3 d = camera_ray(P, fx, fy);
    r.dirW = d;
    r.x[0] = d.x * P.camRight.x + d.y * P.camRight.y + d.z * P.camRight.z;
    r.x[1] = d.x * P.camUp.x + d.y * P.camUp.y + d.z * P.camUp.z;
    r.x[2] = d.x * P.camFwd.x + d.y * P.camFwd.y + d.z * P.camFwd.z;
    r.x[3] = F.aN; r.x[4] = F.qN; r.x[5] = F.rN; r.x[6] = F.iN;
}

// Is the pixel within the critical band (|rho / rho_c(psi) - 1| < band)?
__device__ __forceinline__ bool near_critical(const SgFrame& F, float cx, float cy)
{
    const float rho = sqrtf(cx * cx + cy * cy);
    float psi = atan2f(cy, cx) * (0.159154943f * (float)kCritBins);
    if (psi < 0.f) psi += (float)kCritBins;
    int b0 = (int)psi;
    const float t = psi - (float)b0;
    b0 = min(b0, kCritBins - 1);
    const int b1 = (b0 + 1) % kCritBins;
    const float rc = F.crit[b0] * (1.f - t) + F.crit[b1] * t;
    return fabsf(rho - rc) < F.critBand * rc;
}

// Per-ray decision after the head: shade from the surrogate or queue for RK4.
__device__ void frame_output(const SgFrame& F, unsigned pix, bool valid, const RayIn& r, const float* y)
{
    bool fallback = false, held = false;
    f3 hdr = v3(0.f, 0.f, 0.f);
    if (valid)
    {
        const float m = fmaxf(y[0], fmaxf(y[1], y[2]));
        const float e0 = __expf(y[0] - m), e1 = __expf(y[1] - m), e2 = __expf(y[2] - m);
        const float inv = 1.f / (e0 + e1 + e2);
        const float p0 = e0 * inv, p1 = e1 * inv;
        const int cls = (p0 >= p1 && p0 >= e2 * inv) ? kClsEscaped : (p1 >= e2 * inv ? kClsCaptured : kClsDisk);
        const float pc = cls == kClsEscaped ? p0 : (cls == kClsCaptured ? p1 : e2 * inv);
        const float conf = 1.f / (1.f + __expf(-y[kOConf]));
        // screen-plane position of the ray (tan-space, camera basis)
        const float cx = r.x[0] / r.x[2], cy = r.x[1] / r.x[2];
        fallback = cls == kClsDisk || pc < F.minProb || conf < F.minConf || near_critical(F, cx, cy);
        if (!fallback)
        {
            if (cls == kClsEscaped)
            {
                f3 e = v3(r.x[0] + y[kOEsc], r.x[1] + y[kOEsc + 1], r.x[2] + y[kOEsc + 2]);
                const TraceParams& P = F.tp;
                f3 w = v3(P.camRight.x * e.x + P.camUp.x * e.y + P.camFwd.x * e.z,
                          P.camRight.y * e.x + P.camUp.y * e.y + P.camFwd.y * e.z,
                          P.camRight.z * e.x + P.camUp.z * e.y + P.camFwd.z * e.z);
                hdr = sky_color(w, P.gCam);
                if (!isfinite(hdr.x) || !isfinite(hdr.y) || !isfinite(hdr.z)) hdr = v3(0.f, 0.f, 0.f);
            }
            // held-out check: every heldStride-th surrogate pixel (hashed per frame) is also traced
            unsigned h = pix * 0x9E3779B1u ^ (F.frameSeed * 0x85EBCA77u);
            h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12;
            held = F.heldStride > 0 && (h % (unsigned)F.heldStride) == 0u;
            float4* acc = reinterpret_cast<float4*>(F.tp.out);
            acc[pix] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
        }
    }
    // appends to the RK4 list (fallback pixels; the held-out sample follows the list,
    // sg_append_held): a warp's lanes are 32 consecutive pixels of a row, and a warp
    // with any claims a whole 32-entry group (BH_PIX_SKIP where a lane has none), so
    // each tracing warp takes one coherent row segment
    const unsigned lane = threadIdx.x & 31u;
    const bool push = fallback;
    const unsigned m = __ballot_sync(0xffffffffu, push);
    if (m)
    {
        unsigned base = 0;
        if (lane == 0)
        {
            base = atomicAdd(F.listCount, 32u);
            atomicAdd(F.traced, (unsigned)__popc(m));
        }
        base = __shfl_sync(0xffffffffu, base, 0);
        F.list[base + lane] = push ? pix : BH_PIX_SKIP;
    }
    const unsigned mh = __ballot_sync(0xffffffffu, held);
    if (mh)
    {
        unsigned base = 0;
        if (lane == (unsigned)(__ffs(mh) - 1)) base = atomicAdd(F.heldCount, (unsigned)__popc(mh));
        base = __shfl_sync(0xffffffffu, base, __ffs(mh) - 1);
        if (held)
        {
            const unsigned k = base + __popc(mh & ((1u << lane) - 1u));
            if (k < F.heldCap)
            {
                F.heldPix[k] = pix;
                F.heldPred[k] = make_float4(hdr.x, hdr.y, hdr.z, 1.f);
            }
        }
    }
}

template <bool FRAME>
__global__ void __launch_bounds__(kThreads, 1)
sg_infer_kernel(const __grid_constant__ CUtensorMap tW, const __grid_constant__ CUtensorMap tH,
                const __grid_constant__ SgFrame F, const float* __restrict__ bias, const float* __restrict__ rawIn,
                float* __restrict__ rawOut, unsigned n, unsigned iters, unsigned* __restrict__ err)
{
    extern __shared__ uint8_t smemRaw[];
    __shared__ Bars B;
    __shared__ __align__(16) float sBias[kHidden * kWidth + kOut];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    uint8_t* tiles = smem;                       // 2 x 64 KB operands (this CTA's 128 rows of each group)
    uint8_t* ring = smem + 2 * kTileBytes;       // weight chunks: this CTA's half of the N rows
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();        // 0: leader (issues the MMAs), 1: peer
    const unsigned pair = blockIdx.x >> 1, pairs = gridDim.x >> 1;

    // hidden-layer biases are kept halved (the epilogue forms (acc + bias) / 2); head biases as they are
    for (int i = threadIdx.x; i < kHidden * kWidth + kOut; i += kThreads)
        sBias[i] = i < kHidden * kWidth ? 0.5f * bias[i] : bias[i];
    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kRing; ++s) { mbar_init(&B.full[s], 1); mbar_init(&B.empty[s], 1); }
        for (int g = 0; g < 2; ++g) { mbar_init(&B.aReady[g], 512); mbar_init(&B.accFull[g], 1); }
        mbar_init(&B.done, 1);
        fence_barrier_init();
    }
    if (warp == kProducerWarp)
    {
        __syncwarp();
        tmem_alloc_pair(&B.tmem, 512);
    }
    tc_fence_before();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem = B.tmem;

    if (warp == kProducerWarp)
    {
        if (lane == 0)
        {   // ---- TMA producer (both CTAs): this CTA's half of every weight chunk ----
            tma_prefetch_desc(&tW);
            tma_prefetch_desc(&tH);
            uint32_t q = 0;
            bool ok = true;
            for (unsigned it = 0; it < iters && ok; ++it)
                for (int l = 0; l <= kHidden && ok; ++l)
                    for (int g = 0; g < 2 && ok; ++g)
                        for (int kb = 0; kb < 4 && ok; ++kb, ++q)
                        {
                            const uint32_t s = q % kRing;
                            if (q >= kRing && !(ok = mbar_wait_cluster(&B.empty[s], ((q / kRing) - 1) & 1, err)))
                                break;
                            uint8_t* dst = ring + s * kChunkBytes;
                            const uint32_t leaderFull = mapa_shared(&B.full[s], 0);
                            const uint32_t bytes = l < kHidden ? kChunkBytes : kHeadChunkBytes;
                            if (rank == 0) mbar_expect_tx(&B.full[s], 2u * bytes);
                            if (l < kHidden) tma_load_2d_pair(dst, &tW, leaderFull, kb * 64, l * 256 + (int)rank * 128);
                            else tma_load_2d_pair(dst, &tH, leaderFull, kb * 64, (int)rank * kOut);
                        }
            // drain: the last loads (of both CTAs, which complete on the leader's barriers)
            // must land before the pair may exit -- also after a timed-out wait
            if (rank == 0 && q > 0)
                for (uint32_t k = (q > kRing ? q - kRing : 0); k < q; ++k)
                    if (!mbar_wait_cluster(&B.full[k % kRing], (k / kRing) & 1, err)) break;
        }
    }
    else if (warp == kMmaWarp)
    {
        if (lane == 0 && rank == 0)
        {   // ---- MMA issuer (leader): M = 256 over the pair ----
            const uint32_t idH = idesc_bf16_f32_m256(256), idHead = idesc_bf16_f32_m256(2 * kOut);
            uint32_t q = 0, phA[2] = {0, 0};
            bool ok = true;
            for (unsigned it = 0; it < iters && ok; ++it)
                for (int l = 0; l <= kHidden && ok; ++l)
                    for (int g = 0; g < 2 && ok; ++g)
                    {
                        if (!(ok = mbar_wait_cluster(&B.aReady[g], phA[g], err))) break;
                        phA[g] ^= 1u;
                        tc_fence_after();
                        const uint32_t aBase = smem_u32(tiles + g * kTileBytes);
                        const uint32_t d = tmem + (uint32_t)g * 256u;
                        for (int kb = 0; kb < 4 && ok; ++kb, ++q)
                        {
                            const uint32_t s = q % kRing;
                            if (!(ok = mbar_wait_cluster(&B.full[s], (q / kRing) & 1, err))) break;
                            tc_fence_after();
                            const uint32_t bBase = smem_u32(ring + s * kChunkBytes);
                            const uint32_t aBlk = aBase + (uint32_t)kb * 16384u;
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                mma_bf16_pair(d, sdesc_sw128(aBlk + j * 32), sdesc_sw128(bBase + j * 32),
                                              l < kHidden ? idH : idHead, kb > 0 || j > 0);
                            mma_commit_pair(&B.empty[s]);
                        }
                        mma_commit_pair(&B.accFull[g]);
                    }
            // every MMA issued has completed before the pair frees its TMEM (also
            // after a timed-out wait); the commit arrives on both CTAs' barriers
            mma_commit_pair(&B.done);
        }
        if (lane == 0) mbar_wait_cluster(&B.done, 0, err);
    }
    else
    {   // ---- epilogue groups ----
        const int g = warp >> 3, wq = warp & 3, half = (warp >> 2) & 1;
        const uint32_t row = (uint32_t)(wq * 32 + lane);
        uint8_t* tile = tiles + g * kTileBytes;
        const uint32_t tl = tmem + (uint32_t)g * 256u + ((uint32_t)(wq * 32) << 16);
        const uint32_t aReadyLeader = mapa_shared(&B.aReady[g], 0);
        uint32_t phF = 0;
        bool ok = true;
        for (unsigned it = 0; it < iters && ok; ++it)
        {
            const unsigned superTile = (it * pairs + pair) * 2u + (unsigned)g;
            const unsigned rid = superTile * 256u + rank * 128u + row;
            const bool valid = rid < n;
            RayIn r;
            if constexpr (FRAME)
            {
                const unsigned pix = valid ? (F.evalPix ? __ldg(F.evalPix + rid) : rid) : 0u;
                frame_inputs(F, pix, r);
            }
            else
            {
#pragma unroll
                for (int k = 0; k < kIn; ++k) r.x[k] = valid ? __ldg(rawIn + (size_t)rid * 8 + k) : 0.f;
            }
#pragma unroll 4
            for (int j = half * 16; j < half * 16 + 16; ++j)
                st_chunk(tile, row, (uint32_t)j * 8u, sg_feature_chunk(r.x, j));
            fence_async_smem();
            mbar_arrive_cluster(aReadyLeader);

            for (int l = 0; l < kHidden && ok; ++l)
            {
                ok = __all_sync(0xffffffffu, mbar_wait_cluster(&B.accFull[g], phF, err));
                phF ^= 1u;
                if (!ok) break;
                tc_fence_after();
                const float* bl = sBias + l * kWidth;
#pragma unroll 1
                for (int c = half * 128; c < half * 128 + 128; c += 32)
                {
                    float v[32];
                    tmem_ld32(tl + (uint32_t)c, v);
#pragma unroll
                    for (int q4 = 0; q4 < 4; ++q4)
                    {
                        uint4 o;
                        const int b = c + q4 * 8;
                        const float4 b0 = *reinterpret_cast<const float4*>(bl + b);
                        const float4 b1 = *reinterpret_cast<const float4*>(bl + b + 4);
                        o.x = pack_gelu(v[q4 * 8 + 0], v[q4 * 8 + 1], b0.x, b0.y);
                        o.y = pack_gelu(v[q4 * 8 + 2], v[q4 * 8 + 3], b0.z, b0.w);
                        o.z = pack_gelu(v[q4 * 8 + 4], v[q4 * 8 + 5], b1.x, b1.y);
                        o.w = pack_gelu(v[q4 * 8 + 6], v[q4 * 8 + 7], b1.z, b1.w);
                        st_chunk(tile, row, (uint32_t)b, o);
                    }
                }
                tc_fence_before();
                fence_async_smem();
                mbar_arrive_cluster(aReadyLeader);
            }
            if (!ok) break;
            ok = __all_sync(0xffffffffu, mbar_wait_cluster(&B.accFull[g], phF, err));
            phF ^= 1u;
            if (!ok) break;
            tc_fence_after();
            if (half == 0)
            {   // the head's 16 columns: read and used by the first column half only
                float y[kOut];
                tmem_ld16(tl, y);
                tc_fence_before();
#pragma unroll
                for (int k = 0; k < kOut; ++k) y[k] += sBias[kHidden * kWidth + k];
                if constexpr (FRAME)
                {
                    if (F.gateOut)
                    {   // cell gate of an anchored frame: P(escaped without the disk),
                        // P(captured without the disk)
                        if (valid)
                        {
                            const float m = fmaxf(y[0], fmaxf(y[1], y[2]));
                            const float e0 = __expf(y[0] - m), e1 = __expf(y[1] - m), e2 = __expf(y[2] - m);
                            const float inv = 1.f / (e0 + e1 + e2);
                            F.gateOut[rid] = make_float2(e0 * inv, e1 * inv);
                        }
                    }
                    else frame_output(F, rid, valid, r, y);
                }
                else if (valid)
                {
#pragma unroll
                    for (int k = 0; k < kOut; ++k) rawOut[(size_t)rid * kOut + k] = y[k];
                }
            }
        }
    }
    tc_fence_before();
    cluster_sync();
    if (warp == kProducerWarp)
    {
        __syncwarp();
        tmem_free_pair(tmem, 512);
    }
}

}  // namespace

cudaError_t sg_infer_launch(const SgInferArgs& a, const SgFrame* frame, cudaStream_t s)
{
    if (a.n == 0) return cudaSuccess;
    CUtensorMap tW, tH;
    cudaError_t e = bh_tensor_map_bf16(&tW, a.Whidden, kHidden * kWidth, kWidth, kWidth, 128);
    // the head as 32 rows (16 per CTA of a pair; rows 16..31 are zero in the weight buffer)
    if (e == cudaSuccess) e = bh_tensor_map_bf16(&tH, a.Whead, 2 * kOut, kWidth, kWidth, kOut);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const unsigned superTiles = (a.n + 255u) / 256u;            // 256 rays per pair and group
    const unsigned want = (superTiles + 1u) / 2u;               // pair-iterations of work
    const unsigned pairs = std::max(1u, std::min<unsigned>((unsigned)sms / 2u, want));
    const unsigned iters = (want + pairs - 1u) / pairs;
    SgFrame F{};
    if (frame) F = *frame;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(2u * pairs);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (frame)
    {
        auto k = sg_infer_kernel<true>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes))) return e;
        e = cudaLaunchKernelEx(&cfg, k, tW, tH, F, a.bias, (const float*)nullptr, (float*)nullptr, a.n, iters, a.err);
    }
    else
    {
        auto k = sg_infer_kernel<false>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes))) return e;
        e = cudaLaunchKernelEx(&cfg, k, tW, tH, F, a.bias, a.rawIn, a.rawOut, a.n, iters, a.err);
    }
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

namespace {

__global__ void held_compare_kernel(const float4* __restrict__ accum, const unsigned* __restrict__ heldPix,
                                    const float4* __restrict__ heldPred, const unsigned* __restrict__ heldCount,
                                    unsigned heldCap, int W, float exposure, int swapRB, unsigned* __restrict__ stats)
{
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned n = min(*heldCount, heldCap);
    if (k >= n) return;
    const unsigned pix = heldPix[k];
    const int py = (int)(pix / (unsigned)W), px = (int)(pix - (unsigned)py * (unsigned)W);
    const float4 a = accum[pix], b = heldPred[k];
    const float d = fmaxf(fabsf(a.x - b.x), fmaxf(fabsf(a.y - b.y), fabsf(a.z - b.z)));
    PostConsts pc{exposure, 0.f, 0, swapRB};
    const uchar4 ua = finalize_pixel(v3(a.x, a.y, a.z), v3(0.f, 0.f, 0.f), pc, px, py);
    const uchar4 ub = finalize_pixel(v3(b.x, b.y, b.z), v3(0.f, 0.f, 0.f), pc, px, py);
    const int lsb = max(abs((int)ua.x - (int)ub.x), max(abs((int)ua.y - (int)ub.y), abs((int)ua.z - (int)ub.z)));
    atomicAdd(stats + 0, 1u);
    if (lsb > 1) atomicAdd(stats + 1, 1u);
    atomicMax(stats + 2, __float_as_uint(d));
    const float ref = fmaxf(fabsf(a.x), fmaxf(fabsf(a.y), fabsf(a.z)));
    if (d > 1e-3f * fmaxf(ref, 1e-3f)) atomicAdd(stats + 3, 1u);
}

__global__ void append_held_kernel(unsigned* __restrict__ list, const unsigned* __restrict__ listCount,
                                   const unsigned* __restrict__ heldPix, const unsigned* __restrict__ heldCount,
                                   unsigned heldCap, unsigned* __restrict__ total)
{
    const unsigned base = *listCount, n = min(*heldCount, heldCap);
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        list[base + k] = heldPix[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) *total = base + n;
}

}  // namespace

cudaError_t sg_append_held(unsigned* list, const unsigned* listCount, const unsigned* heldPix,
                           const unsigned* heldCount, unsigned heldCap, unsigned* total, cudaStream_t s)
{
    append_held_kernel<<<32, 256, 0, s>>>(list, listCount, heldPix, heldCount, heldCap, total);
    return cudaGetLastError();
}

cudaError_t sg_held_compare(const float4* accum, const unsigned* heldPix, const float4* heldPred,
                            const unsigned* heldCount, unsigned heldCap, const TraceParams& tp, unsigned* stats,
                            cudaStream_t s)
{
    if (heldCap == 0) return cudaSuccess;
    held_compare_kernel<<<(heldCap + 255) / 256, 256, 0, s>>>(accum, heldPix, heldPred, heldCount, heldCap, tp.W,
                                                              tp.exposure, tp.swapRB, stats);
    return cudaGetLastError();
}
