// ---------------------------------------------------------------------------
// bh_gemm.cu -- BF16 tensor-core GEMM with FP32 accumulation (tcgen05 + TMA),
// the workhorse of the surrogate's training passes:
//
//     C[M x N] (=|+=) A[M x K] . B[N x K]^T (+ bias[N])
//
// A and B are row-major BF16 (K contiguous, i.e. both K-major), C is FP32.
// One CTA computes a 128 x BN tile over a K range: thread 0 streams 64-wide
// K blocks of A and B with TMA into a 4-stage ring, thread 32 issues the
// tcgen05.mma instructions (K = 16 each) into a TMEM accumulator, and the four
// warps read the accumulator back (one row per thread) for the epilogue.
// Split-K (grid.z > 1) accumulates into C with atomics.
// No counterpart in the reference (it has no learned component).
// ---------------------------------------------------------------------------
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include "bh_tc.cuh"
#include "bh_surrogate.h"

using namespace bhtc;

namespace {

constexpr int kStages = 4;
constexpr uint32_t kATileBytes = 128u * 128u;   // 128 rows x 64 BF16

template <int BN>
struct GemmSmem
{
    static constexpr uint32_t kBTileBytes = (uint32_t)BN * 128u;
    static constexpr uint32_t kStageBytes = kATileBytes + kBTileBytes;
    static constexpr uint32_t kBytes = kStages * kStageBytes + 1024u;   // + alignment slack
};

template <int BN>
__global__ void __launch_bounds__(128, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, float* __restrict__ C,
               int ldc, int M, int N, int kBlocks, int accumulate, const float* __restrict__ bias,
               unsigned* __restrict__ err)
{
    extern __shared__ uint8_t smemRaw[];
    __shared__ uint64_t full[kStages], empty[kStages], done;
    __shared__ uint32_t tmemSlot;
    constexpr uint32_t kCols = BN < 32 ? 32 : BN;
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN, kb0 = blockIdx.z * kBlocks;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(&done, 1);
        fence_barrier_init();
        tma_prefetch_desc(&tA);
        tma_prefetch_desc(&tB);
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(&tmemSlot, kCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmemSlot;

    if (threadIdx.x == 0)
    {   // TMA producer
        int issued = 0;
        for (int kb = 0; kb < kBlocks; ++kb, ++issued)
        {
            const int s = kb % kStages;
            if (kb >= kStages && !mbar_wait(&empty[s], ((kb / kStages) - 1) & 1, err)) break;
            uint8_t* st = smem + s * GemmSmem<BN>::kStageBytes;
            mbar_expect_tx(&full[s], GemmSmem<BN>::kStageBytes);
            tma_load_2d(st, &tA, &full[s], (kb0 + kb) * 64, m0);
            tma_load_2d(st + kATileBytes, &tB, &full[s], (kb0 + kb) * 64, n0);
        }
        // the CTA leaves only once its copies have landed, also after a timed-out wait
        // (bounded waits; on the normal path these phases are complete already)
        for (int kb = issued > kStages ? issued - kStages : 0; kb < issued; ++kb)
            if (!mbar_wait(&full[kb % kStages], (kb / kStages) & 1, err)) break;
    }
    else if (threadIdx.x == 32)
    {   // MMA issuer
        constexpr uint32_t idesc = idesc_bf16_f32(BN);
        for (int kb = 0; kb < kBlocks; ++kb)
        {
            const int s = kb % kStages;
            if (!mbar_wait(&full[s], (kb / kStages) & 1, err)) break;
            tc_fence_after();
            const uint32_t sa = smem_u32(smem + s * GemmSmem<BN>::kStageBytes);
            const uint32_t sb = sa + kATileBytes;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                mma_bf16(tmem, sdesc_sw128(sa + j * 32), sdesc_sw128(sb + j * 32), idesc, kb > 0 || j > 0);
            mma_commit(&empty[s]);
        }
        mma_commit(&done);
    }
    __syncwarp();

    // epilogue: warp w owns accumulator rows 32w .. 32w + 31
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&done, 0, err));
    tc_fence_after();
    if (ok)
    {
        const int row = m0 + warp * 32 + lane;
        const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
        constexpr int kChunk = BN < 32 ? 16 : 32;
#pragma unroll 1
        for (int c = 0; c < BN; c += kChunk)
        {
            __syncwarp();
            float v[32];
            if constexpr (kChunk == 16) tmem_ld16(tl + c, v);
            else tmem_ld32(tl + c, v);
            if (row < M)
            {
                float* out = C + (size_t)row * ldc;
#pragma unroll
                for (int i = 0; i < kChunk; ++i)
                {
                    const int n = n0 + c + i;
                    if (n < N)
                    {
                        float x = v[i] + ((bias && blockIdx.z == 0) ? __ldg(bias + n) : 0.f);
                        if (accumulate) atomicAdd(out + n, x);
                        else out[n] = x;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, kCols);
}

PFN_cuTensorMapEncodeTiled_v12000 encodeFn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn)
    {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <int BN>
cudaError_t launchGemm(const CUtensorMap& ta, const CUtensorMap& tb, float* C, int ldc, int M, int N, int K,
                       int splits, bool accumulate, const float* bias, unsigned* err, cudaStream_t s)
{
    auto k = tc_gemm_kernel<BN>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmSmem<BN>::kBytes);
    if (e != cudaSuccess) return e;
    const int kBlocks = K / 64 / splits;
    dim3 grid((M + 127) / 128, (N + BN - 1) / BN, splits);
    k<<<grid, 128, GemmSmem<BN>::kBytes, s>>>(ta, tb, C, ldc, M, N, kBlocks, (accumulate || splits > 1) ? 1 : 0,
                                             bias, err);
    return cudaGetLastError();
}

}  // namespace

cudaError_t bh_tensor_map_bf16(CUtensorMap* map, const void* base, int rows, int cols, int ld, int boxRows)
{
    auto fn = encodeFn();
    if (!fn) return cudaErrorNotSupported;
    if (((uintptr_t)base & 15u) || (ld * 2) % 16 || cols % 64 || boxRows < 1 || boxRows > 256)
        return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {64, (cuuint32_t)boxRows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t bh_gemm_bf16(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K,
                         int splits, bool accumulate, const float* bias, unsigned* err, cudaStream_t s)
{
    if (M < 1 || N < 1 || K < 64 || K % 64 || splits < 1 || (K / 64) % splits || !err) return cudaErrorInvalidValue;
    const int BN = N <= 16 ? 16 : N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
    CUtensorMap ta, tb;
    cudaError_t e = bh_tensor_map_bf16(&ta, A, M, K, lda, 128);
    if (e == cudaSuccess) e = bh_tensor_map_bf16(&tb, B, N, K, ldb, BN);
    if (e != cudaSuccess) return e;
    switch (BN)
    {
        case 16: return launchGemm<16>(ta, tb, C, ldc, M, N, K, splits, accumulate, bias, err, s);
        case 32: return launchGemm<32>(ta, tb, C, ldc, M, N, K, splits, accumulate, bias, err, s);
        case 64: return launchGemm<64>(ta, tb, C, ldc, M, N, K, splits, accumulate, bias, err, s);
        case 128: return launchGemm<128>(ta, tb, C, ldc, M, N, K, splits, accumulate, bias, err, s);
        default: return launchGemm<256>(ta, tb, C, ldc, M, N, K, splits, accumulate, bias, err, s);
    }
}

// ---------------------------------------------------------------------------
// device error word and the exported GEMM
// ---------------------------------------------------------------------------
namespace {
__device__ unsigned gTcError;

// Self-check of the bounded barrier waits: one thread waits for a phase of a
// barrier that nothing arrives at; the wait gives up after limitNs, sets bit 0
// of the error word and the kernel returns (no copy or tensor-memory state is
// involved, so nothing is left in flight).
__global__ void wait_probe_kernel(unsigned* err, unsigned long long limitNs)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait(&bar, 0, err, limitNs);
}
}

cudaError_t bh_tc_error_word(unsigned** out)
{
    return cudaGetSymbolAddress(reinterpret_cast<void**>(out), gTcError);
}

extern "C" cudaError_t bhTcGemm(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N,
                                int K, int splits, int accumulate, const float* bias, cudaStream_t stream)
{
    unsigned* err = nullptr;
    cudaError_t e = bh_tc_error_word(&err);
    if (e != cudaSuccess) return e;
    return bh_gemm_bf16(A, lda, B, ldb, C, ldc, M, N, K, splits, accumulate != 0, bias, err, stream);
}

extern "C" cudaError_t bhTcWaitProbe(int limitUs, cudaStream_t stream)
{
    if (limitUs < 1 || limitUs > 1000000) return cudaErrorInvalidValue;
    unsigned* err = nullptr;
    cudaError_t e = bh_tc_error_word(&err);
    if (e != cudaSuccess) return e;
    wait_probe_kernel<<<1, 32, 0, stream>>>(err, (unsigned long long)limitUs * 1000ull);
    return cudaGetLastError();
}

extern "C" cudaError_t bhTcErrorFlags(unsigned* flags)
{
    unsigned* err = nullptr;
    cudaError_t e = bh_tc_error_word(&err);
    if (e != cudaSuccess) return e;
    unsigned zero = 0;
    if ((e = cudaMemcpy(flags, err, sizeof(unsigned), cudaMemcpyDeviceToHost)) != cudaSuccess) return e;
    return cudaMemcpy(err, &zero, sizeof(unsigned), cudaMemcpyHostToDevice);
}
