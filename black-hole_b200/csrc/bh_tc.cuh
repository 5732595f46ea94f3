// ---------------------------------------------------------------------------
// bh_tc.cuh -- sm_100a tensor-core building blocks for the lensing surrogate:
// tensor memory (TMEM) allocation, UMMA shared-memory and instruction
// descriptors, tcgen05.mma / commit / ld, TMA tiled loads and mbarriers.
//
// Conventions used by every kernel here:
//  * operands are BF16, K-major (the contraction index is contiguous), staged
//    in shared memory in the 128-byte-swizzle layout: a tile of R rows x 64
//    columns is R rows of 128 B, grouped in 8-row / 1024-B atoms, the 16-B
//    chunk index inside a row XOR-ed with (row % 8).  TMA with
//    CU_TENSOR_MAP_SWIZZLE_128B writes exactly this layout; kernels that
//    produce an operand themselves use sw128_offset();
//  * accumulators are FP32 in TMEM with M = 128: row m of the tile is TMEM
//    lane m, column n is TMEM column n;
//  * every wait is bounded: on time-out the waiting thread sets bit 0 of the
//    kernel's error word and reports failure, so the host gets an error code
//    instead of a hung context.
// No TMA multicast is used.
// ---------------------------------------------------------------------------
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bhtc {

// ---- shared-memory addresses and barriers -----------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// One suspending wait: the thread sleeps until the phase completes or about
// `hintNs` nanoseconds pass (no issue slots spent spinning).
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hintNs)
{
    uint32_t ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity), "r"(hintNs) : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete, at most `limitNs`
// nanoseconds.  On time-out sets bit 0 of *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* err,
                                          uint64_t limitNs = 2000000000ull)
{
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (true)
    {
        if (mbar_try_wait_sleep(bar, parity, 200000u)) return true;
        if (global_ns() - t0 > limitNs)
        {
            atomicOr(err, 1u);
            return false;
        }
    }
}

// ---- TMA ---------------------------------------------------------------------
// 2-D tiled load of the box at (x = inner element index, y = row) into
// shared memory, completing `bytes` on the barrier.  x * 2 B must be a
// multiple of 16 B (callers pass multiples of 64 elements).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, uint64_t* bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const void* tmap)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// generic-proxy writes to shared memory -> visible to the async proxy (MMA, TMA)
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- TMEM ----------------------------------------------------------------------
// Whole warp: allocate `cols` columns (power of two, >= 32); the base address
// is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- UMMA descriptors ---------------------------------------------------------
// Shared-memory matrix descriptor, K-major, 128-byte swizzle: rows 128 B
// apart, 8-row atoms 1024 B apart (SBO), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
           ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, A and B K-major,
// M = 128, N = n (multiple of 16, <= 256).
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T for one K = 16 slice; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                         bool accumulate)
{
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }"
        ::"r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive on `bar` once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

// Warp: 32 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Warp: 16 consecutive FP32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- CTA pairs (cluster of 2, tcgen05 cta_group::2) ---------------------------
// A pair computes M = 256 tiles: each CTA holds 128 rows of A and half of the
// N rows of B at the same shared-memory offsets; the leader (cluster rank 0)
// issues the MMAs, and each CTA's TMEM receives its own 128 rows.
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// shared::cluster address of the same variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa_shared(const void* p, uint32_t rank)
{
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_u32(p)), "r"(rank));
    return out;
}

__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// arrive (release, cluster scope) on a barrier given by its shared::cluster address
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t clusterAddr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(clusterAddr) : "memory");
}

// bounded wait with cluster-scope acquire (arrivals that come from the peer CTA)
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, unsigned* err,
                                                  uint64_t limitNs = 2000000000ull)
{
    const uint64_t t0 = global_ns();
    while (true)
    {
        uint32_t ok;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3; "
                     "selp.u32 %0, 1, 0, p; }"
                     : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity), "r"(200000u) : "memory");
        if (ok) return true;
        if (global_ns() - t0 > limitNs)
        {
            atomicOr(err, 1u);
            return false;
        }
    }
}

// 2-D tiled load into this CTA's shared memory, completing on a barrier of
// either CTA of the pair (its shared::cluster address); no multicast.
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const void* tmap, uint32_t barCluster, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(barCluster), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc_pair(uint32_t* slot, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free_pair(uint32_t base, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// Instruction descriptor for the pair: BF16 x BF16 -> FP32, K-major, M = 256.
__host__ __device__ constexpr uint32_t idesc_bf16_f32_m256(uint32_t n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((256u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_pair(uint32_t dTmem, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                              bool accumulate)
{
    asm volatile(
        "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p; }"
        ::"r"(dTmem), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive on the barrier at this offset in both CTAs of the pair once the MMAs
// issued so far have completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar)
{
    asm volatile(
        "{ .reg .b16 m; mov.b16 m, 3;\n\t"
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], m; }"
        ::"r"(smem_u32(bar)) : "memory");
}

// Byte offset of element (row, col) in a 128-row-group operand stored as
// 64-column blocks of `rows` x 128 B with the 128-byte swizzle.
__host__ __device__ __forceinline__ uint32_t sw128_offset(uint32_t row, uint32_t col, uint32_t rows)
{
    const uint32_t kb = col >> 6, c = col & 63u;
    const uint32_t chunk = (c >> 3) ^ (row & 7u);
    return kb * rows * 128u + (row >> 3) * 1024u + (row & 7u) * 128u + chunk * 16u + (c & 7u) * 2u;
}

}  // namespace bhtc
