// tc05.cuh — Blackwell (sm_100a) tensor-core primitives in inline PTX, for the
// learned warm start's network: tensor-memory allocation, tcgen05.mma
// (kind::f16: BF16 operands from shared memory, FP32 accumulators in tensor
// memory), completion through tcgen05.commit on an mbarrier, and tensor-memory
// loads into registers.
//
// Operand tiles use the no-swizzle canonical layout: core matrices of 8 rows x
// 16 bytes (8 BF16), stored contiguously (128 B). A tile of R rows and K columns
// (K a multiple of 8) keeps element (r, k) at byte core_off(r, k, K): core
// matrices adjacent along k are 128 B apart, 8-row groups K*16 B apart. The same
// bytes read as a K-major operand (rows = M or N, columns = K; leading offset
// 128 B, stride offset K*16 B) or as an MN-major operand with the roles swapped
// (columns = M or N, rows = K; stride offset 128 B between 8-column chunks,
// leading offset K*16 B between 8-row groups), which is what the weight
// gradients (sums over the sample rows) need.
#pragma once
#include <cstdint>

namespace sc {

constexpr int TC_SPIN_LIMIT = 1 << 24;     // mbarrier polls before a wait gives up

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__host__ __device__ constexpr uint32_t core_off(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (16-byte units), descriptor version 1 (bits 46-47)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand: a tile of K columns (core_off layout)
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, int K) { return umma_desc(saddr, 128, (uint32_t)K * 16); }
// MN-major operand: the same tile read with its columns as M (or N) and its rows as K
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t saddr, int K) { return umma_desc(saddr, (uint32_t)K * 16, 128); }

// instruction descriptor of kind::f16: A = B = BF16 (format 1), D = FP32
// (format 1), M x N, operand majors (0 = K-major, 1 = MN-major)
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N, int aMN, int bMN)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)aMN << 15) | ((uint32_t)bMN << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (tensor memory) = A * B^T (+ D when accumulate != 0); one thread issues
__device__ __forceinline__ void umma_bf16(uint32_t tmemD, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 :: "r"(tmemD), "l"(a), "l"(b), "r"(idesc), "r"(accumulate),
                    "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

// arrive once on the mbarrier when every earlier tcgen05.mma of this thread is done
__device__ __forceinline__ void umma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the mbarrier phase with parity `phase`; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase)
{
    for (int it = 0; it < TC_SPIN_LIMIT; it++)
    {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor cores' reads
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// CTA barrier between shared-memory operand writes and the MMAs that read them
__device__ __forceinline__ void tc_sync_for_mma()
{
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// warp 0 allocates `cols` tensor-memory columns (a power of two >= 32); the base
// address is written to *slot and returned to every thread
__device__ __forceinline__ uint32_t tmem_alloc(uint32_t* slot, uint32_t cols)
{
    if ((threadIdx.x >> 5) == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_addr(slot)), "r"(cols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *slot;
}

__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols)
{
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(cols) : "memory");
}

// this warp's 32 lanes (rows 32 w .. 32 w + 31 of an M = 128 accumulator): lane
// field of the tensor-memory address
__device__ __forceinline__ uint32_t tmem_lane_base(uint32_t base) { return base + ((uint32_t)((threadIdx.x >> 5) * 32) << 16); }

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr));
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

} // namespace sc
