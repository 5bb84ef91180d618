// tc05_ptx.cuh -- thin inline-PTX wrappers for the sm_100a features the
// tcgen05 kernels use: mbarriers, TMA tensor loads, TMEM allocation,
// tcgen05.mma / commit / ld, and the shared-memory matrix descriptor.
#pragma once

#include <cstdint>
#include <cuda.h>

namespace kami {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bulk copy (TMA engine, no tensor map) of `bytes` from global to this CTA's
// shared memory, completing on `bar` by bytes.  dst and src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: returns false when `limit_ns` elapsed without the phase
// completing (the caller records an error and leaves instead of hanging).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = globaltimer_ns();
    while (true)
    {
        if (mbar_try_wait(bar, parity))
            return true;
        if (globaltimer_ns() - t0 > limit_ns)
            return false;
    }
}

// ---- TMA ------------------------------------------------------------------
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
                 "[%2];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}

// Tiled store shared -> global (elements outside the tensor are not written),
// tracked in the issuing thread's bulk groups.  The shared tile must have been
// made visible to the async proxy first (fence_proxy_async_smem by each writer).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most N of this thread's bulk groups still reading shared memory
template <int N> __device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// all of this thread's bulk groups complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---- TMEM -----------------------------------------------------------------
// Whole warp.  Writes the allocated TMEM base address to *dst_smem.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- MMA ------------------------------------------------------------------
// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::f16 (FP16/BF16 in, FP32 acc)
__device__ __forceinline__ void mma_f16_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                           uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::i8 (signed 8-bit in,
// INT32 accumulator)
__device__ __forceinline__ void mma_i8_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

// Arrive on `bar` once all previously issued tcgen05.mma of this thread
// have completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 bit, 16 consecutive columns: thread t of the warp receives
// lane (base lane + t), columns [col, col+16).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                 "[%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Order the uses of 16 registers filled by tcgen05.ld after a preceding
// tcgen05.wait::ld: the empty statement reads and rewrites them, so the
// compiler cannot hoist their uses above it.
__device__ __forceinline__ void tmem_regs_ready(uint32_t (&v)[16])
{
    asm volatile(""
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15])
                 :
                 : "memory");
}

// thread t of the warp writes lane (base lane + t), columns [col, col+16)
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
                 "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
                 : "memory");
}

__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// D[tmem] (+)= A[tmem] * B[smem desc]^T, kind::f16, A resident in tensor
// memory (row m in lane m, two 16-bit K elements per 32-bit column)
__device__ __forceinline__ void mma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                           uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
                 : "memory");
}

// ---- descriptors ----------------------------------------------------------
// Shared-memory matrix descriptor of a K-major operand written by TMA with
// 128-byte swizzling: rows of 128 bytes, 8-row swizzle atoms 1024 bytes
// apart (SBO = 1024 B), LBO unused (1), descriptor version 1 (sm_100),
// layout type 2 (SWIZZLE_128B).  `addr` must lie in a 1024-byte aligned atom.
__device__ __forceinline__ uint64_t desc_kmajor_sw128(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;           // LBO (16 B, ignored for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32; // SBO
    d |= (uint64_t)1 << 46;           // version
    d |= (uint64_t)2 << 61;           // SWIZZLE_128B
    return d;
}

// Descriptor of an MN-major operand written by TMA with 128-byte swizzling
// in boxes of 64 MN-elements x 64 K-rows: each K-row is 128 bytes (64
// consecutive M or N elements), 8-row groups 1024 bytes apart (SBO), and the
// next 64-element MN chunk `lbo` bytes away (the next box).
__device__ __forceinline__ uint64_t desc_mnmajor_sw128(uint32_t addr, uint32_t lbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16; // LBO: next 64-element MN chunk
    d |= (uint64_t)(1024 >> 4) << 32;          // SBO: next group of 8 K rows
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Descriptors of 16 x 16 16-bit tiles stored with 32-byte swizzling (rows of
// 32 bytes, 8-row atoms of 256 bytes on 256-byte boundaries, the 16-byte
// chunk of rows 4-7 of each atom flipped): layout type 6 (SWIZZLE_32B),
// SBO = 256 bytes to the next 8 rows.  K-major: row = M (or N) index, K
// contiguous; MN-major: row = K index, 16 MN elements contiguous (LBO, the
// step to the next 16 MN elements, is unused for N = 16).
__device__ __forceinline__ uint64_t desc_kmajor_sw32(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;          // LBO (ignored for swizzled K-major)
    d |= (uint64_t)(256 >> 4) << 32; // SBO
    d |= (uint64_t)1 << 46;          // version
    d |= (uint64_t)6 << 61;          // SWIZZLE_32B
    return d;
}

__device__ __forceinline__ uint64_t desc_mnmajor_sw32(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(512 >> 4) << 16; // LBO: next 16 MN elements (unused at N = 16)
    d |= (uint64_t)(256 >> 4) << 32; // SBO: next 8 K rows
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)6 << 61;
    return d;
}

// D[tmem] += A * B^T (kind::f16, both operands in shared memory) with the
// lanes of D whose bit is set in `off` (bit l % 32 of off[l / 32]) left
// unchanged -- the accumulators of other tiles that share these columns.
__device__ __forceinline__ void mma_f16_ss_lanes(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                                 const uint32_t (&off)[4])
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, 1, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%4, %5, %6, %7}, p;\n\t}" ::"r"(d_tmem),
                 "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(off[0]), "r"(off[1]), "r"(off[2]), "r"(off[3])
                 : "memory");
}

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator, given
// M (64 or 128), N (multiple of 16, <= 256) and the operand majors
// (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_f16(bool bf16, int M, int N, int a_mn = 0, int b_mn = 0)
{
    return (1u << 4)                         // D format F32
           | ((bf16 ? 1u : 0u) << 7)         // A format
           | ((bf16 ? 1u : 0u) << 10)        // B format
           | ((uint32_t)(a_mn & 1) << 15)    // A major
           | ((uint32_t)(b_mn & 1) << 16)    // B major
           | ((uint32_t)(N >> 3) << 17)      // N / 8
           | ((uint32_t)(M >> 4) << 24);     // M / 16
}

// Instruction descriptor of tcgen05.mma kind::i8 with both operands signed
// 8-bit, K-major, and an INT32 accumulator (D format 2, A/B format 1 =
// signed), given M and N.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N)
{
    return (2u << 4)                         // D format S32
           | (1u << 7)                       // A signed 8-bit
           | (1u << 10)                      // B signed 8-bit
           | ((uint32_t)(N >> 3) << 17)      // N / 8
           | ((uint32_t)(M >> 4) << 24);     // M / 16
}

} // namespace tc
} // namespace kami
