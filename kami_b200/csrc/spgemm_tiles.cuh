// spgemm_tiles.cuh -- 16 x 16 BSR tile helpers shared by the block SpGEMM
// kernels: the swizzled shared-memory tile layout, its staging copy, the
// ldmatrix addressing of a staged tile, and the m16n8k16 MMA (FP32
// accumulation) that consumes its fragments.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kami_common.cuh"

namespace kami {
namespace sptile {

// Byte offset of row r, 16-byte chunk c of a 16 x 16 16-bit tile (32-byte
// rows): the chunk is flipped for rows 4-7 and 12-15 so that the eight rows
// of an ldmatrix phase fall in distinct banks.  (This is also the 32-byte
// swizzle of the tensor cores' shared-memory layouts when the tile sits on a
// 256-byte boundary.)
__device__ __forceinline__ int tile_swz(int r, int c) { return r * 32 + ((c ^ ((r >> 2) & 1)) << 4); }

// Copy one 512-byte tile (16 bytes per lane) into a swizzled shared tile.
__device__ __forceinline__ void stage_tile(uint8_t *dst, const uint16_t *src, int lane)
{
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(src) + lane);
    *reinterpret_cast<uint4 *>(dst + tile_swz(lane >> 1, lane & 1)) = v;
}

// ldmatrix address of `lane` for the x4 load of a swizzled tile: matrices
// (rows 0-7, chunk 0), (rows 8-15, chunk 0), (rows 0-7, chunk 1), (8-15, 1).
__device__ __forceinline__ uint32_t tile_ldsm_addr(uint32_t base, int lane)
{
    const int m = lane >> 3, i = lane & 7;
    return base + tile_swz((m & 1) * 8 + i, m >> 1);
}

__device__ __forceinline__ void ldsm4(uint32_t a, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

__device__ __forceinline__ void ldsm4_t(uint32_t a, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// d (16 x 8, FP32) += A (16 x 16) * B (16 x 8), FP16 or BF16 operands.
template <bool BF16>
__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    if constexpr (BF16)
        asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    else
        asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}


// Store one C tile held as m16n8k16 accumulators with alpha / beta into
// tile `c` of vc (FP32, FP16 or BF16 tiles, row-major 16 x 16): lane (gq,
// tq) holds rows gq, gq + 8 and columns 2tq, 2tq + 1 (acc0) and 2tq + 8,
// 2tq + 9 (acc1).  beta == 0 never reads C.  FP32 tiles at a 16-byte
// aligned base are written as float4: lane pairs (tq, tq ^ 1) swap one
// column pair, so each lane holds four consecutive columns and every store
// instruction covers eight whole 64-byte rows (512 contiguous bytes) instead
// of eight 32-byte halves of them (n = 16384, 1 % numeric pass: best of 25
// 36.8 against 37.7 us, medians equal).  Every caller runs this with the
// whole warp.
__device__ __forceinline__ void store_tile_frag(void *vc, int64_t c, int out_type, float alpha, float beta, int gq,
                                                int tq, const float (&acc0)[4], const float (&acc1)[4])
{
    const int r0 = gq, r1 = gq + 8, c0 = 2 * tq;
    if (out_type == KAMI_F32)
    {
        float *out = reinterpret_cast<float *>(vc) + c * 256;
        if ((reinterpret_cast<uintptr_t>(vc) & 15) == 0)
        {
            const bool odd = tq & 1;
            const int col = (tq & 1) * 8 + (tq >> 1) * 4;
            const float s0 = odd ? acc0[0] : acc1[0], s1 = odd ? acc0[1] : acc1[1];
            const float s2 = odd ? acc0[2] : acc1[2], s3 = odd ? acc0[3] : acc1[3];
            const float g0 = __shfl_xor_sync(0xffffffffu, s0, 1), g1 = __shfl_xor_sync(0xffffffffu, s1, 1);
            const float g2 = __shfl_xor_sync(0xffffffffu, s2, 1), g3 = __shfl_xor_sync(0xffffffffu, s3, 1);
            float4 w0 = odd ? make_float4(g0, g1, acc1[0], acc1[1]) : make_float4(acc0[0], acc0[1], g0, g1);
            float4 w1 = odd ? make_float4(g2, g3, acc1[2], acc1[3]) : make_float4(acc0[2], acc0[3], g2, g3);
            float4 *o0 = reinterpret_cast<float4 *>(out + r0 * 16 + col);
            float4 *o1 = reinterpret_cast<float4 *>(out + r1 * 16 + col);
            if (alpha != 1.f || beta != 0.f)
            {
                float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0;
                if (beta != 0.f)
                {
                    p0 = *o0;
                    p1 = *o1;
                }
                w0 = make_float4(alpha * w0.x + beta * p0.x, alpha * w0.y + beta * p0.y, alpha * w0.z + beta * p0.z,
                                 alpha * w0.w + beta * p0.w);
                w1 = make_float4(alpha * w1.x + beta * p1.x, alpha * w1.y + beta * p1.y, alpha * w1.z + beta * p1.z,
                                 alpha * w1.w + beta * p1.w);
            }
            *o0 = w0;
            *o1 = w1;
            return;
        }
        float2 v00 = make_float2(acc0[0], acc0[1]), v01 = make_float2(acc1[0], acc1[1]);
        float2 v10 = make_float2(acc0[2], acc0[3]), v11 = make_float2(acc1[2], acc1[3]);
        if (alpha != 1.f || beta != 0.f)
        {
            const float a = alpha, b = beta;
            float2 o00 = make_float2(0.f, 0.f), o01 = o00, o10 = o00, o11 = o00;
            if (b != 0.f)
            {
                o00 = *reinterpret_cast<float2 *>(out + r0 * 16 + c0);
                o01 = *reinterpret_cast<float2 *>(out + r0 * 16 + c0 + 8);
                o10 = *reinterpret_cast<float2 *>(out + r1 * 16 + c0);
                o11 = *reinterpret_cast<float2 *>(out + r1 * 16 + c0 + 8);
            }
            v00 = make_float2(a * v00.x + b * o00.x, a * v00.y + b * o00.y);
            v01 = make_float2(a * v01.x + b * o01.x, a * v01.y + b * o01.y);
            v10 = make_float2(a * v10.x + b * o10.x, a * v10.y + b * o10.y);
            v11 = make_float2(a * v11.x + b * o11.x, a * v11.y + b * o11.y);
        }
        *reinterpret_cast<float2 *>(out + r0 * 16 + c0) = v00;
        *reinterpret_cast<float2 *>(out + r0 * 16 + c0 + 8) = v01;
        *reinterpret_cast<float2 *>(out + r1 * 16 + c0) = v10;
        *reinterpret_cast<float2 *>(out + r1 * 16 + c0 + 8) = v11;
    }
    else
    {
        uint16_t *out = reinterpret_cast<uint16_t *>(vc) + c * 256;
        const bool bf = out_type == KAMI_BF16;
        auto cvt = [&](float x, uint16_t old) -> uint16_t {
            float y = alpha * x;
            if (beta != 0.f)
                y += beta * to_float(old, bf);
            return bf ? __bfloat16_as_ushort(__float2bfloat16_rn(y)) : __half_as_ushort(__float2half_rn(y));
        };
        const int offs[4] = {r0 * 16 + c0, r0 * 16 + c0 + 8, r1 * 16 + c0, r1 * 16 + c0 + 8};
        const float vals[4][2] = {{acc0[0], acc0[1]}, {acc1[0], acc1[1]}, {acc0[2], acc0[3]}, {acc1[2], acc1[3]}};
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            uint32_t *dst = reinterpret_cast<uint32_t *>(out + offs[q]);
            const uint32_t old = beta != 0.f ? *dst : 0u;
            const uint16_t lo16 = cvt(vals[q][0], (uint16_t)(old & 0xffff));
            const uint16_t hi16 = cvt(vals[q][1], (uint16_t)(old >> 16));
            *dst = (uint32_t)lo16 | ((uint32_t)hi16 << 16);
        }
    }
}

} // namespace sptile
} // namespace kami
