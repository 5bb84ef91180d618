// tc05_epi.cuh -- epilogue of the tcgen05 kernels: accumulator rows read
// from tensor memory, transposed through a small shared tile per warp, and
// written to C with alpha / beta and the output type applied.
#pragma once
#include "kami_common.cuh"

namespace kami {

// ---------------------------------------------------------------------------
// Coalesced epilogue.  tcgen05.ld leaves each thread 16 consecutive columns of
// its own row; stored directly that is 32 rows touched per instruction with
// half-used sectors.  Each warp transposes through a 32 x 20-float shared
// tile so that every store instruction writes 8 rows x 64 contiguous bytes.
// ---------------------------------------------------------------------------
constexpr int kEpiStride = 20;                       // floats per staged row (16 + pad)
constexpr int kEpiTileBytes = 32 * kEpiStride * 4;   // per warp

__device__ __forceinline__ void store4(const GemmArgs &g, void *Cb, int r, int c, float4 x)
{
    if (g.c_vec4 && c + 3 < g.N)
    {
        const int64_t off = (int64_t)r * g.ldc + c;
        const float a = (float)g.alpha, b = (float)g.beta;
        if (g.out_type == KAMI_F32)
        {
            float4 *dst = reinterpret_cast<float4 *>(reinterpret_cast<float *>(Cb) + off);
            if (g.alpha != 1.0 || g.beta != 0.0)
            {
                const float4 o = g.beta != 0.0 ? *dst : make_float4(0.f, 0.f, 0.f, 0.f);
                x = make_float4(a * x.x + b * o.x, a * x.y + b * o.y, a * x.z + b * o.z, a * x.w + b * o.w);
            }
            *dst = x;
        }
        else
        {
            const bool bf = g.out_type == KAMI_BF16;
            uint2 *dst = reinterpret_cast<uint2 *>(reinterpret_cast<uint16_t *>(Cb) + off);
            float y[4] = {x.x, x.y, x.z, x.w};
            if (g.alpha != 1.0 || g.beta != 0.0)
            {
                const uint2 o = g.beta != 0.0 ? *dst : make_uint2(0u, 0u);
                const uint16_t ob[4] = {(uint16_t)(o.x & 0xffff), (uint16_t)(o.x >> 16), (uint16_t)(o.y & 0xffff),
                                        (uint16_t)(o.y >> 16)};
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    y[e] = a * y[e] + (g.beta != 0.0 ? b * to_float(ob[e], bf) : 0.f);
            }
            uint32_t h[4];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                h[e] = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(y[e])) : __half_as_ushort(__float2half_rn(y[e]));
            *dst = make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
        }
        return;
    }
    store_pair<float>(g, Cb, r, c, x.x, x.y);
    store_pair<float>(g, Cb, r, c + 2, x.z, x.w);
}

// two values rounded to the 16-bit output type, packed low column first
__device__ __forceinline__ uint32_t pack2(float x, float y, bool bf)
{
    const uint32_t lo = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(x)) : __half_as_ushort(__float2half_rn(x));
    const uint32_t hi = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(y)) : __half_as_ushort(__float2half_rn(y));
    return lo | (hi << 16);
}

// f: the calling thread's 16 values of row (row_base + lane), columns
// c0..c0+15; nrows: rows this warp holds (32, or 16 for M = 64 MMAs).  Rows
// past g.M are skipped, and with kRowsBelowZero rows below 0 too (a band that
// starts before the problem: several problems in one accumulator).
template <bool kRowsBelowZero = false>
__device__ __forceinline__ void store_chunk(const GemmArgs &g, void *Cb, const float (&f)[16], int row_base,
                                            int nrows, int c0, float *T)
{
    const int lane = threadIdx.x & 31;
    float4 *t4 = reinterpret_cast<float4 *>(T + lane * kEpiStride);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        t4[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
    __syncwarp();
    const int rr = lane >> 2, cq = (lane & 3) * 4;
    // plain stores (alpha 1, beta 0, 4-element vectors allowed): the value goes
    // out as one 16-byte (FP32) or 8-byte (16-bit) store with no per-element
    // scaling or type dispatch
    const bool plain = g.c_vec4 && g.alpha == 1.0 && g.beta == 0.0;
    const int ot = g.out_type;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int lr = 8 * i + rr;
        if (lr < nrows)
        {
            const int r = row_base + lr;
            const int c = c0 + cq;
            const float4 x = *reinterpret_cast<const float4 *>(T + lr * kEpiStride + cq);
            if (kRowsBelowZero && r < 0)
                continue;
            if (plain && r < g.M && c + 3 < g.N)
            {
                const int64_t off = (int64_t)r * g.ldc + c;
                if (ot == KAMI_F32)
                    *reinterpret_cast<float4 *>(reinterpret_cast<float *>(Cb) + off) = x;
                else
                {
                    const bool bf = ot == KAMI_BF16;
                    *reinterpret_cast<uint2 *>(reinterpret_cast<uint16_t *>(Cb) + off) =
                        make_uint2(pack2(x.x, x.y, bf), pack2(x.z, x.w, bf));
                }
            }
            else if (r < g.M && c < g.N)
                store4(g, Cb, r, c, x);
        }
    }
    __syncwarp();
}

} // namespace kami
