// kami_common.cuh -- shared definitions of the kami_b200 device code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "../../include/kami.h"

namespace kami {

// Everything a batched block-GEMM kernel needs, passed by value.
struct GemmArgs {
    int M, N, K;
    int64_t batch;
    const void *A;
    int64_t lda, sA;
    int a_layout;
    const void *B;
    int64_t ldb, sB;
    int b_layout;
    void *C;
    int64_t ldc, sC;
    int out_type;
    int c_vec;    // 1: pairs of C elements may be stored as one vector
    int c_vec4;   // 1: groups of 4 C elements (4-aligned columns) may be stored as one vector
    double alpha, beta;
    int num_iter;
    int problems_per_cta;
    unsigned long long *trace; // traced instances: per-warp {communication, computation} cycles of problem 0
    int one_per_sm;            // launch hint: at most one CTA of the repeated-products kernel per SM
};

// Host-side description of a resolved launch (kami_gemm_describe).
struct LaunchInfo {
    int variant, partition, P, threads, smem, problems_per_cta;
    int64_t grid;
};

// Named barrier over `nthreads` threads (a multiple of 32).  Warps that
// exited early are not counted, unlike __syncthreads().
__device__ __forceinline__ void named_barrier(int id, int nthreads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ float to_float(uint16_t bits, bool bf16)
{
    if (bf16)
        return __uint_as_float(((uint32_t)bits) << 16);
    return __half2float(__ushort_as_half(bits));
}

// Store one accumulator pair (row r, columns c, c+1) with alpha/beta.
template <typename Acc>
__device__ __forceinline__ void store_pair(const GemmArgs &g, void *Cb, int r, int c, Acc v0, Acc v1)
{
    if (r >= g.M || c >= g.N)
        return;
    const bool two = c + 1 < g.N;
    const int64_t off = (int64_t)r * g.ldc + c;
    if (g.out_type == KAMI_F64)
    {
        double *p = reinterpret_cast<double *>(Cb) + off;
        double x0 = g.alpha * (double)v0, x1 = g.alpha * (double)v1;
        if (g.beta != 0.0)
        {
            x0 += g.beta * p[0];
            if (two)
                x1 += g.beta * p[1];
        }
        if (two && g.c_vec)
            *reinterpret_cast<double2 *>(p) = make_double2(x0, x1);
        else
        {
            p[0] = x0;
            if (two)
                p[1] = x1;
        }
    }
    else if (g.out_type == KAMI_F32)
    {
        float *p = reinterpret_cast<float *>(Cb) + off;
        float x0 = (float)(g.alpha * (double)v0), x1 = (float)(g.alpha * (double)v1);
        if (g.alpha == 1.0)
        {
            x0 = (float)v0;
            x1 = (float)v1;
        }
        if (g.beta != 0.0)
        {
            x0 += (float)g.beta * p[0];
            if (two)
                x1 += (float)g.beta * p[1];
        }
        if (two && g.c_vec)
            *reinterpret_cast<float2 *>(p) = make_float2(x0, x1);
        else
        {
            p[0] = x0;
            if (two)
                p[1] = x1;
        }
    }
    else
    {
        const bool bf = g.out_type == KAMI_BF16;
        uint16_t *p = reinterpret_cast<uint16_t *>(Cb) + off;
        float x0 = (float)v0, x1 = (float)v1;
        if (g.alpha != 1.0)
        {
            x0 = (float)(g.alpha * (double)v0);
            x1 = (float)(g.alpha * (double)v1);
        }
        if (g.beta != 0.0)
        {
            x0 += (float)g.beta * to_float(p[0], bf);
            if (two)
                x1 += (float)g.beta * to_float(p[1], bf);
        }
        uint16_t h0, h1;
        if (bf)
        {
            h0 = __bfloat16_as_ushort(__float2bfloat16_rn(x0));
            h1 = __bfloat16_as_ushort(__float2bfloat16_rn(x1));
        }
        else
        {
            h0 = __half_as_ushort(__float2half_rn(x0));
            h1 = __half_as_ushort(__float2half_rn(x1));
        }
        if (two && g.c_vec)
            *reinterpret_cast<uint32_t *>(p) = (uint32_t)h0 | ((uint32_t)h1 << 16);
        else
        {
            p[0] = h0;
            if (two)
                p[1] = h1;
        }
    }
}

} // namespace kami
