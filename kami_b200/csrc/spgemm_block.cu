// spgemm_block.cu -- the reference's block SpGEMM method: one CTA computes
// C = A * B for one small BSR matrix (at most 16 x 16 blocks of 16 x 16
// tiles per side), its warps owning the C tiles by the 1D / 2D / 3D
// partitions of KAMI.
//
// Reference: src/sparse/spgemm/{1d,2d,3d}/block_spgemm_{1d,2d,3d}_half_mma.cu
// (1d:107, 2d:171, 3d:175).  There every CTA of a 16384-CTA grid multiplies
// the same 128 x 128 BSR pair NUM_ITER times; warp w (1D), (r, c) (2D) or
// (r, c, d) (3D) keeps its slice of A and B in registers as mma fragments,
// publishes its B (and for 2D / 3D A) panel through shared memory stage by
// stage, searches the C column of each product linearly, and accumulates in
// FP16; the 3D form leaves P partial C slices for the host.
//
// Here the ownership maps are the same -- which warp accumulates which C
// tiles, over which k range -- but the operands are laid out for B200: the
// whole problem is small (<= 512 tiles), so every A and B tile is staged once
// into 227 KB of shared memory (swizzled for conflict-free ldmatrix) and the
// stage exchange disappears; a warp gathers the fragments of each C tile's
// products (A(i, k) and B(k, j), found by a search in the staged sorted
// column lists) into registers and repeats the m16n8k16 MMAs num_iter times
// on them (FP32 accumulation), so the repeats run on register-resident
// operands as in the reference.  The 3D form splits each C tile's products
// by k into P depth ranks and reduces their partial accumulators on the
// device through shared memory (named barrier per (r, c) group).
//
// The batch: `batch` problems share one sparsity structure (RowPtr / ColIdx
// of A, B and C) and take their tile values at per-problem strides (0 =
// shared, as the reference's 16384 CTAs share one matrix).
#include <cstdint>

#include "kami_common.cuh"
#include "spgemm_tiles.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

namespace {

using namespace sptile;

constexpr int kBlkMaxDim = 16;     // blocks per side (256 rows / columns)
constexpr int kBlkMaxTiles = 384;  // A and B tiles staged together (192 KB)
constexpr int kBlkChunk = 8;       // products whose fragments stay in registers over the repeats

struct SpBlockArgs
{
    int mb, kb, nb;
    int nnza, nnzb, nnzc;
    const int *rpa, *cia, *rpb, *cib, *rpc, *cic;
    const uint16_t *va, *vb;
    int64_t sva, svb; // per-problem value strides (elements; 0 = shared)
    void *vc;
    int64_t svc;
    int64_t batch;
    int out_type;
    float alpha, beta;
    int num_iter;
};

template <int PART, int P>
struct BlkShape
{
    static constexpr int warps = PART == 1 ? P : PART == 2 ? P * P : P * P * P;
};

__host__ __device__ constexpr int split_lo(int n, int parts, int i) { return (n * i) / parts; }

// shared memory: [A tiles][B tiles][rpa][cia][rpb][cib][rpc][cic][3D partials]
struct BlkSmem
{
    int off_b, off_rpa, off_cia, off_rpb, off_cib, off_rpc, off_cic, off_red, bytes;
};

__host__ __device__ inline BlkSmem blk_smem(int mb, int kb, int nnza, int nnzb, int nnzc, int groups, int depth)
{
    BlkSmem s{};
    s.off_b = nnza * 512;
    int o = (nnza + nnzb) * 512;
    s.off_rpa = o;
    o += (mb + 1) * 4;
    s.off_cia = o;
    o += nnza * 4;
    s.off_rpb = o;
    o += (kb + 1) * 4;
    s.off_cib = o;
    o += nnzb * 4;
    s.off_rpc = o;
    o += (mb + 1) * 4;
    s.off_cic = o;
    o += nnzc * 4;
    o = (o + 15) & ~15;
    s.off_red = o;
    o += depth > 1 ? groups * (depth - 1) * 32 * 8 * 4 : 0;
    s.bytes = o;
    return s;
}

template <int PART, int P, bool BF16>
__global__ void __launch_bounds__(BlkShape<PART, P>::warps * 32) spgemm_block_kernel(const SpBlockArgs p)
{
    constexpr int W = BlkShape<PART, P>::warps;
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gq = lane >> 2, tq = lane & 3;
    const int groups = PART == 3 ? P * P : 1;
    const BlkSmem L = blk_smem(p.mb, p.kb, p.nnza, p.nnzb, p.nnzc, groups, PART == 3 ? P : 1);
    int *s_rpa = reinterpret_cast<int *>(smem + L.off_rpa);
    int *s_cia = reinterpret_cast<int *>(smem + L.off_cia);
    int *s_rpb = reinterpret_cast<int *>(smem + L.off_rpb);
    int *s_cib = reinterpret_cast<int *>(smem + L.off_cib);
    int *s_rpc = reinterpret_cast<int *>(smem + L.off_rpc);
    int *s_cic = reinterpret_cast<int *>(smem + L.off_cic);
    const uint32_t sA = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t sB = sA + (uint32_t)L.off_b;

    // the structure is shared by every problem: stage it once
    for (int t = threadIdx.x; t <= p.mb; t += blockDim.x)
    {
        s_rpa[t] = p.rpa[t];
        s_rpc[t] = p.rpc[t];
    }
    for (int t = threadIdx.x; t <= p.kb; t += blockDim.x)
        s_rpb[t] = p.rpb[t];
    for (int t = threadIdx.x; t < p.nnza; t += blockDim.x)
        s_cia[t] = p.cia[t];
    for (int t = threadIdx.x; t < p.nnzb; t += blockDim.x)
        s_cib[t] = p.cib[t];
    for (int t = threadIdx.x; t < p.nnzc; t += blockDim.x)
        s_cic[t] = p.cic[t];

    // this warp's C tiles: rows [r0, r1), columns [c0, c1), products with k in [k0, k1)
    int r0 = 0, r1 = p.mb, c0 = 0, c1 = p.nb, k0 = 0, k1 = p.kb, depth = 0, group = 0;
    if constexpr (PART == 1)
    {
        r0 = split_lo(p.mb, P, warp);
        r1 = split_lo(p.mb, P, warp + 1);
    }
    else if constexpr (PART == 2)
    {
        const int wr = warp / P, wc = warp % P;
        r0 = split_lo(p.mb, P, wr);
        r1 = split_lo(p.mb, P, wr + 1);
        c0 = split_lo(p.nb, P, wc);
        c1 = split_lo(p.nb, P, wc + 1);
    }
    else
    {
        const int wr = warp / (P * P), wc = (warp / P) % P;
        depth = warp % P;
        group = wr * P + wc;
        r0 = split_lo(p.mb, P, wr);
        r1 = split_lo(p.mb, P, wr + 1);
        c0 = split_lo(p.nb, P, wc);
        c1 = split_lo(p.nb, P, wc + 1);
        k0 = split_lo(p.kb, P, depth);
        k1 = split_lo(p.kb, P, depth + 1);
    }
    float *red = reinterpret_cast<float *>(smem + L.off_red);

    for (int64_t b = blockIdx.x; b < p.batch; b += gridDim.x)
    {
        // stage this problem's A and B tiles (skipped after the first problem
        // when the values are shared)
        if (b == blockIdx.x || p.sva != 0 || p.svb != 0)
        {
            __syncthreads(); // the previous problem's fragments have been read
            const uint16_t *va = p.va + b * p.sva;
            const uint16_t *vb = p.vb + b * p.svb;
            for (int t = warp; t < p.nnza; t += W)
                stage_tile(smem + t * 512, va + (int64_t)t * 256, lane);
            for (int t = warp; t < p.nnzb; t += W)
                stage_tile(smem + L.off_b + t * 512, vb + (int64_t)t * 256, lane);
            __syncthreads();
        }
        void *vc = reinterpret_cast<uint8_t *>(p.vc) + b * p.svc * (p.out_type == KAMI_F32 ? 4 : 2);

        for (int i = r0; i < r1; ++i)
        {
            const int ca = s_rpc[i], cz = s_rpc[i + 1];
            const int ea = s_rpa[i], ez = s_rpa[i + 1];
            for (int c = ca; c < cz; ++c)
            {
                const int j = s_cic[c];
                if (j < c0 || j >= c1)
                    continue;
                float acc0[4] = {0.f, 0.f, 0.f, 0.f}, acc1[4] = {0.f, 0.f, 0.f, 0.f};
                int e = ea;
                while (true)
                {
                    // gather up to kBlkChunk products A(i, k) B(k, j), k ascending
                    int pa[kBlkChunk], pb[kBlkChunk], n = 0;
                    for (; e < ez && n < kBlkChunk; ++e)
                    {
                        const int k = s_cia[e];
                        if (k < k0 || k >= k1)
                            continue;
                        for (int q = s_rpb[k], qz = s_rpb[k + 1]; q < qz; ++q)
                        {
                            const int cb = s_cib[q];
                            if (cb == j)
                            {
                                pa[n] = e;
                                pb[n] = q;
                                ++n;
                                break;
                            }
                            if (cb > j)
                                break;
                        }
                    }
                    if (n == 0)
                        break;
                    uint32_t fa[kBlkChunk][4], fb[kBlkChunk][4];
#pragma unroll
                    for (int q = 0; q < kBlkChunk; ++q)
                        if (q < n)
                        {
                            ldsm4(tile_ldsm_addr(sA + pa[q] * 512, lane), fa[q]);
                            ldsm4_t(tile_ldsm_addr(sB + pb[q] * 512, lane), fb[q]);
                        }
                    for (int it = 0; it < p.num_iter; ++it)
                    {
#pragma unroll
                        for (int q = 0; q < kBlkChunk; ++q)
                            if (q < n)
                            {
                                mma16816<BF16>(acc0, fa[q][0], fa[q][1], fa[q][2], fa[q][3], fb[q][0], fb[q][1]);
                                mma16816<BF16>(acc1, fa[q][0], fa[q][1], fa[q][2], fa[q][3], fb[q][2], fb[q][3]);
                            }
                    }
                    if (e >= ez)
                        break;
                }
                if constexpr (PART == 3)
                {
                    // depth ranks 1..P-1 hand their partials to rank 0 of the (r, c) group
                    float *slot = red + ((group * (P - 1)) * 32 + lane) * 8;
                    if (depth > 0)
                    {
                        float *d = slot + (depth - 1) * 32 * 8;
#pragma unroll
                        for (int t = 0; t < 4; ++t)
                        {
                            d[t] = acc0[t];
                            d[4 + t] = acc1[t];
                        }
                    }
                    named_barrier(1 + group, P * 32);
                    if (depth == 0)
                    {
                        for (int d = 1; d < P; ++d)
                        {
                            const float *s = slot + (d - 1) * 32 * 8;
#pragma unroll
                            for (int t = 0; t < 4; ++t)
                            {
                                acc0[t] += s[t];
                                acc1[t] += s[4 + t];
                            }
                        }
                        store_tile_frag(vc, c, p.out_type, p.alpha, p.beta, gq, tq, acc0, acc1);
                    }
                    named_barrier(1 + group, P * 32);
                }
                else
                    store_tile_frag(vc, c, p.out_type, p.alpha, p.beta, gq, tq, acc0, acc1);
            }
        }
    }
}

template <int PART, int P>
const void *blk_fn(bool bf16)
{
    return bf16 ? (const void *)spgemm_block_kernel<PART, P, true> : (const void *)spgemm_block_kernel<PART, P, false>;
}

// compiled instances: 1D P = 1, 2, 4, 8; 2D P = 2, 4; 3D P = 2
const void *blk_select(int part, int P, bool bf16)
{
    if (part == KAMI_PARTITION_1D)
        switch (P)
        {
        case 1: return blk_fn<1, 1>(bf16);
        case 2: return blk_fn<1, 2>(bf16);
        case 4: return blk_fn<1, 4>(bf16);
        case 8: return blk_fn<1, 8>(bf16);
        }
    if (part == KAMI_PARTITION_2D)
        switch (P)
        {
        case 2: return blk_fn<2, 2>(bf16);
        case 4: return blk_fn<2, 4>(bf16);
        }
    if (part == KAMI_PARTITION_3D && P == 2)
        return blk_fn<3, 2>(bf16);
    return nullptr;
}

} // namespace
} // namespace kami

using namespace kami;

extern "C" int kami_spgemm_bsr_block(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition, int P,
                                     int bsr, int mb, int kb, int nb, int64_t batch, const int *row_ptr_a,
                                     const int *col_idx_a, const void *val_a, int64_t stride_val_a, int nnz_a,
                                     const int *row_ptr_b, const int *col_idx_b, const void *val_b,
                                     int64_t stride_val_b, int nnz_b, const int *row_ptr_c, const int *col_idx_c,
                                     void *val_c, int64_t stride_val_c, int nnz_c, double alpha, double beta,
                                     int num_iter, void *stream)
{
    if (bsr != 16)
        return fail(KAMI_ERR_UNSUPPORTED, "block spgemm: only 16 x 16 BSR tiles are supported (got %d)", bsr);
    if (in_type != KAMI_F16 && in_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "block spgemm: FP16/BF16 tiles only");
    if (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "block spgemm: FP32/FP16/BF16 output only");
    if (mb < 1 || kb < 1 || nb < 1 || batch < 0 || num_iter < 1 || nnz_a < 0 || nnz_b < 0 || nnz_c < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "block spgemm: bad dimensions, batch, counts or num_iter");
    if (mb > kBlkMaxDim || kb > kBlkMaxDim || nb > kBlkMaxDim)
        return fail(KAMI_ERR_UNSUPPORTED,
                    "block spgemm: %d x %d x %d blocks exceed one CTA's block (at most %d per side); use "
                    "kami_spgemm_bsr_numeric",
                    mb, kb, nb, kBlkMaxDim);
    if (nnz_a > mb * kb || nnz_b > kb * nb || nnz_c > mb * nb)
        return fail(KAMI_ERR_INVALID_VALUE, "block spgemm: more entries than block positions");
    if (nnz_a + nnz_b > kBlkMaxTiles)
        return fail(KAMI_ERR_UNSUPPORTED, "block spgemm: %d A + B tiles exceed the %d staged in shared memory",
                    nnz_a + nnz_b, kBlkMaxTiles);
    if (stride_val_a < 0 || stride_val_b < 0 || stride_val_c < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "block spgemm: negative stride");
    if (batch == 0 || nnz_c == 0)
        return KAMI_OK;
    if (!row_ptr_a || !row_ptr_b || !row_ptr_c || !col_idx_c || !val_c || (nnz_a && (!col_idx_a || !val_a)) ||
        (nnz_b && (!col_idx_b || !val_b)))
        return fail(KAMI_ERR_INVALID_VALUE, "block spgemm: null pointer");
    if ((reinterpret_cast<uintptr_t>(val_a) & 15) || (reinterpret_cast<uintptr_t>(val_b) & 15) ||
        (reinterpret_cast<uintptr_t>(val_c) & 7) || (stride_val_a & 7) || (stride_val_b & 7) || (stride_val_c & 3))
        return fail(KAMI_ERR_MISALIGNED, "block spgemm: tile arrays must be 16-byte aligned (C 8-byte), strides "
                                         "whole 16-byte steps");
    if (partition == KAMI_PARTITION_AUTO)
    {
        partition = KAMI_PARTITION_1D;
        if (P == 0)
            P = 4;
    }
    if (P == 0)
        P = partition == KAMI_PARTITION_1D ? 4 : 2;
    const void *fn = blk_select(partition, P, in_type == KAMI_BF16);
    if (!fn)
        return fail(KAMI_ERR_UNSUPPORTED,
                    "block spgemm: no instance for partition %d with P = %d (1D: 1, 2, 4, 8; 2D: 2, 4; 3D: 2)",
                    (int)partition, P);
    const int warps = partition == KAMI_PARTITION_1D ? P : partition == KAMI_PARTITION_2D ? P * P : P * P * P;
    const BlkSmem L = blk_smem(mb, kb, nnz_a, nnz_b, nnz_c, partition == KAMI_PARTITION_3D ? P * P : 1,
                               partition == KAMI_PARTITION_3D ? P : 1);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, L.bytes)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(spgemm_block_kernel)");
    SpBlockArgs p{};
    p.mb = mb;
    p.kb = kb;
    p.nb = nb;
    p.nnza = nnz_a;
    p.nnzb = nnz_b;
    p.nnzc = nnz_c;
    p.rpa = row_ptr_a;
    p.cia = col_idx_a;
    p.rpb = row_ptr_b;
    p.cib = col_idx_b;
    p.rpc = row_ptr_c;
    p.cic = col_idx_c;
    p.va = reinterpret_cast<const uint16_t *>(val_a);
    p.vb = reinterpret_cast<const uint16_t *>(val_b);
    p.sva = stride_val_a;
    p.svb = stride_val_b;
    p.vc = val_c;
    p.svc = stride_val_c;
    p.batch = batch;
    p.out_type = out_type;
    p.alpha = (float)alpha;
    p.beta = (float)beta;
    p.num_iter = num_iter;
    const unsigned grid = (unsigned)(batch < 0x7fffffff ? batch : 0x7fffffff);
    void *args[] = {&p};
    if ((e = cudaLaunchKernel(fn, dim3(grid), dim3(warps * 32), args, (size_t)L.bytes,
                              reinterpret_cast<cudaStream_t>(stream))) != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(spgemm_block_kernel)");
    return KAMI_OK;
}
