// spmm.cu -- block SpMM C = A * op(B): A sparse in BSR form (16 x 16 tiles,
// or the reference's tiled-BSR form), B and C dense.
//
// Reference path (src/sparse/spmm/{1d,2d,3d}/block_spmm_*_half_mma.cu):
// one CTA computes one M_BLOCK x N_BLOCK block C = A * B^T with A an
// M_BLOCK x K_BLOCK BSR block (BSR_M = BSR_K = 16), B dense N x K row-major
// ("Bref", 1d/...:121-127 reads B[n * K_BLOCK + k]) and C row-major; FP16
// tiles, FP16 accumulation, NUM_ITER in-register repeats.  The 1D kernel
// (1d/...:78-195) reads BSR directly; the 2D and 3D kernels (2d/...:72-253,
// 3d/...:73-239) read a tiled-BSR re-grouping built on the host by
// bsr2tilebsr (2d/...:264-293): per row tile of NUMS_ROW block-rows and
// column tile of NUMS_COL block-columns, the row pointers of the tile's
// block-rows and the column indices relative to the tile.
//
// This implementation takes either form through one description: block-row
// r of A is the union over column tiles s of the entries
//   [rowptr[q], rowptr[q + 1]),  q = (r / R) * R * T + s * R + r % R,
// with block column colidx[e] + s * Cw (R = tile rows, T = column tiles,
// Cw = tile columns); plain BSR is R = 1, T = 1.  Values are tiles in entry
// order (vals[e * 256 + row * 16 + col], 1d/...:95-115).
//
// Kernel (mma.sync m16n8k16, FP32 accumulation): a CTA of 4 warps owns 4
// block-rows x 64 columns of one problem; each warp one block-row.  When
// the whole K extent fits (K <= 256) the CTA first stages its 64-column
// panel of B in shared memory (rows padded to 16-byte multiples + 16 bytes,
// so ldmatrix reads are conflict-free) and every nonzero tile costs one
// 4 x 32-bit A fragment load plus four ldmatrix.x4 (non-transposed for the
// N x K layout, transposed for K x N) per eight MMAs.  Larger K streams the
// B fragments from global memory (L2-resident for the sizes of interest).
// num_iter repeats the products over the resident operands (the reference's
// NUM_ITER methodology).  A block column outside [0, kb) is skipped, so a
// malformed index array cannot make the kernel read outside B.
#include <cstdint>

#include "kami_common.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
int spmm_tc05_launch(bool bf16, int out_type, int mb, int kb, int N, const int *rowptr, const int *colidx,
                     const void *vals, const void *B, int64_t ldb, bool b_nk, void *C, int64_t ldc, double alpha,
                     double beta, int num_iter, cudaStream_t s);

namespace {

constexpr int kWarps = 4;       // block-rows per CTA
constexpr int kCols = 64;       // output columns per CTA (8 n8 tiles)
constexpr int kPanelMaxK = 256; // K extent staged in shared memory

struct SpmmParams
{
    int mb, kb, N;
    int64_t batch;
    const int *rowptr;
    const int *colidx;
    int64_t s_rowptr, s_colidx;
    const uint16_t *vals;
    int64_t s_vals; // elements
    const uint16_t *B;
    int64_t ldb, sB;
    int refnk; // 1: B is N x K row-major (the reference layout); 0: K x N
    void *C;
    int64_t ldc, sC;
    int out_type;
    int bf16;
    double alpha, beta;
    int num_iter;
    int tile_rows, ntiles, tile_cols;
    int c_vec;
    int b_vec; // 1: B rows are 16-byte aligned (vector staging)
};

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1, bool bf)
{
    if (bf)
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    else
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4])
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

// A fragment of tile e: rows g, g+8 and columns 2c, 2c+1, 2c+8, 2c+9 of the
// row-major 16 x 16 tile (g = lane / 4, c = lane % 4).
__device__ __forceinline__ void load_a(const uint16_t *tile, int lane, uint32_t (&a)[4])
{
    const int g = lane >> 2, c = (lane & 3) * 2;
    const uint32_t *t = reinterpret_cast<const uint32_t *>(tile);
    a[0] = __ldg(t + (g * 16 + c) / 2);
    a[1] = __ldg(t + ((g + 8) * 16 + c) / 2);
    a[2] = __ldg(t + (g * 16 + c + 8) / 2);
    a[3] = __ldg(t + ((g + 8) * 16 + c + 8) / 2);
}

__device__ __forceinline__ uint32_t pack_h2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

// B fragments of n8 tile (n0 + 8 t) and k block kk, straight from global
// memory (K beyond the panel): b0 = (k = 16 kk + 2c + {0,1}, n = n0 + 8t + g),
// b1 = the same with k + 8; zero for n >= N.
__device__ __forceinline__ void load_b_global(const SpmmParams &p, const uint16_t *B, int n, int k, uint32_t &b0,
                                              uint32_t &b1)
{
    if (n >= p.N)
    {
        b0 = b1 = 0u;
        return;
    }
    if (p.refnk)
    {
        const uint16_t *q = B + (int64_t)n * p.ldb + k;
        if (p.b_vec)
        {
            b0 = __ldg(reinterpret_cast<const uint32_t *>(q));
            b1 = __ldg(reinterpret_cast<const uint32_t *>(q + 8));
        }
        else
        {
            b0 = pack_h2(__ldg(q), __ldg(q + 1));
            b1 = pack_h2(__ldg(q + 8), __ldg(q + 9));
        }
    }
    else
    {
        const uint16_t *q = B + (int64_t)k * p.ldb + n;
        b0 = pack_h2(__ldg(q), __ldg(q + p.ldb));
        b1 = pack_h2(__ldg(q + 8 * p.ldb), __ldg(q + 9 * p.ldb));
    }
}

__device__ __forceinline__ void store_c(const SpmmParams &p, void *Cb, int r, int c, float v0, float v1)
{
    GemmArgs g{};
    g.M = p.mb * 16;
    g.N = p.N;
    g.ldc = p.ldc;
    g.out_type = p.out_type;
    g.c_vec = p.c_vec;
    g.alpha = p.alpha;
    g.beta = p.beta;
    store_pair<float>(g, Cb, r, c, v0, v1);
}

template <bool PANEL>
__global__ void __launch_bounds__(kWarps * 32) spmm_kernel(const SpmmParams p)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int K = p.kb * 16;
    const int n0 = blockIdx.y * kCols;
    // panel row stride in bytes: N x K layout -> rows n of K halves; K x N
    // layout -> rows k of kCols halves; both padded by 16 bytes
    const int pstride = p.refnk ? K * 2 + 16 : kCols * 2 + 16;
    const uint32_t panel = (uint32_t)__cvta_generic_to_shared(smem);

    for (int64_t prob = blockIdx.z; prob < p.batch; prob += gridDim.z)
    {
        const uint16_t *B = p.B + prob * p.sB;
        if (PANEL)
        {
            // stage B[n0 .. n0+63][0 .. K) (or B[0 .. K)[n0 .. n0+63]), zero past N
            __syncthreads(); // the previous problem's readers are done
            const int rows = p.refnk ? kCols : K, rowlen = p.refnk ? K : kCols; // halves
            const int chunks = rowlen / 8;                                       // 16-byte chunks per row
            for (int idx = threadIdx.x; idx < rows * chunks; idx += blockDim.x)
            {
                const int rr = idx / chunks, ch = idx % chunks;
                uint4 v = make_uint4(0, 0, 0, 0);
                const int nrow = p.refnk ? n0 + rr : 0;
                if (p.refnk ? nrow < p.N : true)
                {
                    const uint16_t *src = p.refnk ? B + (int64_t)nrow * p.ldb + ch * 8
                                                  : B + (int64_t)rr * p.ldb + n0 + ch * 8;
                    const int valid = p.refnk ? 8 : min(8, p.N - (n0 + ch * 8));
                    if (p.b_vec && valid == 8)
                        v = __ldg(reinterpret_cast<const uint4 *>(src));
                    else
                    {
                        uint16_t h[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            h[q] = q < valid ? __ldg(src + q) : (uint16_t)0;
                        v = make_uint4(pack_h2(h[0], h[1]), pack_h2(h[2], h[3]), pack_h2(h[4], h[5]),
                                       pack_h2(h[6], h[7]));
                    }
                }
                *reinterpret_cast<uint4 *>(smem + rr * pstride + ch * 16) = v;
            }
            __syncthreads();
        }

        const int r = blockIdx.x * kWarps + warp; // block-row of this warp
        if (r >= p.mb)
            continue;
        const int *rowptr = p.rowptr + prob * p.s_rowptr;
        const int *colidx = p.colidx + prob * p.s_colidx;
        const uint16_t *vals = p.vals + prob * p.s_vals;
        const int ntile8 = min(8, (p.N - n0 + 7) / 8);

        float acc[8][4];
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[t][q] = 0.f;

        const int rt = r / p.tile_rows, ri = r % p.tile_rows;
        const int m = lane >> 3, i8 = lane & 7;
        // eight MMAs of one nonzero tile: B fragments from the staged panel
        auto panel_products = [&](const uint32_t (&a)[4], int kk) {
#pragma unroll
            for (int t = 0; t < 8; t += 2)
            {
                if (t >= ntile8)
                    break;
                uint32_t b[4];
                if (p.refnk)
                {
                    // matrices: (tile t, k lo), (t, k hi), (t+1, lo), (t+1, hi)
                    const int nrow = (t + (m >> 1)) * 8 + i8;
                    const int kcol = kk * 16 + (m & 1) * 8;
                    ldsm_x4(panel + nrow * pstride + kcol * 2, b);
                }
                else
                {
                    const int krow = kk * 16 + (m & 1) * 8 + i8;
                    const int ncol = (t + (m >> 1)) * 8;
                    ldsm_x4_t(panel + krow * pstride + ncol * 2, b);
                }
                mma16816(acc[t], a, b[0], b[1], p.bf16);
                if (t + 1 < ntile8)
                    mma16816(acc[t + 1], a, b[2], b[3], p.bf16);
            }
        };
        // ... B fragments straight from global memory
        auto global_products = [&](const uint32_t (&a)[4], int kk) {
            const int k = kk * 16 + (lane & 3) * 2;
#pragma unroll
            for (int t = 0; t < 8; ++t)
            {
                if (t >= ntile8)
                    break;
                uint32_t b0, b1;
                load_b_global(p, B, n0 + t * 8 + (lane >> 2), k, b0, b1);
                mma16816(acc[t], a, b0, b1, p.bf16);
            }
        };
        // visit the row's nonzero tiles (entry, block column) in order
        auto for_each_tile = [&](auto &&fn) {
            for (int s = 0; s < p.ntiles; ++s)
            {
                const int q = rt * p.tile_rows * p.ntiles + s * p.tile_rows + ri;
                const int e1 = rowptr[q + 1];
                for (int e = rowptr[q]; e < e1; ++e)
                {
                    const int kk = colidx[e] + s * p.tile_cols;
                    if (kk >= 0 && kk < p.kb)
                        fn(e, kk);
                }
            }
        };

        for (int it = 0; it < p.num_iter; ++it)
            for_each_tile([&](int e, int kk) {
                uint32_t a[4];
                load_a(vals + (int64_t)e * 256, lane, a);
                if (PANEL)
                    panel_products(a, kk);
                else
                    global_products(a, kk);
            });

        void *Cb = reinterpret_cast<uint8_t *>(p.C) +
                   prob * p.sC * (p.out_type == KAMI_F32 ? 4 : (p.out_type == KAMI_F64 ? 8 : 2));
        const int g = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
        for (int t = 0; t < 8; ++t)
        {
            if (t >= ntile8)
                break;
            const int col = n0 + t * 8 + c;
            store_c(p, Cb, r * 16 + g, col, acc[t][0], acc[t][1]);
            store_c(p, Cb, r * 16 + g + 8, col, acc[t][2], acc[t][3]);
        }
    }
}

// ---------------------------------------------------------------------------
// Streamed form (K beyond the panel, 16-byte aligned tiles and B rows): per
// warp, a three-stage cp.async pipeline over the row's nonzero tiles -- while
// the MMAs of tile e run, tiles e+1 and e+2 (each a 512-byte A tile and the
// 16 x 64 (or 64 x 16) slice of B it multiplies) are in flight.  Column
// indices are read 32 at a time, one per lane, and broadcast by shuffle, so
// no load sits on the issue path of a tile.  A and B fragments come from
// shared memory by ldmatrix (B transposed for the K x N layout).
// ---------------------------------------------------------------------------
constexpr int kStageA = 512;
constexpr int kStageB = 64 * 48;             // N x K slice: 64 rows of 32 bytes + 16 pad (K x N: 16 x 144)
constexpr int kStage = kStageA + kStageB;    // bytes per stage
constexpr int kStages = 3;                   // cp.async stages per warp
constexpr int kWarpSmem = kStages * kStage;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_stages() { asm volatile("cp.async.wait_group %0;" ::"n"(kStages - 1) : "memory"); }

__global__ void __launch_bounds__(kWarps * 32) spmm_stream_kernel(const SpmmParams p)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.y * kCols;
    const uint32_t wbase = (uint32_t)__cvta_generic_to_shared(smem) + warp * kWarpSmem;
    const int ntile8 = min(8, (p.N - n0 + 7) / 8);
    const int m = lane >> 3, i8 = lane & 7;

    for (int64_t prob = blockIdx.z; prob < p.batch; prob += gridDim.z)
    {
        const int r = blockIdx.x * kWarps + warp;
        if (r >= p.mb)
            continue; // no CTA-wide barrier in this kernel
        const uint16_t *B = p.B + prob * p.sB;
        const int *rowptr = p.rowptr + prob * p.s_rowptr;
        const int *colidx = p.colidx + prob * p.s_colidx;
        const uint16_t *vals = p.vals + prob * p.s_vals;

        float acc[8][4];
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[t][q] = 0.f;

        // copy tile e (block column kk) and its B slice into stage st
        auto stage = [&](int st, int e, int kk) {
            const uint32_t sa = wbase + st * kStage, sb = sa + kStageA;
            cp_async16(sa + lane * 16, vals + (int64_t)e * 256 + lane * 8, true);
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int c = lane + 32 * j;
                if (p.refnk)
                {
                    const int i = c >> 1, ch = c & 1; // row n0 + i, k chunk ch
                    const bool ok = n0 + i < p.N;
                    cp_async16(sb + i * 48 + ch * 16,
                               ok ? B + (int64_t)(n0 + i) * p.ldb + kk * 16 + ch * 8 : B, ok);
                }
                else
                {
                    const int i = c >> 3, ch = c & 7; // row kk*16 + i, n chunk ch
                    const bool ok = n0 + ch * 8 < p.N;
                    cp_async16(sb + i * 144 + ch * 16, ok ? B + (int64_t)(kk * 16 + i) * p.ldb + n0 + ch * 8 : B,
                               ok);
                }
            }
        };
        auto compute = [&](int st) {
            const uint32_t sa = wbase + st * kStage, sb = sa + kStageA;
            uint32_t a[4];
            // A: matrices (rows 0-7, k 0-7), (8-15, 0-7), (0-7, 8-15), (8-15, 8-15)
            ldsm_x4(sa + ((m & 1) * 8 + i8) * 32 + (m >> 1) * 16, a);
#pragma unroll
            for (int t = 0; t < 8; t += 2)
            {
                if (t >= ntile8)
                    break;
                uint32_t b[4];
                if (p.refnk)
                    ldsm_x4(sb + ((t + (m >> 1)) * 8 + i8) * 48 + (m & 1) * 16, b);
                else
                    ldsm_x4_t(sb + ((m & 1) * 8 + i8) * 144 + (t + (m >> 1)) * 16, b);
                mma16816(acc[t], a, b[0], b[1], p.bf16);
                if (t + 1 < ntile8)
                    mma16816(acc[t + 1], a, b[2], b[3], p.bf16);
            }
        };

        const int rt = r / p.tile_rows, ri = r % p.tile_rows;
        for (int it = 0; it < p.num_iter; ++it)
            for (int s = 0; s < p.ntiles; ++s)
            {
                const int q = rt * p.tile_rows * p.ntiles + s * p.tile_rows + ri;
                const int e0 = rowptr[q], e1 = rowptr[q + 1];
                for (int w0 = e0; w0 < e1; w0 += 32)
                {
                    const int n = min(32, e1 - w0);
                    int kk = -1;
                    if (lane < n)
                        kk = colidx[w0 + lane] + s * p.tile_cols;
                    if (kk >= p.kb)
                        kk = -1; // skipped: outside [0, kb)
                    // prologue: tiles 0 .. kStages-2 in flight
#pragma unroll
                    for (int j = 0; j < kStages - 1; ++j)
                    {
                        const int kj = __shfl_sync(0xffffffffu, kk, j);
                        if (j < n && kj >= 0)
                            stage(j, w0 + j, kj);
                        cp_async_commit();
                    }
                    for (int i = 0; i < n; ++i)
                    {
                        const int ia = i + kStages - 1; // tile issued now
                        const int kn = __shfl_sync(0xffffffffu, kk, ia & 31);
                        if (ia < n && kn >= 0)
                            stage(ia % kStages, w0 + ia, kn);
                        cp_async_commit();
                        cp_async_wait_stages(); // tile i has landed
                        __syncwarp();
                        if (__shfl_sync(0xffffffffu, kk, i) >= 0)
                            compute(i % kStages);
                        __syncwarp(); // stage i % kStages is refilled kStages - 1 tiles later
                    }
                }
            }

        void *Cb = reinterpret_cast<uint8_t *>(p.C) + prob * p.sC * (p.out_type == KAMI_F32 ? 4 : 2);
        const int g = lane >> 2, c = (lane & 3) * 2;
#pragma unroll
        for (int t = 0; t < 8; ++t)
        {
            if (t >= ntile8)
                break;
            const int col = n0 + t * 8 + c;
            store_c(p, Cb, r * 16 + g, col, acc[t][0], acc[t][1]);
            store_c(p, Cb, r * 16 + g + 8, col, acc[t][2], acc[t][3]);
        }
    }
}

int spmm_launch(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int N, int64_t batch,
                const int *rowptr, const int *colidx, int64_t s_rowptr, int64_t s_colidx, const void *vals,
                int64_t s_vals, const void *B, int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, void *C,
                int64_t ldc, int64_t strideC, double alpha, double beta, int num_iter, int tile_rows,
                int ntiles, int tile_cols, void *stream)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "spmm: in_type must be KAMI_F16 or KAMI_BF16");
    if (out_type != KAMI_F16 && out_type != KAMI_BF16 && out_type != KAMI_F32)
        return fail(KAMI_ERR_UNSUPPORTED, "spmm: out_type must be KAMI_F32, KAMI_F16 or KAMI_BF16");
    if (bsr != 16)
        return fail(KAMI_ERR_UNSUPPORTED, "spmm: only 16 x 16 tiles (bsr = 16)");
    if (mb < 0 || kb < 1 || N < 0 || batch < 0 || num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: bad shape or num_iter");
    if (b_layout != KAMI_B_REF_NK && b_layout != KAMI_B_ROW_KN)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: bad b_layout");
    if (mb == 0 || N == 0 || batch == 0)
        return KAMI_OK;
    if (!rowptr || !colidx || !vals || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: null pointer");
    const int64_t K = (int64_t)kb * 16;
    if (ldb < (b_layout == KAMI_B_REF_NK ? K : N) || ldc < N)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: leading dimension too small");
    if ((reinterpret_cast<uintptr_t>(vals) & 3) || (s_vals & 1))
        return fail(KAMI_ERR_MISALIGNED, "spmm: value tiles must be 4-byte aligned");
    if (tile_rows < 1 || ntiles < 1 || (ntiles > 1 && tile_cols < 1) || mb % tile_rows)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: bad tile description");

    SpmmParams p{};
    p.mb = mb;
    p.kb = kb;
    p.N = N;
    p.batch = batch;
    p.rowptr = rowptr;
    p.colidx = colidx;
    p.s_rowptr = s_rowptr;
    p.s_colidx = s_colidx;
    p.vals = reinterpret_cast<const uint16_t *>(vals);
    p.s_vals = s_vals;
    p.B = reinterpret_cast<const uint16_t *>(B);
    p.ldb = ldb;
    p.sB = strideB;
    p.refnk = b_layout == KAMI_B_REF_NK;
    p.C = C;
    p.ldc = ldc;
    p.sC = strideC;
    p.out_type = out_type;
    p.bf16 = in_type == KAMI_BF16;
    p.alpha = alpha;
    p.beta = beta;
    p.num_iter = num_iter;
    p.tile_rows = tile_rows;
    p.ntiles = ntiles;
    p.tile_cols = ntiles > 1 ? tile_cols : 0;
    const int osz = out_type == KAMI_F32 ? 4 : 2;
    p.c_vec = !(reinterpret_cast<uintptr_t>(C) % (2 * osz)) && !(ldc & 1) && !(strideC & 1);
    p.b_vec = !(reinterpret_cast<uintptr_t>(B) & 15) && !(ldb & 7) && !(strideB & 7);

    const bool panel = K <= kPanelMaxK;
    const int pstride = p.refnk ? (int)K * 2 + 16 : kCols * 2 + 16;
    const size_t smem = panel ? (size_t)(p.refnk ? kCols : K) * pstride : 0;
    const dim3 grid((unsigned)((mb + kWarps - 1) / kWarps), (unsigned)((N + kCols - 1) / kCols),
                    (unsigned)(batch < 65535 ? batch : 65535));
    if (grid.y > 65535)
        return fail(KAMI_ERR_UNSUPPORTED, "spmm: N above %d", 65535 * kCols);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // one large problem: the tcgen05 kernel (spmm_tc05.cu), B as K x N or N x K
    if (!panel && batch == 1 && tile_rows == 1 && ntiles == 1)
    {
        const int s5 = spmm_tc05_launch(p.bf16 != 0, out_type, mb, kb, N, rowptr, colidx, vals, B, ldb, p.refnk != 0,
                                        C, ldc, alpha, beta, num_iter, st);
        if (s5 != KAMI_ERR_UNSUPPORTED)
            return s5;
    }
    void *args[] = {&p};
    cudaError_t e;
    // streamed form: 16-byte aligned tiles and B rows, whole 8-column groups
    const bool streamable = !panel && p.b_vec && !(reinterpret_cast<uintptr_t>(vals) & 15) && !(s_vals & 7) &&
                            (p.refnk || !(N & 7));
    if (panel) // at most 64 x 528 or 256 x 144 bytes: below the 48 KB default limit
        e = cudaLaunchKernel((const void *)&spmm_kernel<true>, grid, dim3(kWarps * 32), args, smem, st);
    else if (streamable) // 4 warps x 10.5 KB
        e = cudaLaunchKernel((const void *)&spmm_stream_kernel, grid, dim3(kWarps * 32), args,
                             (size_t)kWarps * kWarpSmem, st);
    else
        e = cudaLaunchKernel((const void *)&spmm_kernel<false>, grid, dim3(kWarps * 32), args, 0, st);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(spmm_kernel)");
    return KAMI_OK;
}

} // namespace
} // namespace kami

using namespace kami;

extern "C" int kami_spmm_bsr(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int N,
                             int64_t batch, const int *row_ptr, const int *col_idx, int64_t stride_row_ptr,
                             int64_t stride_col_idx, const void *vals, int64_t stride_vals, const void *B,
                             int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, void *C, int64_t ldc,
                             int64_t strideC, double alpha, double beta, int num_iter, void *stream)
{
    return spmm_launch(in_type, out_type, bsr, mb, kb, N, batch, row_ptr, col_idx, stride_row_ptr,
                       stride_col_idx, vals, stride_vals, B, ldb, strideB, b_layout, C, ldc, strideC, alpha, beta,
                       num_iter, 1, 1, 0, stream);
}

extern "C" int kami_spmm_tilebsr(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int N,
                                 int64_t batch, int tile_rows, int tile_cols, const int *blk_row_ptr,
                                 const int *blk_col_idx, int64_t stride_row_ptr, int64_t stride_col_idx,
                                 const void *vals, int64_t stride_vals, const void *B, int64_t ldb,
                                 int64_t strideB, kami_b_layout_t b_layout, void *C, int64_t ldc, int64_t strideC,
                                 double alpha, double beta, int num_iter, void *stream)
{
    if (tile_rows < 1 || tile_cols < 1 || mb % tile_rows || kb % tile_cols)
        return fail(KAMI_ERR_INVALID_VALUE, "spmm: tile_rows must divide mb and tile_cols must divide kb");
    return spmm_launch(in_type, out_type, bsr, mb, kb, N, batch, blk_row_ptr, blk_col_idx, stride_row_ptr,
                       stride_col_idx, vals, stride_vals, B, ldb, strideB, b_layout, C, ldc, strideC, alpha, beta,
                       num_iter, tile_rows, kb / tile_cols, tile_cols, stream);
}

extern "C" int kami_bsr_to_tilebsr(int mb, int kb, int tile_rows, int tile_cols, const int *row_ptr,
                                   const int *col_idx, int *blk_row_ptr, int *blk_col_idx, int *perm)
{
    if (mb < 0 || kb < 1 || tile_rows < 1 || tile_cols < 1 || mb % tile_rows || kb % tile_cols)
        return fail(KAMI_ERR_INVALID_VALUE, "bsr_to_tilebsr: tile_rows must divide mb and tile_cols must divide kb");
    if (!row_ptr || !blk_row_ptr || (row_ptr[mb] > 0 && (!col_idx || !blk_col_idx)))
        return fail(KAMI_ERR_INVALID_VALUE, "bsr_to_tilebsr: null pointer");
    const int row_tiles = mb / tile_rows, col_tiles = kb / tile_cols;
    int count = 0;
    blk_row_ptr[0] = 0;
    for (int i = 0; i < row_tiles; ++i)
        for (int s = 0; s < col_tiles; ++s)
        {
            const int lo = s * tile_cols, hi = lo + tile_cols;
            for (int ri = 0; ri < tile_rows; ++ri)
            {
                const int r = i * tile_rows + ri;
                for (int e = row_ptr[r]; e < row_ptr[r + 1]; ++e)
                {
                    const int c = col_idx[e];
                    if (c >= lo && c < hi)
                    {
                        if (perm)
                            perm[count] = e;
                        blk_col_idx[count++] = c - lo;
                    }
                }
                blk_row_ptr[(i * col_tiles + s) * tile_rows + ri + 1] = count;
            }
        }
    return count;
}
