// tc05_gemm.cu -- the tcgen05 variant of the block GEMM (FP16/BF16 inputs,
// FP32 accumulation in tensor memory).
//
// One CTA (4 warps) per problem.  Thread 0 loads the whole problem -- A
// (M x K) and B (N x K, the reference's operand) -- into shared memory with
// TMA (128-byte swizzle, 64-element K boxes), then issues every
// tcgen05.mma of the problem back to back into a TMEM accumulator
// (M = 64 or 128 rows of TMEM lanes, N columns) and commits to an mbarrier;
// all four warps read the accumulator back with tcgen05.ld and store C.
// Several CTAs share an SM (shared memory and TMEM permitting), so one
// CTA's loads and stores overlap another CTA's MMAs.
//
// The reference's partitions map onto how the MMAs are issued:
//   1D  one M x N MMA per k-step (N <= 256);
//   2D  N split into P column panels, P MMAs of M x N/P per k-step, each
//       into its own accumulator columns;
//   3D  K split into P depth slices, each accumulated in its own TMEM
//       accumulator, the P partials summed on the device in the epilogue
//       (the reference sums its 3D slices on the host,
//       block_gemm_3d_half_mma.cu:291-300).
// num_iter repeats the MMA chain on the resident operands, the reference's
// in-register repeat (NUM_ITER, block_gemm_1d_half_mma.cu:130).
//
// Every mbarrier wait is bounded; on a timeout the kernel records an error
// in g_tc05_error, waits (bounded) for its copies in flight, frees TMEM and
// returns.
#include <mutex>

#include "kami_common.cuh"
#include "tc05_gemm.cuh"
#include "tc05_ptx.cuh"

namespace kami {

__device__ int g_tc05_error = 0;

struct Tc05Params
{
    GemmArgs g;
    int bm;             // MMA M (64 or 128)
    int bn;             // padded N (B box rows)
    int nkb;            // 64-element K boxes
    int ksteps;         // 16-element MMA k-steps
    int part, P;
    int a_mn, b_mn;     // operand stored MN-major (A as K x M, B as K x N)
    int a_tmem;         // A resident in tensor memory (TS form) instead of shared memory
    uint32_t a_col;     // first TMEM column of A in the TS form
    uint32_t idesc;     // instruction descriptor (N = bn, or bn / P for 2D)
    uint32_t tmem_cols; // allocated TMEM columns (power of two >= 32)
    uint64_t timeout_ns;
};

__device__ __forceinline__ void tc05_flag(int code) { atomicExch(&g_tc05_error, code); }

template <bool BF16>
__global__ void __launch_bounds__(128) tc05_block_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB,
                                                         const Tc05Params p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment of the swizzle atoms
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_box = p.a_tmem ? 0 : p.bm * 128, b_box = p.bn * 128;
    uint8_t *sA = smem;
    uint8_t *sB = sA + p.nkb * a_box;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + p.nkb * b_box); // [0] loads landed, [1] MMAs done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
    int *ok_slot = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int prob = blockIdx.x;
    const GemmArgs &g = p.g;

    if (threadIdx.x == 0)
    {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::fence_mbar_init();
        *ok_slot = 1;
    }
    __syncwarp();
    if (warp == 0)
    {
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0)
    {
        const uint32_t bytes = (uint32_t)(p.nkb * (a_box + b_box)); // a_box is 0 when A lives in TMEM
        tc::mbar_expect_tx(&bars[0], bytes);
        for (int kb = 0; kb < p.nkb; ++kb)
        {
            if (!p.a_tmem)
            {
                if (p.a_mn)
                    for (int mc = 0; mc < p.bm / 64; ++mc)
                        tc::tma_load_3d(sA + kb * a_box + mc * 8192, &tmA, &bars[0], mc * 64, kb * 64, prob);
                else
                    tc::tma_load_3d(sA + kb * a_box, &tmA, &bars[0], kb * 64, 0, prob);
            }
            if (p.b_mn)
                for (int nc = 0; nc < p.bn / 64; ++nc)
                    tc::tma_load_3d(sB + kb * b_box + nc * 8192, &tmB, &bars[0], nc * 64, kb * 64, prob);
            else
                tc::tma_load_3d(sB + kb * b_box, &tmB, &bars[0], kb * 64, 0, prob);
        }
    }
    __syncwarp(); // tcgen05.st below is .sync.aligned
    if (p.a_tmem)
    {
        // A -> TMEM: warp w writes lanes 32w..32w+31, thread t holds row 32w+t,
        // 16 columns (32 K elements) per tcgen05.st; zero beyond M and K
        const int row = warp * 32 + lane;
        const uint16_t *arow = reinterpret_cast<const uint16_t *>(g.A) + (int64_t)prob * g.sA + (int64_t)row * g.lda;
        const int ncols = ((p.ksteps * 8) + 15) / 16 * 16;
        for (int c0 = 0; c0 < ncols; c0 += 16)
        {
            uint32_t v[16];
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int k = c0 * 2 + q * 8;
                uint4 x = make_uint4(0, 0, 0, 0);
                if (row < g.M && k < g.K)
                    x = __ldg(reinterpret_cast<const uint4 *>(arow + k));
                v[4 * q + 0] = x.x;
                v[4 * q + 1] = x.y;
                v[4 * q + 2] = x.z;
                v[4 * q + 3] = x.w;
            }
            tc::tmem_st16(tmem + ((uint32_t)(warp * 32) << 16) + p.a_col + c0, v);
        }
        tc::tmem_st_wait();
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
    }
    if (threadIdx.x == 0)
    {
        if (!tc::mbar_wait_bounded(&bars[0], 0, p.timeout_ns))
        {
            tc05_flag(1);
            *ok_slot = 0;
            tc::mbar_wait_bounded(&bars[0], 0, p.timeout_ns); // copies still in flight
            tc::mbar_arrive(&bars[1]);
        }
        else
        {
            tc::tc_fence_after();
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            const int depth = p.part == 3 ? p.P : 1;
            const int panels = p.part == 2 ? p.P : 1;
            const int pn = p.bn / panels;
            for (int it = 0; it < g.num_iter; ++it)
            {
                for (int d = 0; d < depth; ++d)
                {
                    const int k_lo = p.ksteps * d / depth, k_hi = p.ksteps * (d + 1) / depth;
                    const uint32_t acc_col = (uint32_t)(d * p.bn);
                    for (int ks = k_lo; ks < k_hi; ++ks)
                    {
                        const int kb = ks >> 2, kin = ks & 3;
                        const uint64_t adesc = p.a_mn ? tc::desc_mnmajor_sw128(a0 + kb * a_box + kin * 2048, 8192)
                                                      : tc::desc_kmajor_sw128(a0 + kb * a_box + kin * 32);
                        const uint32_t acc = (it > 0 || ks > k_lo) ? 1u : 0u;
                        const uint32_t a_tm = tmem + p.a_col + (uint32_t)ks * 8;
                        for (int q = 0; q < panels; ++q)
                        {
                            const uint64_t bdesc =
                                p.b_mn ? tc::desc_mnmajor_sw128(b0 + kb * b_box + (q * pn / 64) * 8192 + kin * 2048, 8192)
                                       : tc::desc_kmajor_sw128(b0 + kb * b_box + q * pn * 128 + kin * 32);
                            if (p.a_tmem)
                                tc::mma_f16_ts(tmem + acc_col + q * pn, a_tm, bdesc, p.idesc, acc);
                            else
                                tc::mma_f16_ss(tmem + acc_col + q * pn, adesc, bdesc, p.idesc, acc);
                        }
                    }
                }
            }
            tc::mma_commit(&bars[1]);
        }
    }
    __syncwarp();

    // ---- epilogue: TMEM -> registers -> C ----
    // tcgen05.ld is .sync.aligned: the outcome must be warp-uniform
    const bool done = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&bars[1], 0, p.timeout_ns));
    tc::tc_fence_after();
    if (!done)
        tc05_flag(2);
    const bool ok = done && *reinterpret_cast<volatile int *>(ok_slot);
    if (ok)
    {
        const int row = p.bm == 128 ? warp * 32 + lane : warp * 16 + lane;
        const bool row_ok = (p.bm == 128 || lane < 16) && row < g.M;
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        const int depth = p.part == 3 ? p.P : 1;
        const int osz = g.out_type == KAMI_F32 ? 4 : 2;
        void *Cb = reinterpret_cast<char *>(g.C) + (int64_t)prob * g.sC * osz;
        const bool fast = g.out_type == KAMI_F32 && g.alpha == 1.0 && g.beta == 0.0 && g.c_vec &&
                          (g.ldc % 4 == 0) && (g.sC % 4 == 0) && ((reinterpret_cast<uintptr_t>(g.C) & 15) == 0);
        for (int c0 = 0; c0 < p.bn; c0 += 16)
        {
            uint32_t v[16];
            tc::tmem_ld16(tmem + lane_addr + c0, v);
            tc::tmem_ld_wait();
            float f[16];
#pragma unroll
            for (int e = 0; e < 16; ++e)
                f[e] = __uint_as_float(v[e]);
            for (int d = 1; d < depth; ++d)
            {
                uint32_t w[16];
                tc::tmem_ld16(tmem + lane_addr + d * p.bn + c0, w);
                tc::tmem_ld_wait();
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    f[e] += __uint_as_float(w[e]);
            }
            if (row_ok)
            {
                if (fast && c0 + 16 <= g.N)
                {
                    float4 *dst = reinterpret_cast<float4 *>(reinterpret_cast<float *>(Cb) + (int64_t)row * g.ldc + c0);
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        dst[e] = make_float4(f[4 * e], f[4 * e + 1], f[4 * e + 2], f[4 * e + 3]);
                }
                else
                {
#pragma unroll
                    for (int e = 0; e < 16; e += 2)
                        store_pair<float>(g, Cb, row, c0 + e, f[e], f[e + 1]);
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        __syncwarp();
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, p.tmem_cols);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    });
    return fn;
}

// 3D map {K, rows, batch} over a K-major operand, box {64, box_rows, 1},
// 128-byte swizzle, zero fill out of bounds.  With mn_major the operand is
// stored K x rows (rows contiguous): map {rows, K, batch}, box {64, 64, 1}.
static int make_map(CUtensorMap *map, bool bf16, const void *base, int K, int rows, int64_t batch, int64_t ld,
                    int64_t stride, int box_rows, bool mn_major = false)
{
    if (mn_major)
    {
        EncodeTiledFn fn = encode_fn();
        if (!fn)
            return fail(KAMI_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
        cuuint64_t dims[3] = {(cuuint64_t)rows, (cuuint64_t)K, (cuuint64_t)batch};
        const int64_t s2 = batch > 1 ? stride : (int64_t)K * ld;
        cuuint64_t strides[2] = {(cuuint64_t)(ld * 2), (cuuint64_t)(s2 * 2)};
        cuuint32_t box[3] = {64, 64, 1};
        cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = fn(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                        const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return fail(KAMI_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled failed (%d) for an MN-major operand", (int)r);
        return KAMI_OK;
    }
    EncodeTiledFn fn = encode_fn();
    if (!fn)
        return fail(KAMI_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
    const int64_t s2 = batch > 1 ? stride : (int64_t)rows * ld;
    cuuint64_t strides[2] = {(cuuint64_t)(ld * 2), (cuuint64_t)(s2 * 2)};
    cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                    const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(KAMI_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled failed (%d) for K=%d rows=%d ld=%lld", (int)r, K,
                    rows, (long long)ld);
    return KAMI_OK;
}

struct Tc05Shape
{
    int bm, bn, nkb, ksteps, part, P, a_mn, b_mn, a_tmem;
    uint32_t a_col;
    uint32_t tmem_cols;
    size_t smem;
};

static size_t smem_bytes(int bm, int bn, int nkb) { return (size_t)nkb * (bm + bn) * 128 + 1024 + 64; }

static int tc05_shape(int in_type, int out_type, int partition, int P, int M, int N, int K, int a_layout,
                      int b_layout, Tc05Shape *s, int a_tmem = 0)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: FP16/BF16 inputs only");
    if (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: FP32/FP16/BF16 output only");
    const int a_mn = a_layout == KAMI_A_COL_MK ? 1 : 0, b_mn = b_layout == KAMI_B_ROW_KN ? 1 : 0;
    if (M > 128 || N > 256 || K > 256)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: M <= 128, N <= 256, K <= 256 (got %d, %d, %d)", M, N, K);
    if (K % 8)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: K must be a multiple of 8");
    const int part = partition == KAMI_PARTITION_AUTO ? KAMI_PARTITION_1D : partition;
    const int bm = M <= 64 ? 64 : 128;
    const int ngran = 16; // MMA N granule; also keeps every 16-column TMEM read inside the allocation
    int p = part == KAMI_PARTITION_1D ? 1 : (P > 0 ? P : 2);
    if (part != KAMI_PARTITION_1D && p != 2 && p != 4)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: P must be 2 or 4 for 2D/3D");
    int bn = (N + ngran - 1) / ngran * ngran;
    if (part == KAMI_PARTITION_2D)
        bn = (N + ngran * p - 1) / (ngran * p) * (ngran * p);
    if (b_mn)
    {
        // MN-major B is staged in 64-column swizzle boxes; 2D panels must be whole boxes
        bn = (N + 63) / 64 * 64;
        if (part == KAMI_PARTITION_2D && (bn / p) % 64)
            return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: 2D panels of an N-major B must be multiples of 64");
    }
    if (bn > 256)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: padded N %d exceeds 256", bn);
    const int ksteps = (K + 15) / 16;
    if (part == KAMI_PARTITION_3D && ksteps < p)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: 3D needs at least P k-steps of 16");
    const int acc_cols = (part == KAMI_PARTITION_3D ? p : 1) * bn;
    int cols = acc_cols;
    if (a_tmem)
    {
        if (bm != 128 || a_mn)
            return fail(KAMI_ERR_UNSUPPORTED,
                        "tcgen05 A-in-TMEM form: M must be 65..128 and A row-major (M x K)");
        cols += ((K + 15) / 16 * 8 + 15) / 16 * 16; // two K elements per 32-bit column
    }
    if (cols > 512)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: %d TMEM columns needed, 512 available", cols);
    uint32_t tc = 32;
    while ((int)tc < cols)
        tc <<= 1;
    const int nkb = (K + 63) / 64;
    s->bm = bm;
    s->bn = bn;
    s->nkb = nkb;
    s->ksteps = ksteps;
    s->part = part;
    s->P = p;
    s->a_mn = a_mn;
    s->b_mn = b_mn;
    s->a_tmem = a_tmem;
    s->a_col = (uint32_t)acc_cols;
    s->tmem_cols = tc;
    s->smem = smem_bytes(a_tmem ? 0 : bm, bn, nkb);
    if (s->smem > 227 * 1024)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: %zu bytes of shared memory", s->smem);
    return KAMI_OK;
}

bool tc05_prefer(int in_type, int partition, int M, int N, int K, int a_layout, int b_layout)
{
    // the tensor-memory path wins where one MMA tile holds the problem
    // densely; tiny problems stay on mma.sync (see the variant sweep)
    (void)a_layout;
    (void)b_layout;
    return (in_type == KAMI_F16 || in_type == KAMI_BF16) && M > 32 && M <= 128 && N <= 256 && N >= 32 && K <= 256 &&
           K % 8 == 0;
}

// AUTO keeps A in shared memory until the TS form is measured faster
bool tc05_prefer_ts(int M, int a_layout) { return false && M > 64 && a_layout == KAMI_A_ROW_MK; }

int tc05_plan(int in_type, int out_type, int partition, int P, int M, int N, int K, int64_t batch, int a_layout,
              int b_layout, LaunchInfo *info, int a_tmem)
{
    Tc05Shape s;
    int st = tc05_shape(in_type, out_type, partition, P, M, N, K, a_layout, b_layout, &s, a_tmem);
    if (st)
        return st;
    info->variant = a_tmem ? KAMI_VARIANT_TCGEN05_TS : KAMI_VARIANT_TCGEN05;
    info->partition = s.part;
    info->P = s.P;
    info->threads = 128;
    info->smem = (int)s.smem;
    info->problems_per_cta = 1;
    info->grid = batch;
    return KAMI_OK;
}

int tc05_launch(const GemmArgs &g, int in_type, int partition, int P, void *, size_t, cudaStream_t stream,
                int a_tmem)
{
    Tc05Shape s;
    int st = tc05_shape(in_type, g.out_type, partition, P, g.M, g.N, g.K, g.a_layout, g.b_layout, &s, a_tmem);
    if (st)
        return st;
    const bool bf16 = in_type == KAMI_BF16;
    if ((reinterpret_cast<uintptr_t>(g.A) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15) || g.lda % 8 ||
        g.ldb % 8 || (g.batch > 1 && (g.sA % 8 || g.sB % 8 || g.sA == 0 || g.sB == 0)))
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: TMA needs 16-byte aligned bases and strides");
    if (g.batch > 0x7fffffff)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant: batch above 2^31-1");
    CUtensorMap ma, mb;
    st = make_map(&ma, bf16, g.A, g.K, g.M, g.batch, g.lda, g.sA, s.bm, s.a_mn != 0);
    if (st)
        return st;
    st = make_map(&mb, bf16, g.B, g.K, g.N, g.batch, g.ldb, g.sB, s.bn, s.b_mn != 0);
    if (st)
        return st;
    Tc05Params p{};
    p.g = g;
    p.bm = s.bm;
    p.bn = s.bn;
    p.nkb = s.nkb;
    p.ksteps = s.ksteps;
    p.part = s.part;
    p.P = s.P;
    p.a_mn = s.a_mn;
    p.b_mn = s.b_mn;
    p.a_tmem = s.a_tmem;
    p.a_col = s.a_col;
    p.idesc = tc::idesc_f16(bf16, s.bm, s.part == KAMI_PARTITION_2D ? s.bn / s.P : s.bn, s.a_mn, s.b_mn);
    p.tmem_cols = s.tmem_cols;
    const double mmas = (double)g.num_iter * s.ksteps * (s.part == KAMI_PARTITION_2D ? s.P : 1);
    p.timeout_ns = (uint64_t)(5e8 + mmas * 2000.0);

    const void *fn = bf16 ? (const void *)&tc05_block_kernel<true> : (const void *)&tc05_block_kernel<false>;
    static std::once_flag once[2];
    cudaError_t e = cudaSuccess;
    std::call_once(once[bf16 ? 1 : 0], [&] {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(tc05_block_kernel)");
    void *args[] = {&ma, &mb, &p};
    e = cudaLaunchKernel(fn, dim3((unsigned)g.batch), dim3(128), args, s.smem, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(tc05_block_kernel)");
    return KAMI_OK;
}

// Failure-detection self test: one thread waits on an mbarrier that nothing
// arrives at, with the same bounded wait the GEMM kernels use, and records
// code 4 in the status word when the wait gives up.
__global__ void bounded_wait_selftest_kernel(uint64_t limit_ns)
{
    __shared__ uint64_t bar;
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
    if (!tc::mbar_wait_bounded(&bar, 0, limit_ns))
        tc05_flag(4);
}

int tc05_selftest_bounded_wait(uint64_t limit_ns, cudaStream_t s)
{
    bounded_wait_selftest_kernel<<<1, 1, 0, s>>>(limit_ns);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(e, "bounded_wait_selftest_kernel");
    return KAMI_OK;
}

int tc05_read_error(int *flag)
{
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(flag, g_tc05_error, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyFromSymbol(g_tc05_error)");
    e = cudaMemcpyToSymbol(g_tc05_error, &zero, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyToSymbol(g_tc05_error)");
    return KAMI_OK;
}

} // namespace kami
