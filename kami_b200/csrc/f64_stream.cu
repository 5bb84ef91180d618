// f64_stream.cu -- persistent batched FP64 block GEMM for the streamed regime
// (M, N, K <= 64, few repeats), the shape of the reference's batched FP64
// programs (src/batched_gemm/KAMI/{1d,2d,3d}/batched_gemm_*_double_mma.cu:
// one problem per CTA, operands loaded, DMMA m16n8k8, C stored).
//
// There, and in this library's per-problem kernel, a CTA first loads its
// problem and then multiplies it, so the loads and the DMMAs of one CTA never
// overlap; at 64^3 the two take about the same time (HBM: 64 KB per problem;
// DMMA: 0.5 MFLOP per problem) and the kernel runs near their sum.  Here one
// CTA per SM walks its problems j = blockIdx.x, + gridDim.x, ... through a
// ring of three shared-memory stages:
//   warp 8      (one lane) issues the TMA box loads of problems j + 1 and
//               j + 2 into the free stages while problem j is multiplied --
//               16 boxes per problem (per-row bulk copies and per-thread
//               16-byte copies both measured slower);
//   warps 0-7   multiply problem j from shared memory: warp w owns the
//               16-row band (w % 4) and the 32-column half (w / 4) of C, all
//               of K, four n8 tiles of m16n8k8 DMMAs, and store C straight
//               from their accumulators.
// The k index is permuted identically for A and B within each k-step of 8
// (lane t holds k = 2t, 2t+1), so every operand fetch is one 16-byte shared
// load; K = 64 has a fully unrolled body.  Barriers: full[s] (TMA, by bytes),
// empty[s] (8 compute warps).  Every wait is bounded; a failed wait sets the
// library's device status word and ends the CTA's loop.
#include <cstdint>
#include <mutex>

#include "kami_common.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device status of the bounded waits (read and cleared by kami_device_status)
__device__ int g_f64s_error = 0;

namespace {

// One stage holds a problem's A and B as eight 8-column boxes each (64 rows x
// 64 bytes, the TMA 64-byte swizzle: the 16-byte chunk c of row r sits at
// chunk c ^ ((r / 2) % 4)), so the two rows a quarter-warp's fragment fetch
// touches share one 128-byte line without bank conflicts.
constexpr int kBox = 64 * 64;                     // bytes of one 64 x 8 box
constexpr int kTile = 8 * kBox;                   // one operand: K up to 64
constexpr int kStage = 2 * kTile;                 // A then B
constexpr int kStages = 3;                        // two problems in flight while one is multiplied
constexpr int kComputeWarps = 8;
constexpr int kThreads = (kComputeWarps + 1) * 32;
constexpr size_t kSmem = kStages * kStage + 64 + 1024; // stages, barriers, alignment slack

struct F64sParams
{
    CUtensorMap mapA, mapB; // {K, rows, batch}, box {8, 64, 1}, 64-byte swizzle, zero fill
    GemmArgs g;
    int kboxes;             // boxes per operand: ceil(K / 8)
    uint64_t timeout_ns;
};

__device__ __forceinline__ double2 lds_d2(uint32_t a)
{
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a) : "memory");
    return v;
}

__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], double b0, double b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

// shared address of elements (r, 8 ks + 2 t) and (r, 8 ks + 2 t + 1) of a staged operand
__device__ __forceinline__ uint32_t frag_addr(uint32_t base, int r, int ks, int t)
{
    return base + ks * kBox + r * 64 + ((t ^ ((r >> 1) & 3)) << 4);
}

// One k-step of 8 for this warp: the A fragment of its 16 rows and the B
// fragments of its n8 tiles (ntl of 4 live), then the DMMAs.  The k index is
// permuted identically for A and B: lane t holds k = 2t, 2t+1 of the step.
__device__ __forceinline__ void kstep(uint32_t sa, uint32_t sb, int row0, int col0, int gq, int tq, int ks, int ntl,
                                      double (&acc)[4][4])
{
    const double2 lo = lds_d2(frag_addr(sa, row0 + gq, ks, tq));
    const double2 hi = lds_d2(frag_addr(sa, row0 + gq + 8, ks, tq));
    const double a[4] = {lo.x, hi.x, lo.y, hi.y};
#pragma unroll
    for (int n = 0; n < 4; ++n)
    {
        if (n >= ntl)
            break;
        const double2 v = lds_d2(frag_addr(sb, col0 + 8 * n + gq, ks, tq));
        dmma(acc[n], a, v.x, v.y);
    }
}

template <bool K64>
__global__ void __launch_bounds__(kThreads, 1) f64_stream_kernel(const __grid_constant__ F64sParams fp)
{
    const GemmArgs &g = fp.g;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kStages * kStage);
    uint64_t *empty = full + kStages;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const uint64_t limit = fp.timeout_ns;
    if (t == 0)
    {
        for (int b = 0; b < kStages; ++b)
        {
            tc::mbar_init(&full[b], 1);
            tc::mbar_init(&empty[b], kComputeWarps);
        }
        tc::fence_mbar_init();
    }
    __syncthreads();

    if (warp == kComputeWarps)
    {
        // ---- producer: 2 x kboxes TMA boxes per problem (rows past M / N
        //      and columns past K arrive as zeros) ----
        if (lane == 0)
        {
            tc::prefetch_tmap(&fp.mapA);
            tc::prefetch_tmap(&fp.mapB);
            const uint32_t bytes = (uint32_t)(2 * fp.kboxes * kBox);
            int j = 0;
            for (int64_t prob = blockIdx.x; prob < g.batch; prob += gridDim.x, ++j)
            {
                const int b = j % kStages;
                if (j >= kStages && !tc::mbar_wait_bounded(&empty[b], ((j / kStages) - 1) & 1, limit))
                {
                    atomicExch(&g_f64s_error, 1);
                    break;
                }
                uint8_t *st = smem + b * kStage;
                tc::mbar_expect_tx(&full[b], bytes);
                for (int kb = 0; kb < fp.kboxes; ++kb)
                {
                    tc::tma_load_3d(st + kb * kBox, &fp.mapA, &full[b], 8 * kb, 0, (int)prob);
                    tc::tma_load_3d(st + kTile + kb * kBox, &fp.mapB, &full[b], 8 * kb, 0, (int)prob);
                }
            }
            // no copy may still be landing when the CTA exits (only possible
            // after a failed wait of the compute warps)
            if (j > 0 && !tc::mbar_wait_bounded(&full[(j - 1) % kStages], ((j - 1) / kStages) & 1, limit))
                atomicExch(&g_f64s_error, 2);
        }
        return;
    }

    // ---- compute: warp w -> rows 16 (w % 4) .. +15, columns 32 (w / 4) .. +31 ----
    const int mt = warp & 3, nh = warp >> 2;
    const int gq = lane >> 2, tq = lane & 3;
    const int row0 = 16 * mt, col0 = 32 * nh;
    const bool rows_live = row0 < g.M;
    int ntl = (g.N - col0 + 7) / 8; // live n8 tiles of this warp
    ntl = ntl < 0 ? 0 : (ntl > 4 ? 4 : ntl);
    const int ksteps = fp.kboxes;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    int j = 0;
    for (int64_t prob = blockIdx.x; prob < g.batch; prob += gridDim.x, ++j)
    {
        const int b = j % kStages;
        if (!__all_sync(0xffffffffu, tc::mbar_wait_bounded(&full[b], (j / kStages) & 1, limit)))
        {
            atomicExch(&g_f64s_error, 3);
            break;
        }
        const uint32_t sa = sbase + b * kStage, sb = sa + kTile;
        double acc[4][4];
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                acc[n][e] = 0.0;
        if (rows_live && ntl > 0)
        {
            for (int it = 0; it < g.num_iter; ++it)
            {
                if constexpr (K64)
                {
#pragma unroll
                    for (int ks = 0; ks < 8; ++ks)
                        kstep(sa, sb, row0, col0, gq, tq, ks, ntl, acc);
                }
                else
                {
                    for (int ks = 0; ks < ksteps; ++ks)
                        kstep(sa, sb, row0, col0, gq, tq, ks, ntl, acc);
                }
            }
        }
        // the stage is free once every compute warp has read it
        __syncwarp();
        if (lane == 0)
            tc::mbar_arrive(&empty[b]);
        if (rows_live)
        {
            void *Cb = reinterpret_cast<double *>(g.C) + prob * g.sC;
#pragma unroll
            for (int n = 0; n < 4; ++n)
            {
                if (n >= ntl)
                    break;
                const int col = col0 + 8 * n + 2 * tq;
                store_pair<double>(g, Cb, row0 + gq, col, acc[n][0], acc[n][1]);
                store_pair<double>(g, Cb, row0 + gq + 8, col, acc[n][2], acc[n][3]);
            }
        }
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
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

// {K, rows, batch} FP64 map, box {8, 64, 1}, 64-byte swizzle, zero fill
bool make_map_f64(CUtensorMap *map, const void *base, int K, int rows, int64_t batch, int64_t ld, int64_t stride)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn)
        return false;
    cuuint64_t dims[3] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)batch};
    const int64_t s2 = batch > 1 ? stride : (int64_t)rows * ld;
    cuuint64_t strides[2] = {(cuuint64_t)(ld * 8), (cuuint64_t)((s2 > 0 ? s2 : ld * rows) * 8)};
    cuuint32_t box[3] = {8, 64, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace

// Runs the persistent streamed FP64 kernel when it applies (FP64 in and out,
// 48 < M <= 64, 32 < N <= 64, 32 <= K <= 64, row-major A and the reference's
// N x K B, 16-byte aligned rows and problem strides for the tensor maps); else
// returns
// KAMI_ERR_UNSUPPORTED without launching anything.
int f64_stream_launch(const GemmArgs &g, cudaStream_t s)
{
    if (g.M > 64 || g.N > 64 || g.K > 64 || g.a_layout != KAMI_A_ROW_MK || g.b_layout != KAMI_B_REF_NK ||
        g.out_type != KAMI_F64 || g.batch > 0x7fffffff)
        return KAMI_ERR_UNSUPPORTED;
    // all eight compute warps hold live rows and columns, and a problem
    // carries enough bytes to be worth a stage (32^3 x 1024 measured 18 us
    // here against 12 us one CTA per problem)
    if (g.M <= 48 || g.N <= 32 || g.K < 32)
        return KAMI_ERR_UNSUPPORTED;
    auto ok = [](const void *p, int64_t ld, int64_t st) {
        return !(reinterpret_cast<uintptr_t>(p) & 15) && !(ld & 1) && !(st & 1);
    };
    if (!ok(g.A, g.lda, g.sA) || !ok(g.B, g.ldb, g.sB) || (g.batch > 1 && (g.sA == 0 || g.sB == 0)))
        return KAMI_ERR_UNSUPPORTED;
    F64sParams fp{};
    if (!make_map_f64(&fp.mapA, g.A, g.K, g.M, g.batch, g.lda, g.sA) ||
        !make_map_f64(&fp.mapB, g.B, g.K, g.N, g.batch, g.ldb, g.sB))
        return KAMI_ERR_UNSUPPORTED;
    fp.g = g;
    fp.kboxes = (g.K + 7) / 8;
    fp.timeout_ns = (uint64_t)(5e8 + (double)g.num_iter * 1e6); // generous: a problem takes microseconds
    const void *fn = g.K == 64 ? (const void *)&f64_stream_kernel<true> : (const void *)&f64_stream_kernel<false>;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    static std::once_flag once[2];
    static cudaError_t attr_err[2];
    const int which = g.K == 64 ? 1 : 0;
    std::call_once(once[which], [&] {
        attr_err[which] = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    });
    cudaError_t e = attr_err[which];
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(f64_stream_kernel)");
    const int64_t grid = g.batch < sms ? g.batch : sms;
    void *args[] = {&fp};
    e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kThreads), args, kSmem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(f64_stream_kernel)");
    return KAMI_OK;
}

int f64s_read_error(int *flag)
{
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(flag, g_f64s_error, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyFromSymbol(g_f64s_error)");
    e = cudaMemcpyToSymbol(g_f64s_error, &zero, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyToSymbol(g_f64s_error)");
    return KAMI_OK;
}

} // namespace kami
