// kami_abi.cu -- the C ABI of libkami_b200.so: argument validation, kernel
// selection (the reference's compile-time -D knobs become run-time
// arguments), launch configuration and error reporting.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "kami_common.cuh"
#include "mma_engine.cuh"
#include "tc05_gemm.cuh"

namespace kami {

int f64_stream_launch(const GemmArgs &g, cudaStream_t s);
int f64s_read_error(int *flag);
int grouped_tc05_read_error(int *flag);
int spgemm_read_error(int *flag);
int grouped_f64s_read_error(int *flag);
int spmm_tc05_read_error(int *flag);
int spgemm_tc05_read_error(int *flag);
int split_read_error(int *flag);
int grouped_fallback(const GemmArgs &g, int in_type, cudaStream_t stream);

static thread_local char g_err[512] = "no error";

int fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(KAMI_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

static int elem_size(int t)
{
    switch (t)
    {
    case KAMI_F16:
    case KAMI_BF16:
        return 2;
    case KAMI_F32:
        return 4;
    case KAMI_F64:
        return 8;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// mma.sync instance selection
// ---------------------------------------------------------------------------
static const MmaInstance *instances(int in_type, int *count)
{
    switch (in_type)
    {
    case KAMI_F16:
        return mma_instances_f16(count);
    case KAMI_BF16:
        return mma_instances_bf16(count);
    case KAMI_F64:
        return mma_instances_f64(count);
    }
    *count = 0;
    return nullptr;
}

// Smallest compiled instance that covers (M, N, K) with the requested
// partition and P (0 = any).  Ties go to more warps (up to 16), which hides
// more MMA latency per SM.
static const MmaInstance *select_mma(int in_type, int part, int P, int M, int N, int K)
{
    int n = 0;
    const MmaInstance *t = instances(in_type, &n);
    const MmaInstance *best = nullptr;
    double best_cost = 0;
    for (int i = 0; i < n; ++i)
    {
        const MmaInstance &c = t[i];
        if (part != KAMI_PARTITION_AUTO && c.part != part)
            continue;
        if (P > 0 && c.P != P)
            continue;
        if (c.BM < M || c.BN < N || c.BK < K)
            continue;
        double cost = (double)c.BM * c.BN * c.BK;
        int w = c.nwarps > 16 ? 32 - c.nwarps : c.nwarps;
        cost -= w * 1e-3;
        // equal tiles: the 1D mapping (no exchange of C slices) measured
        // fastest for FP64, streamed and repeated (64^3: 0.26 ms vs 0.34 ms
        // for 2D); for 16-bit inputs it only breaks ties of warp count
        if (c.part == KAMI_PARTITION_1D)
            cost -= in_type == KAMI_F64 ? 0.5 : 0.5e-3; // FP64: before any warp count
        if (!best || cost < best_cost)
        {
            best = &c;
            best_cost = cost;
        }
    }
    return best;
}

struct FnCache
{
    const void *fn;
    int dev;
    int max_threads;
    int smem_set;
};
static std::mutex g_cache_mu;
static FnCache g_cache[256];
static int g_cache_n = 0;

// Per-device: raise the kernel's dynamic shared-memory limit once and read
// its register-limited maximum block size.
static int prepare_fn(const void *fn, size_t smem, int *max_threads)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (int i = 0; i < g_cache_n; ++i)
        if (g_cache[i].fn == fn && g_cache[i].dev == dev && (size_t)g_cache[i].smem_set >= smem)
        {
            *max_threads = g_cache[i].max_threads;
            return KAMI_OK;
        }
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncGetAttributes");
    int set = (int)smem;
    if (smem > 48 * 1024)
    {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(MaxDynamicSharedMemorySize)");
    }
    if (g_cache_n < 256)
        g_cache[g_cache_n++] = FnCache{fn, dev, fa.maxThreadsPerBlock, set};
    *max_threads = fa.maxThreadsPerBlock;
    return KAMI_OK;
}

static constexpr size_t kMaxSmem = 227 * 1024;

// Resolve a request to an mma.sync launch.  fills info; returns status.
static int plan_mma(int in_type, int part, int P, int alloc_warps, int M, int N, int K, int64_t batch,
                    const MmaInstance **inst_out, LaunchInfo *info, bool query_device)
{
    const int kstep = in_type == KAMI_F64 ? 8 : 16;
    const int kpad = (K + kstep - 1) / kstep * kstep;
    const MmaInstance *inst = select_mma(in_type, part, P, M, N, kpad);
    if (!inst)
        return fail(KAMI_ERR_UNSUPPORTED,
                    "no mma.sync block-GEMM instance for in_type=%d partition=%d P=%d M=%d N=%d K=%d", in_type, part,
                    P, M, N, K);
    int max_threads = 1024;
    if (query_device)
    {
        int st = prepare_fn(inst->fn, 0, &max_threads);
        if (st)
            return st;
    }
    int Q = 1;
    if (alloc_warps > 0)
    {
        if (alloc_warps < inst->nwarps)
            return fail(KAMI_ERR_INVALID_VALUE, "alloc_warps=%d is below the %d warps the partition needs",
                        alloc_warps, inst->nwarps);
    }
    else
    {
        // at least 4 warps per CTA when problems are tiny
        while (Q * inst->nwarps < 4 && (Q + 1) <= 15 && (size_t)(Q + 1) * inst->smem_per_group <= kMaxSmem &&
               (Q + 1) * inst->nwarps * 32 <= max_threads && (Q + 1) <= batch)
            ++Q;
    }
    const int warps = alloc_warps > 0 ? alloc_warps : Q * inst->nwarps;
    if (warps * 32 > max_threads)
        return fail(KAMI_ERR_UNSUPPORTED, "%d threads per CTA exceed this kernel's register-limited maximum %d",
                    warps * 32, max_threads);
    *inst_out = inst;
    info->variant = KAMI_VARIANT_MMA_SYNC;
    info->partition = inst->part;
    info->P = inst->P;
    info->threads = warps * 32;
    info->smem = (int)((size_t)Q * inst->smem_per_group);
    info->problems_per_cta = Q;
    info->grid = (batch + Q - 1) / Q;
    return KAMI_OK;
}

static int check_request(int in_type, int out_type, int M, int N, int K, int64_t batch, int a_layout, int b_layout,
                         int num_iter)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16 && in_type != KAMI_F64)
        return fail(KAMI_ERR_INVALID_VALUE, "in_type %d is not KAMI_F16, KAMI_BF16 or KAMI_F64", in_type);
    if (in_type == KAMI_F64 && out_type != KAMI_F64)
        return fail(KAMI_ERR_UNSUPPORTED, "FP64 inputs need out_type KAMI_F64");
    if (in_type != KAMI_F64 && out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "16-bit inputs need out_type KAMI_F32, KAMI_F16 or KAMI_BF16");
    if (M < 1 || N < 1 || K < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "M, N, K must be positive (got %d, %d, %d)", M, N, K);
    if (batch < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "batch must be >= 0");
    if (num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "num_iter must be >= 1");
    if (a_layout != KAMI_A_ROW_MK && a_layout != KAMI_A_COL_MK)
        return fail(KAMI_ERR_INVALID_VALUE, "bad a_layout %d", a_layout);
    if (b_layout != KAMI_B_REF_NK && b_layout != KAMI_B_ROW_KN)
        return fail(KAMI_ERR_INVALID_VALUE, "bad b_layout %d", b_layout);
    const int kq = in_type == KAMI_F64 ? 2 : 4;
    if (K % kq)
        return fail(KAMI_ERR_UNSUPPORTED, "K=%d must be a multiple of %d for this precision", K, kq);
    return KAMI_OK;
}

static bool aligned(const void *p, int64_t ld, int64_t s, int vec_elems, int esz)
{
    return ((uintptr_t)p % (uintptr_t)(vec_elems * esz)) == 0 && ld % vec_elems == 0 && s % vec_elems == 0;
}

} // namespace kami

using namespace kami;

extern "C" {

const char *kami_last_error_string(void) { return g_err; }

int kami_version(void) { return 100; }

int kami_selftest_bounded_wait(uint64_t timeout_ns, void *stream)
{
    if (timeout_ns > 10000000000ull)
        return fail(KAMI_ERR_INVALID_VALUE, "self-test timeout above 10 s");
    return tc05_selftest_bounded_wait(timeout_ns, reinterpret_cast<cudaStream_t>(stream));
}

int kami_device_status(int *code)
{
    if (!code)
        return fail(KAMI_ERR_INVALID_VALUE, "code is NULL");
    int st = tc05_read_error(code);
    if (st)
        return st;
    int c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0, c7 = 0;
    if ((st = split_read_error(&c2)))
        return st;
    if ((st = f64s_read_error(&c3)))
        return st;
    if ((st = grouped_tc05_read_error(&c4)))
        return st;
    if ((st = spgemm_read_error(&c5)))
        return st;
    if ((st = grouped_f64s_read_error(&c6)))
        return st;
    if ((st = spmm_tc05_read_error(&c7)))
        return st;
    int c8 = 0;
    if ((st = spgemm_tc05_read_error(&c8)))
        return st;
    if (!*code)
        *code = c2;
    if (!*code)
        *code = c3;
    if (!*code)
        *code = c4;
    if (!*code)
        *code = c5;
    if (!*code)
        *code = c6;
    if (!*code)
        *code = c7;
    if (!*code)
        *code = c8;
    if (*code)
        return fail(KAMI_ERR_TIMEOUT, "a bounded device wait gave up (code %d)", *code);
    return KAMI_OK;
}

int kami_gemm_workspace_size(kami_dtype_t in_type, kami_partition_t partition, kami_variant_t variant, int M, int N,
                             int K, int P, int64_t batch, size_t *bytes)
{
    if (!bytes)
        return fail(KAMI_ERR_INVALID_VALUE, "bytes is NULL");
    *bytes = 0;
    return KAMI_OK;
}

int kami_gemm_backward_batched(kami_dtype_t in_type, kami_dtype_t out_type, int M, int N, int K, int64_t batch,
                               const void *A, const void *B, const void *dC, void *dA, void *dB, void *stream)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16 && in_type != KAMI_F64)
        return fail(KAMI_ERR_INVALID_VALUE, "backward: in_type must be KAMI_F16, KAMI_BF16 or KAMI_F64");
    if ((in_type == KAMI_F64) != (out_type == KAMI_F64) ||
        (in_type != KAMI_F64 && out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16))
        return fail(KAMI_ERR_UNSUPPORTED, "backward: output type does not match the input type");
    if (M < 1 || N < 1 || K < 1 || batch < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "backward: M, N, K must be positive and batch >= 0");
    if (!A || !B || !dC)
        return fail(KAMI_ERR_INVALID_VALUE, "backward: A, B and dC must be non-null device pointers");
    if ((!dA && !dB) || batch == 0)
        return KAMI_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int st = tc05_backward_launch(in_type, out_type, M, N, K, batch, A, B, dC, dA, dB, s);
    if (st != KAMI_ERR_UNSUPPORTED)
        return st;
    // two products on the forward kernels: dA = dC (M x N) times B read as the
    // reference's N x K operand (B is K x N row-major); dB = A read transposed
    // (col_mk) times dC as the K x N operand
    if (dA && (st = kami_gemm_batched(in_type, out_type, KAMI_PARTITION_AUTO, KAMI_VARIANT_AUTO, M, K, N, 0, 0, batch,
                                      dC, N, (int64_t)M * N, KAMI_A_ROW_MK, B, N, (int64_t)K * N, KAMI_B_REF_NK, dA, K,
                                      (int64_t)M * K, 1.0, 0.0, 1, nullptr, 0, stream)))
        return st;
    if (dB && (st = kami_gemm_batched(in_type, out_type, KAMI_PARTITION_AUTO, KAMI_VARIANT_AUTO, K, N, M, 0, 0, batch,
                                      A, K, (int64_t)M * K, KAMI_A_COL_MK, dC, N, (int64_t)M * N, KAMI_B_ROW_KN, dB, N,
                                      (int64_t)K * N, 1.0, 0.0, 1, nullptr, 0, stream)))
        return st;
    return KAMI_OK;
}

int kami_gemm_describe(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition,
                       kami_variant_t variant, int M, int N, int K, int P, int alloc_warps, int64_t batch,
                       kami_a_layout_t a_layout, kami_b_layout_t b_layout, int out[8])
{
    int st = check_request(in_type, out_type, M, N, K, batch, a_layout, b_layout, 1);
    if (st)
        return st;
    LaunchInfo info{};
    if (variant == KAMI_VARIANT_TCGEN05 || variant == KAMI_VARIANT_TCGEN05_TS ||
        (variant == KAMI_VARIANT_AUTO && tc05_prefer(in_type, partition, M, N, K, a_layout, b_layout)))
    {
        const int ts = variant == KAMI_VARIANT_TCGEN05_TS ||
                       (variant == KAMI_VARIANT_AUTO && tc05_prefer_ts(M, a_layout));
        st = tc05_plan(in_type, out_type, partition, P, M, N, K, batch, a_layout, b_layout, &info, ts);
        if (st && variant != KAMI_VARIANT_AUTO)
            return st;
    }
    if (info.variant != KAMI_VARIANT_TCGEN05 && info.variant != KAMI_VARIANT_TCGEN05_TS)
    {
        const MmaInstance *inst = nullptr;
        st = plan_mma(in_type, partition, P, alloc_warps, M, N, K, batch, &inst, &info, false);
        if (st)
            return st;
    }
    out[0] = info.variant;
    out[1] = info.partition;
    out[2] = info.P;
    out[3] = info.threads;
    out[4] = info.smem;
    out[5] = info.problems_per_cta;
    out[6] = (int)(info.grid > 0x7fffffff ? 0x7fffffff : info.grid);
    out[7] = 0;
    return KAMI_OK;
}

} // extern "C"

namespace kami {

// kami_gemm_batched with launch hints for callers inside the library.
// one_per_sm: at most one CTA of the repeated-products kernel per SM -- for
// the host pipeline, whose chunks run as concurrent launches: with one CTA
// per SM the SMs free up in the order they started, so each SM runs its
// problems back to back and the last results are spread over time like the
// first inputs were.
int gemm_batched_hinted(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition,
                        kami_variant_t variant, int M, int N, int K, int P, int alloc_warps, int64_t batch,
                        const void *A, int64_t lda, int64_t strideA, kami_a_layout_t a_layout, const void *B,
                        int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, void *C, int64_t ldc,
                        int64_t strideC, double alpha, double beta, int num_iter, void *workspace, size_t ws_bytes,
                        void *stream, int one_per_sm)
{
    int st = check_request(in_type, out_type, M, N, K, batch, a_layout, b_layout, num_iter);
    if (st)
        return st;
    if (batch == 0)
        return KAMI_OK;
    if (!A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "A, B and C must be non-null device pointers");
    if (variant != KAMI_VARIANT_AUTO && variant != KAMI_VARIANT_MMA_SYNC && variant != KAMI_VARIANT_TCGEN05 &&
        variant != KAMI_VARIANT_TCGEN05_TS)
        return fail(KAMI_ERR_INVALID_VALUE, "bad variant %d", variant);
    if (partition < KAMI_PARTITION_AUTO || partition > KAMI_PARTITION_3D)
        return fail(KAMI_ERR_INVALID_VALUE, "bad partition %d", partition);
    if (P < 0 || alloc_warps < 0 || alloc_warps > 32)
        return fail(KAMI_ERR_INVALID_VALUE, "P must be >= 0 and alloc_warps in [0, 32]");
    const int64_t min_lda = a_layout == KAMI_A_ROW_MK ? K : M;
    const int64_t min_ldb = b_layout == KAMI_B_REF_NK ? K : N;
    if (lda < min_lda || ldb < min_ldb || ldc < N)
        return fail(KAMI_ERR_INVALID_VALUE, "leading dimensions too small (lda=%lld ldb=%lld ldc=%lld)",
                    (long long)lda, (long long)ldb, (long long)ldc);
    if (strideA < 0 || strideB < 0 || strideC < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "negative problem stride");
    const int esz = elem_size(in_type);
    const int vec = in_type == KAMI_F64 ? 2 : 4;
    if (a_layout == KAMI_A_ROW_MK && !aligned(A, lda, strideA, vec, esz))
        return fail(KAMI_ERR_MISALIGNED, "A: pointer must be %d-byte aligned and lda/strideA multiples of %d",
                    vec * esz, vec);
    if (b_layout == KAMI_B_REF_NK && !aligned(B, ldb, strideB, vec, esz))
        return fail(KAMI_ERR_MISALIGNED, "B: pointer must be %d-byte aligned and ldb/strideB multiples of %d",
                    vec * esz, vec);

    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = batch;
    g.A = A;
    g.lda = lda;
    g.sA = strideA;
    g.a_layout = a_layout;
    g.B = B;
    g.ldb = ldb;
    g.sB = strideB;
    g.b_layout = b_layout;
    g.C = C;
    g.ldc = ldc;
    g.sC = strideC;
    g.out_type = out_type;
    const int osz = elem_size(out_type);
    g.c_vec = ((uintptr_t)C % (uintptr_t)(2 * osz)) == 0 && ldc % 2 == 0 && strideC % 2 == 0;
    g.c_vec4 = ((uintptr_t)C % (uintptr_t)(4 * osz)) == 0 && ldc % 4 == 0 && strideC % 4 == 0;
    g.alpha = alpha;
    g.beta = beta;
    g.num_iter = num_iter;
    g.one_per_sm = one_per_sm;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    if (variant == KAMI_VARIANT_TCGEN05 || variant == KAMI_VARIANT_TCGEN05_TS ||
        (variant == KAMI_VARIANT_AUTO && tc05_prefer(in_type, partition, M, N, K, a_layout, b_layout)))
    {
        const int ts = variant == KAMI_VARIANT_TCGEN05_TS ||
                       (variant == KAMI_VARIANT_AUTO && tc05_prefer_ts(M, a_layout));
        st = tc05_launch(g, in_type, partition, P, workspace, ws_bytes, s, ts);
        if (st == KAMI_OK || variant != KAMI_VARIANT_AUTO)
            return st;
    }

    // streamed FP64 problems up to 64^3 (the batched FP64 programs' regime):
    // the persistent kernel that overlaps each problem's loads with the
    // DMMAs of the previous ones, when the choice is left to the library and
    // there are at least two problems per SM (148 SMs)
    if (in_type == KAMI_F64 && variant == KAMI_VARIANT_AUTO && partition == KAMI_PARTITION_AUTO && P == 0 &&
        alloc_warps == 0 && num_iter <= 4 && batch >= 296)
    {
        st = f64_stream_launch(g, s);
        if (st != KAMI_ERR_UNSUPPORTED)
            return st;
    }

    const MmaInstance *inst = nullptr;
    LaunchInfo info{};
    st = plan_mma(in_type, partition, P, alloc_warps, M, N, K, batch, &inst, &info, true);
    if (st == KAMI_ERR_UNSUPPORTED && variant == KAMI_VARIANT_AUTO && partition == KAMI_PARTITION_AUTO && P == 0 &&
        alloc_warps == 0)
    {
        g.problems_per_cta = 1;
        return grouped_fallback(g, in_type, s);
    }
    if (st)
        return st;
    int max_threads = 0;
    st = prepare_fn(inst->fn, (size_t)info.smem, &max_threads);
    if (st)
        return st;
    g.problems_per_cta = info.problems_per_cta;
    void *params[] = {&g};
    for (int64_t done = 0; done < info.grid;)
    {
        // grids above 2^31-1 CTAs are split
        const int64_t chunk = info.grid - done > 0x7fffffff ? 0x7fffffff : info.grid - done;
        GemmArgs gc = g;
        const int64_t first = done * info.problems_per_cta;
        gc.A = reinterpret_cast<const char *>(g.A) + first * g.sA * esz;
        gc.B = reinterpret_cast<const char *>(g.B) + first * g.sB * esz;
        gc.C = reinterpret_cast<char *>(g.C) + first * g.sC * osz;
        gc.batch = g.batch - first;
        params[0] = &gc;
        cudaError_t e = cudaLaunchKernel(inst->fn, dim3((unsigned)chunk), dim3(info.threads), params,
                                         (size_t)info.smem, s);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaLaunchKernel(block_mma_kernel)");
        done += chunk;
    }
    return KAMI_OK;
}

} // namespace kami

extern "C" int kami_gemm_batched(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition,
                                 kami_variant_t variant, int M, int N, int K, int P, int alloc_warps, int64_t batch,
                                 const void *A, int64_t lda, int64_t strideA, kami_a_layout_t a_layout, const void *B,
                                 int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, void *C, int64_t ldc,
                                 int64_t strideC, double alpha, double beta, int num_iter, void *workspace,
                                 size_t ws_bytes, void *stream)
{
    return kami::gemm_batched_hinted(in_type, out_type, partition, variant, M, N, K, P, alloc_warps, batch, A, lda,
                                     strideA, a_layout, B, ldb, strideB, b_layout, C, ldc, strideC, alpha, beta,
                                     num_iter, workspace, ws_bytes, stream, 0);
}
