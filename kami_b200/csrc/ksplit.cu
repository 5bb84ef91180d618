// ksplit.cu -- two forms of the mma.sync block GEMM that the plain launch
// path does not use:
//   * the register / shared-memory K split of the 1D partition (only RK of
//     each rank's k-steps in registers, the rest cached in shared memory,
//     mma_engine.cuh), selectable per request or chosen by measurement --
//     the reference explores it with one compile-time split
//     (src/reg_smem/block_gemm_1d_half_mma.cu:30-46, REG_K_SPLIT_BLOCK);
//   * traced instances that count, per warp, the cycles spent communicating
//     and computing (the reference's src/usage_cycle/ kernels, which print
//     them; here they land in a device buffer).
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "kami_common.cuh"
#include "mma_engine.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

namespace {

using TrF16 = TrH16<false>;
using TrBF16 = TrH16<true>;

struct SplitInst
{
    int in_type, BM, P, part, rk, trace; // square BM^3 tiles; rk -1 = every k-step in registers
    int nwarps;
    size_t smem;
    const void *fn;
};

#define KAMI_KS(TR, IT, BM, P, RK)                                                                               \
    SplitInst                                                                                                    \
    {                                                                                                            \
        IT, BM, P, 1, RK, 0, BlockGeom<TR, BM, BM, BM, P, 1, RK>::NW, BlockGeom<TR, BM, BM, BM, P, 1, RK>::SMEM, \
            (const void *)&block_mma_kernel<TR, BM, BM, BM, P, 1, RK, false>                                     \
    }
#define KAMI_KT(BM, P, PART, RK)                                                                                 \
    SplitInst                                                                                                    \
    {                                                                                                            \
        KAMI_F16, BM, P, PART, RK, 1, BlockGeom<TrF16, BM, BM, BM, P, PART, RK>::NW,                             \
            BlockGeom<TrF16, BM, BM, BM, P, PART, RK>::SMEM,                                                     \
            (const void *)&block_mma_kernel<TrF16, BM, BM, BM, P, PART, RK, true>                                \
    }

// K-split forms (and, for the tuner, the all-register forms of the same
// tiles where those fit the register file: 1D 128^3 with P = 4 does not).
const SplitInst kSplit[] = {
    KAMI_KS(TrF16, KAMI_F16, 128, 4, 0),    KAMI_KS(TrF16, KAMI_F16, 128, 4, 2),
    KAMI_KS(TrF16, KAMI_F16, 128, 4, 4),    KAMI_KS(TrF16, KAMI_F16, 128, 8, 0),
    KAMI_KS(TrF16, KAMI_F16, 128, 8, 4),    KAMI_KS(TrF16, KAMI_F16, 128, 8, -1),
    KAMI_KS(TrF16, KAMI_F16, 64, 2, 0),     KAMI_KS(TrF16, KAMI_F16, 64, 2, 2),
    KAMI_KS(TrF16, KAMI_F16, 64, 2, -1),    KAMI_KS(TrF16, KAMI_F16, 64, 4, 0),
    KAMI_KS(TrF16, KAMI_F16, 64, 4, 2),     KAMI_KS(TrF16, KAMI_F16, 64, 4, -1),
    KAMI_KS(TrBF16, KAMI_BF16, 128, 4, 0),  KAMI_KS(TrBF16, KAMI_BF16, 128, 4, 2),
    KAMI_KS(TrBF16, KAMI_BF16, 128, 4, 4),  KAMI_KS(TrBF16, KAMI_BF16, 128, 8, 0),
    KAMI_KS(TrBF16, KAMI_BF16, 128, 8, 4),  KAMI_KS(TrBF16, KAMI_BF16, 128, 8, -1),
    KAMI_KS(TrBF16, KAMI_BF16, 64, 2, 0),   KAMI_KS(TrBF16, KAMI_BF16, 64, 2, 2),
    KAMI_KS(TrBF16, KAMI_BF16, 64, 2, -1),  KAMI_KS(TrBF16, KAMI_BF16, 64, 4, 0),
    KAMI_KS(TrBF16, KAMI_BF16, 64, 4, 2),   KAMI_KS(TrBF16, KAMI_BF16, 64, 4, -1),
};

// Traced instances (FP16): the partitions of the reference's usage-cycle
// programs at 128^3 and 64^3, and the 1D K split.
const SplitInst kTrace[] = {
    KAMI_KT(128, 8, 1, -1), KAMI_KT(128, 4, 2, -1), KAMI_KT(128, 2, 3, -1), KAMI_KT(64, 2, 1, -1),
    KAMI_KT(64, 4, 1, -1),  KAMI_KT(64, 2, 2, -1),  KAMI_KT(64, 2, 3, -1),  KAMI_KT(128, 4, 1, 4),
    KAMI_KT(128, 4, 1, 0),  KAMI_KT(128, 8, 1, 4),
};

constexpr int kSplitN = (int)(sizeof(kSplit) / sizeof(kSplit[0]));
constexpr int kTraceN = (int)(sizeof(kTrace) / sizeof(kTrace[0]));

// raise the dynamic shared-memory limit of a kernel once per device
int prepare(const SplitInst &in)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, cudaError_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair(in.fn, dev);
    auto it = done.find(key);
    if (it == done.end())
    {
        cudaError_t e = cudaSuccess;
        if (in.smem > 48 * 1024)
            e = cudaFuncSetAttribute(in.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)in.smem);
        it = done.emplace(key, e).first;
    }
    if (it->second != cudaSuccess)
        return cuda_fail(it->second, "cudaFuncSetAttribute(block_mma_kernel)");
    return KAMI_OK;
}

int launch(const SplitInst &in, GemmArgs g, cudaStream_t s)
{
    int st = prepare(in);
    if (st)
        return st;
    g.problems_per_cta = 1;
    void *params[] = {&g};
    cudaError_t e = cudaLaunchKernel(in.fn, dim3((unsigned)g.batch), dim3(in.nwarps * 32), params, in.smem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(block_mma_kernel, K split)");
    return KAMI_OK;
}

// smallest tile BM covering the request among the given instances
int covering_tile(const SplitInst *set, int n, int in_type, int part, int M, int N, int K)
{
    int best = 0;
    for (int i = 0; i < n; ++i)
        if (set[i].in_type == in_type && set[i].part == part && set[i].BM >= M && set[i].BM >= N &&
            set[i].BM >= (K + 15) / 16 * 16 && (best == 0 || set[i].BM < best))
            best = set[i].BM;
    return best;
}

std::mutex g_tune_mu;
std::map<std::vector<int64_t>, int> g_tune; // request -> index into kSplit

} // namespace
} // namespace kami

using namespace kami;

extern "C" {

int kami_gemm_batched_ksplit(kami_dtype_t in_type, kami_dtype_t out_type, int M, int N, int K, int P,
                             int64_t batch, const void *A, int64_t lda, int64_t strideA, const void *B, int64_t ldb,
                             int64_t strideB, void *C, int64_t ldc, int64_t strideC, double alpha, double beta,
                             int num_iter, int reg_k_steps, int *reg_k_used, void *stream)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "K split: FP16 / BF16 inputs only");
    if (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "K split: out_type KAMI_F32, KAMI_F16 or KAMI_BF16");
    if (M < 1 || N < 1 || K < 1 || batch < 0 || batch > 0x7fffffff || num_iter < 1 || P < 0 || reg_k_steps < -1)
        return fail(KAMI_ERR_INVALID_VALUE, "K split: bad M, N, K, batch, num_iter, P or reg_k_steps");
    if (lda < K || ldb < K || ldc < N || strideA < 0 || strideB < 0 || strideC < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "K split: leading dimensions or strides too small");
    if (!A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "K split: null buffer");
    if ((reinterpret_cast<uintptr_t>(A) & 7) || (reinterpret_cast<uintptr_t>(B) & 7) || (lda & 3) || (ldb & 3) ||
        (strideA & 3) || (strideB & 3))
        return fail(KAMI_ERR_MISALIGNED, "K split: A and B 8-byte aligned, lda, ldb and strides multiples of 4");
    const int bm = covering_tile(kSplit, kSplitN, in_type, 1, M, N, K);
    if (!bm)
        return fail(KAMI_ERR_UNSUPPORTED, "K split: no 1D tile covers M=%d N=%d K=%d", M, N, K);
    std::vector<int> cand;
    for (int i = 0; i < kSplitN; ++i)
        if (kSplit[i].in_type == in_type && kSplit[i].BM == bm && (P == 0 || kSplit[i].P == P) &&
            (reg_k_steps < 0 || kSplit[i].rk == reg_k_steps ||
             (kSplit[i].rk == -1 && reg_k_steps == bm / 16)))
            cand.push_back(i);
    if (cand.empty())
        return fail(KAMI_ERR_UNSUPPORTED, "K split: no %d^3 instance with P=%d and %d register k-steps", bm, P,
                    reg_k_steps);
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = batch;
    g.A = A;
    g.lda = lda;
    g.sA = strideA;
    g.a_layout = KAMI_A_ROW_MK;
    g.B = B;
    g.ldb = ldb;
    g.sB = strideB;
    g.b_layout = KAMI_B_REF_NK;
    g.C = C;
    g.ldc = ldc;
    g.sC = strideC;
    g.out_type = out_type;
    const int osz = out_type == KAMI_F32 ? 4 : 2;
    g.c_vec = ((uintptr_t)C % (uintptr_t)(2 * osz)) == 0 && ldc % 2 == 0 && strideC % 2 == 0;
    g.c_vec4 = ((uintptr_t)C % (uintptr_t)(4 * osz)) == 0 && ldc % 4 == 0 && strideC % 4 == 0;
    g.alpha = alpha;
    g.beta = beta;
    g.num_iter = num_iter;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (batch == 0)
        return KAMI_OK;
    int pick = cand[0];
    if (cand.size() > 1)
    {
        // measured choice, cached per request shape: every candidate on the
        // caller's A and B with a scratch C (the caller's C is untouched)
        int dev = 0;
        cudaGetDevice(&dev);
        const int64_t tb = batch < 2048 ? batch : 2048;
        std::vector<int64_t> key = {dev, in_type, out_type, M, N, K, P, tb, num_iter, lda, ldb, strideA, strideB};
        bool have = false;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune.find(key);
            if (it != g_tune.end())
            {
                pick = it->second;
                have = true;
            }
        }
        if (!have)
        {
            void *tC = nullptr;
            cudaError_t e = cudaMalloc(&tC, (size_t)tb * M * N * osz);
            if (e != cudaSuccess)
                return cuda_fail(e, "cudaMalloc(K-split tuning scratch)");
            GemmArgs t = g;
            t.batch = tb;
            t.C = tC;
            t.ldc = N;
            t.sC = (int64_t)M * N;
            t.beta = 0.0;
            t.c_vec = N % 2 == 0;
            t.c_vec4 = N % 4 == 0;
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            float best = 1e30f;
            int st = KAMI_OK;
            for (int c : cand)
            {
                if ((st = launch(kSplit[c], t, s)))
                    break;
                cudaEventRecord(e0, s);
                for (int r = 0; r < 3 && st == KAMI_OK; ++r)
                    st = launch(kSplit[c], t, s);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (st == KAMI_OK && ms < best)
                {
                    best = ms;
                    pick = c;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            cudaFree(tC);
            if (st)
                return st;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune[key] = pick;
        }
    }
    if (reg_k_used)
        *reg_k_used = kSplit[pick].rk < 0 ? kSplit[pick].BM / 16 : kSplit[pick].rk;
    return launch(kSplit[pick], g, s);
}

int kami_gemm_trace(kami_partition_t partition, int M, int N, int K, int P, int reg_k_steps, const void *A,
                    const void *B, void *C, int num_iter, unsigned long long *cycles, int *nwarps, void *stream)
{
    if (partition < KAMI_PARTITION_1D || partition > KAMI_PARTITION_3D)
        return fail(KAMI_ERR_INVALID_VALUE, "trace: partition must be 1D, 2D or 3D");
    if (M < 1 || N < 1 || K < 1 || num_iter < 1 || P < 1 || reg_k_steps < -1)
        return fail(KAMI_ERR_INVALID_VALUE, "trace: bad M, N, K, P, num_iter or reg_k_steps");
    if (!A || !B || !C || !cycles)
        return fail(KAMI_ERR_INVALID_VALUE, "trace: null buffer");
    if ((reinterpret_cast<uintptr_t>(A) & 7) || (reinterpret_cast<uintptr_t>(B) & 7) || (K & 3))
        return fail(KAMI_ERR_MISALIGNED, "trace: A and B 8-byte aligned, K a multiple of 4");
    const int bm = covering_tile(kTrace, kTraceN, KAMI_F16, partition, M, N, K);
    int pick = -1;
    for (int i = 0; i < kTraceN && bm; ++i)
        if (kTrace[i].BM == bm && kTrace[i].part == partition && kTrace[i].P == P &&
            (kTrace[i].rk == reg_k_steps || (kTrace[i].rk == -1 && reg_k_steps == bm / 16)))
            pick = i;
    if (pick < 0)
        return fail(KAMI_ERR_UNSUPPORTED, "trace: no traced instance for partition %d, P=%d, reg_k_steps=%d at %dx%dx%d",
                    partition, P, reg_k_steps, M, N, K);
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = 1;
    g.A = A;
    g.lda = K;
    g.a_layout = KAMI_A_ROW_MK;
    g.B = B;
    g.ldb = K;
    g.b_layout = KAMI_B_REF_NK;
    g.C = C;
    g.ldc = N;
    g.out_type = KAMI_F32;
    g.c_vec = ((uintptr_t)C % 8) == 0 && N % 2 == 0;
    g.c_vec4 = ((uintptr_t)C % 16) == 0 && N % 4 == 0;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.num_iter = num_iter;
    g.trace = cycles;
    if (nwarps)
        *nwarps = kTrace[pick].nwarps;
    return launch(kTrace[pick], g, reinterpret_cast<cudaStream_t>(stream));
}

} // extern "C"
