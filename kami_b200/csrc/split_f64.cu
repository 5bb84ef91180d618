// split_f64.cu -- FP64-accurate batched GEMM on the FP16/BF16 tensor cores
// (tcgen05) by exact operand splitting (an Ozaki-type scheme).
//
// Per problem (one CTA, 128 threads), for C = A * op(B) with M, N, K <= 64:
//   1. scaling: row i of A is scaled by 2^-eA[i] and row j of B (column j of
//      op(B)) by 2^-eB[j], with eA/eB the binary exponents of the row
//      maxima (frexp), so every scaled value r0 satisfies |r0| < 1;
//   2. splitting: s integer digits per element, d_p = rint(r * 2^beta),
//      r <- r * 2^beta - d_p (both steps exact in FP64), so that
//      a = 2^eA * sum_p d_p 2^(-beta p) + (a remainder below 2^(-beta s));
//      |d_1| <= 2^beta and |d_p| <= 2^(beta-1) for p >= 2.  Digits are exact
//      binary16 (beta = 9) or bfloat16 (beta = 7) integers, written to
//      shared memory in the 128-byte-swizzled K-major layout of the MMA;
//   3. products: slices of A are stacked in pairs -- stack t holds digit
//      2t+1 in rows 0..63 and digit 2t+2 in rows 64..127 -- so one M = 128
//      MMA multiplies two A digits by one B digit q.  Stack t times digit q
//      is accumulated (FP32, in TMEM) in column block c = 2t+1+q, so the top
//      half of block c collects the digit pairs with p + q = c and the bottom
//      half those with p + q = c + 1.  Products with 2t+1+q > s+1 are
//      dropped (their weight is below 2^(-beta (s+2))).  With at most
//      ceil(s/2) digit pairs per half, |d| <= 2^(beta-1) and K <= 64, every
//      partial sum is an integer of magnitude <= ceil(s/2) * 2^(2 beta - 2) *
//      64 <= 2^24 (beta = 9, s <= 7; beta = 7, s <= 8), so the FP32
//      accumulation is exact;
//   4. recombination in FP64: C_ij = 2^(eA_i + eB_j) * sum_c (top_c 2^(-beta c)
//      + bottom_c 2^(-beta (c+1))), smallest weights first.
// FP64 is used only in steps 1, 2 and 4; all products run on the tensor
// cores.  num_iter repeats step 3 on the resident digits (the in-register
// repeat used to measure the block GEMM).
#include <mutex>

#include "kami_common.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device-side status of the split kernel's bounded waits (read and cleared
// by kami_device_status)
__device__ int g_split_error = 0;

namespace {

struct SplitParams
{
    const double *A;
    const double *B;
    double *C;
    int M, N, K;
    int64_t lda, sA, ldb, sB, ldc, sC;
    int b_layout;
    int s;        // digits per element
    int beta;     // bits per digit
    double alpha, beta_c;
    int num_iter;
    uint32_t idesc;
    uint32_t tmem_cols;
    uint64_t timeout_ns;
};

constexpr int kStackBytes = 128 * 128; // 128 rows x 64 K x 2 bytes
constexpr int kSliceBytes = 64 * 128;  // 64 rows x 64 K x 2 bytes

// byte offset of element (row, k) in a K-major tile of 128-byte rows with
// the 128-byte swizzle (16-byte chunk index XOR row % 8)
__device__ __forceinline__ int swz(int row, int chunk) { return row * 128 + ((chunk ^ (row & 7)) << 4); }

template <bool BF16S>
__device__ __forceinline__ uint32_t pack2(double x, double y)
{
    if constexpr (BF16S)
    {
        const uint32_t a = __bfloat16_as_ushort(__double2bfloat16(x));
        const uint32_t b = __bfloat16_as_ushort(__double2bfloat16(y));
        return a | (b << 16);
    }
    else
    {
        const uint32_t a = __half_as_ushort(__double2half(x));
        const uint32_t b = __half_as_ushort(__double2half(y));
        return a | (b << 16);
    }
}

// Split 32 values of one operand row (this thread's half of K) into s
// digits and write digit p to tile_of(p) at row row_of(p).
template <bool BF16S, class TileFn>
__device__ __forceinline__ void split_row(double (&r)[32], int e, int s, int beta, int half, TileFn tile_row)
{
    const double two_beta = (double)(1 << beta);
#pragma unroll
    for (int i = 0; i < 32; ++i)
        r[i] = ldexp(r[i], -e);
    for (int p = 1; p <= s; ++p)
    {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 32; i += 2)
        {
            const double y0 = r[i] * two_beta, y1 = r[i + 1] * two_beta;
            const double d0 = rint(y0), d1 = rint(y1);
            r[i] = y0 - d0;
            r[i + 1] = y1 - d1;
            w[i >> 1] = pack2<BF16S>(d0, d1);
        }
        uint8_t *base;
        int row;
        tile_row(p, base, row);
#pragma unroll
        for (int c = 0; c < 4; ++c)
            *reinterpret_cast<uint4 *>(base + swz(row, half * 4 + c)) =
                make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
    }
}

template <bool BF16S>
__global__ void __launch_bounds__(128) split_f64_kernel(const SplitParams p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int nstack = (p.s + 1) / 2;
    uint8_t *sA = smem;                           // nstack x 16 KB
    uint8_t *sB = sA + nstack * kStackBytes;      // s x 8 KB
    int *eA = reinterpret_cast<int *>(sB + p.s * kSliceBytes);
    int *eB = eA + 64;
    uint64_t *bar = reinterpret_cast<uint64_t *>(eB + 64);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
    int *ok_slot = reinterpret_cast<int *>(tmem_slot + 1);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int64_t prob = blockIdx.x;
    const double *A = p.A + prob * p.sA;
    const double *B = p.B + prob * p.sB;

    if (t == 0)
    {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
        *ok_slot = 1;
    }

    // ---- 1 + 2: scale and split A (two threads per row, 32 k each) ----
    const int row = t >> 1, half = t & 1;
    {
        double r[32];
        double mx = 0.0;
#pragma unroll
        for (int i = 0; i < 32; i += 2)
        {
            const int k = half * 32 + i;
            double x0 = 0.0, x1 = 0.0;
            if (row < p.M)
            {
                if (k + 1 < p.K)
                {
                    const double2 v = *reinterpret_cast<const double2 *>(A + row * p.lda + k);
                    x0 = v.x;
                    x1 = v.y;
                }
                else if (k < p.K)
                    x0 = A[row * p.lda + k];
            }
            r[i] = x0;
            r[i + 1] = x1;
            mx = fmax(mx, fmax(fabs(x0), fabs(x1)));
        }
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
        int e = 0;
        if (mx > 0.0)
            frexp(mx, &e);
        e += 1; // |scaled| < 1/2, so every digit satisfies |d| <= 2^(beta-1)
        if (half == 0)
            eA[row] = e;
        split_row<BF16S>(r, e, p.s, p.beta, half, [&](int d, uint8_t *&base, int &rr) {
            base = sA + ((d - 1) >> 1) * kStackBytes;
            rr = ((d - 1) & 1) * 64 + row;
        });
        if (p.s & 1)
        {
            // odd digit count: the bottom half of the last stack is zero
            uint8_t *base = sA + (nstack - 1) * kStackBytes;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                *reinterpret_cast<uint4 *>(base + swz(64 + row, half * 4 + c)) = make_uint4(0, 0, 0, 0);
        }
    }
    // ---- B: row j of the N x K operand (column j of op(B)) ----
    {
        double r[32];
        double mx = 0.0;
#pragma unroll
        for (int i = 0; i < 32; i += 2)
        {
            const int k = half * 32 + i;
            double x0 = 0.0, x1 = 0.0;
            if (row < p.N)
            {
                if (p.b_layout == KAMI_B_REF_NK)
                {
                    if (k + 1 < p.K)
                    {
                        const double2 v = *reinterpret_cast<const double2 *>(B + row * p.ldb + k);
                        x0 = v.x;
                        x1 = v.y;
                    }
                    else if (k < p.K)
                        x0 = B[row * p.ldb + k];
                }
                else
                {
                    if (k < p.K)
                        x0 = B[(int64_t)k * p.ldb + row];
                    if (k + 1 < p.K)
                        x1 = B[(int64_t)(k + 1) * p.ldb + row];
                }
            }
            r[i] = x0;
            r[i + 1] = x1;
            mx = fmax(mx, fmax(fabs(x0), fabs(x1)));
        }
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
        int e = 0;
        if (mx > 0.0)
            frexp(mx, &e);
        e += 1;
        if (half == 0)
            eB[row] = e;
        split_row<BF16S>(r, e, p.s, p.beta, half, [&](int d, uint8_t *&base, int &rr) {
            base = sB + (d - 1) * kSliceBytes;
            rr = row;
        });
    }
    // make the digit tiles visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    if (warp == 0)
    {
        __syncwarp();
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // ---- 3: products on the tensor core ----
    if (t == 0)
    {
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
        for (int it = 0; it < p.num_iter; ++it)
        {
            uint32_t started = 0;
            for (int st = 0; st < nstack; ++st)
                for (int q = 1; q <= p.s; ++q)
                {
                    const int c = 2 * st + 1 + q;
                    if (c > p.s + 1)
                        continue;
                    const uint32_t col = (uint32_t)(c - 2) * 64;
                    for (int kin = 0; kin < 4; ++kin)
                    {
                        const uint64_t ad = tc::desc_kmajor_sw128(a0 + st * kStackBytes + kin * 32);
                        const uint64_t bd = tc::desc_kmajor_sw128(b0 + (q - 1) * kSliceBytes + kin * 32);
                        const uint32_t acc = (it > 0 || kin > 0 || (started >> c & 1)) ? 1u : 0u;
                        tc::mma_f16_ss(tmem + col, ad, bd, p.idesc, acc);
                    }
                    started |= 1u << c;
                }
        }
        tc::mma_commit(bar);
    }
    __syncwarp();
    const bool done = __all_sync(0xffffffffu, tc::mbar_wait_bounded(bar, 0, p.timeout_ns));
    tc::tc_fence_after();
    if (!done)
        atomicExch(&g_split_error, 3);

    // ---- 4: recombination in FP64, 16 output columns at a time ----
    // lanes 0..63 of TMEM hold the top halves (rows i), lanes 64..127 the
    // bottom halves (rows i - 64); the bottom threads hand their partial sums
    // to the top threads through shared memory (the digit tiles are dead).
    double *xfer = reinterpret_cast<double *>(smem); // 64 x 16 doubles
    const int L = warp * 32 + lane;
    const bool top = L < 64;
    const int i = top ? L : L - 64;
    const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
    const int64_t osz = 8;
    double *Cp = p.C + prob * p.sC;
    for (int j0 = 0; j0 < 64; j0 += 16)
    {
        double S[16];
#pragma unroll
        for (int e = 0; e < 16; ++e)
            S[e] = 0.0;
        if (done)
        {
            for (int c = p.s + 1; c >= 2; --c)
            {
                uint32_t v[16];
                tc::tmem_ld16(tmem + lane_addr + (uint32_t)(c - 2) * 64 + j0, v);
                tc::tmem_ld_wait();
                const int w = top ? c : c + 1;
                const double scale = ldexp(1.0, -p.beta * w);
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    S[e] += (double)__uint_as_float(v[e]) * scale;
            }
        }
        __syncthreads(); // previous chunk's readers are done with xfer
        if (!top)
        {
#pragma unroll
            for (int e = 0; e < 16; ++e)
                xfer[i * 16 + e] = S[e];
        }
        __syncthreads();
        if (top && done && i < p.M)
        {
            const int ea = eA[i];
            for (int e = 0; e < 16; ++e)
            {
                const int j = j0 + e;
                if (j >= p.N)
                    break;
                double v = ldexp(xfer[i * 16 + e] + S[e], ea + eB[j]);
                double *dst = Cp + (int64_t)i * p.ldc + j;
                v = p.alpha * v + (p.beta_c != 0.0 ? p.beta_c * *dst : 0.0);
                *dst = v;
            }
        }
    }
    (void)osz;
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0)
    {
        __syncwarp();
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, p.tmem_cols);
    }
}

} // namespace

int split_read_error(int *flag)
{
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(flag, g_split_error, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyFromSymbol(g_split_error)");
    e = cudaMemcpyToSymbol(g_split_error, &zero, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyToSymbol(g_split_error)");
    return KAMI_OK;
}

namespace {

size_t split_smem(int s) { return (size_t)((s + 1) / 2) * kStackBytes + (size_t)s * kSliceBytes + 1024 + 1024; }

} // namespace
} // namespace kami

using namespace kami;

extern "C" int kami_split_f64_gemm_batched(int nslices, kami_dtype_t slice_type, int M, int N, int K, int64_t batch,
                                           const double *A, int64_t lda, int64_t strideA, const double *B,
                                           int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, double *C,
                                           int64_t ldc, int64_t strideC, double alpha, double beta, int num_iter,
                                           void *stream)
{
    const bool bf = slice_type == KAMI_BF16;
    if (slice_type != KAMI_F16 && slice_type != KAMI_BF16)
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: slice_type must be KAMI_F16 or KAMI_BF16");
    const int smax = bf ? 8 : 7;
    if (nslices < 2 || nslices > smax)
        return fail(KAMI_ERR_UNSUPPORTED, "split-FP64: %d slices; supported 2..%d for this slice type", nslices,
                    smax);
    if (M < 1 || N < 1 || K < 1 || batch < 0 || num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: bad shape or num_iter");
    if (M > 64 || N > 64 || K > 64)
        return fail(KAMI_ERR_UNSUPPORTED, "split-FP64: M, N, K <= 64 (got %d, %d, %d)", M, N, K);
    if (b_layout != KAMI_B_REF_NK && b_layout != KAMI_B_ROW_KN)
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: bad b_layout");
    if (batch == 0)
        return KAMI_OK;
    if (!A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: null pointer");
    if (lda < K || ldc < N || ldb < (b_layout == KAMI_B_REF_NK ? K : N))
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: leading dimension too small");
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (lda & 1) || (strideA & 1) ||
        (b_layout == KAMI_B_REF_NK && ((reinterpret_cast<uintptr_t>(B) & 15) || (ldb & 1) || (strideB & 1))))
        return fail(KAMI_ERR_MISALIGNED, "split-FP64: 16-byte aligned rows required");
    if (batch > 0x7fffffff)
        return fail(KAMI_ERR_UNSUPPORTED, "split-FP64: batch above 2^31-1");

    SplitParams p{};
    p.A = A;
    p.B = B;
    p.C = C;
    p.M = M;
    p.N = N;
    p.K = K;
    p.lda = lda;
    p.sA = strideA;
    p.ldb = ldb;
    p.sB = strideB;
    p.ldc = ldc;
    p.sC = strideC;
    p.b_layout = b_layout;
    p.s = nslices;
    p.beta = bf ? 7 : 9;
    p.alpha = alpha;
    p.beta_c = beta;
    p.num_iter = num_iter;
    p.idesc = tc::idesc_f16(bf, 128, 64);
    uint32_t cols = 32;
    while ((int)cols < nslices * 64)
        cols <<= 1;
    p.tmem_cols = cols;
    p.timeout_ns = (uint64_t)(5e8 + (double)num_iter * nslices * nslices * 4 * 2000.0);
    const size_t smem = split_smem(nslices);
    const void *fn = bf ? (const void *)&split_f64_kernel<true> : (const void *)&split_f64_kernel<false>;
    static std::once_flag once[2];
    cudaError_t e = cudaSuccess;
    std::call_once(once[bf ? 1 : 0],
                   [&] { e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024); });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(split_f64_kernel)");
    void *args[] = {&p};
    e = cudaLaunchKernel(fn, dim3((unsigned)batch), dim3(128), args, smem, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(split_f64_kernel)");
    return KAMI_OK;
}
