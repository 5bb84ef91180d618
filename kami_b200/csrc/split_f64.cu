// split_f64.cu -- FP64-accurate batched GEMM on the FP16/BF16 tensor cores
// (tcgen05) by exact operand splitting (an Ozaki-type scheme).
//
// Per problem (one CTA, 128 threads), for C = A * op(B) with M, N, K <= 64:
//   1. scaling: row i of A is scaled by 2^-eA[i] and row j of B (column j of
//      op(B)) by 2^-eB[j], with eA/eB = floor(log2 of the row maximum) + 2
//      (read from the exponent bits), so every scaled value r satisfies
//      |r| < 1/2;
//   2. splitting: each scaled value is rounded to the integer
//      X = round(r * 2^(beta s)) (built from the mantissa bits with one
//      shift) and X is written in balanced base 2^beta, least significant
//      digit first: d = ((X + 2^(beta-1)) mod 2^beta) - 2^(beta-1),
//      X <- (X - d) / 2^beta; the most significant digit d_1 takes what is
//      left.  So a = 2^eA * sum_p d_p 2^(-beta p) + (at most half a unit of
//      2^(eA - beta s)) and every |d_p| <= 2^(beta-1).  The digits are exact
//      binary16 (beta = 9) or bfloat16 (beta = 7) integers, encoded from
//      their leading-one position with integer instructions and written to
//      shared memory in the 128-byte-swizzled K-major layout of the MMA;
//   3. products: digits are stacked in pairs on both sides -- A stack t
//      holds digit 2t+1 in rows 0..63 and 2t+2 in rows 64..127, B pair u
//      digit 2u+1 in rows 0..63 and 2u+2 in rows 64..127 -- so one
//      128 x 128 x 16 MMA multiplies four digit pairs at once.  Stack t times
//      pair u accumulates (FP32, in TMEM) into column block b = t + u, whose
//      four 64 x 64 quadrants then hold the digit products of weight
//      2^(-beta (2b+2)) (top-left), 2^(-beta (2b+3)) (top-right and
//      bottom-left) and 2^(-beta (2b+4)) (bottom-right).  Blocks with
//      2b + 2 > s + 1 are dropped (weight below 2^(-beta (s+2))).  At most
//      4 products share a quadrant and |d| <= 2^(beta-1), so with K <= 64
//      every partial sum is an integer of magnitude <= 4 * 2^(2 beta - 2) *
//      64 <= 2^24 (beta = 9 for FP16 digits, beta = 7 for BF16): the FP32
//      accumulation is exact;
//   4. recombination in FP64: C_ij = 2^(eA_i + eB_j) * sum_b (TL + TR + BL
//      + BR with their weights), smallest weights first.
// FP64 arithmetic is used only in step 4; all products run on the tensor
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
    int64_t batch;
    int64_t lda, sA, ldb, sB, ldc, sC;
    int b_layout;
    int c_vec;    // 1: C rows may be written as 16-byte pairs (aligned base, even ldc and stride)
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


// Digit encoding without conversion instructions.  A balanced digit is
// d = f - 2^(beta-1) with f a field of beta (top digit: beta + 1) bits.  The
// 16-bit pattern OFF + f is the binary16 (bfloat16) number 1280 + f (128 + f),
// exact and linear in f over the whole range (the spacing is 1 there), so one
// packed half-precision subtraction of 1536 (192) turns two patterns into the
// two digits d exactly.
// Slice kinds: binary16 digits (beta = 9), bfloat16 digits (beta = 7),
// int8 digits (beta = 8, exact INT32 accumulation).
enum SliceKind
{
    kSliceF16 = 0,
    kSliceBF16 = 1,
    kSliceI8 = 2
};

template <int SK> struct DigitCode;
template <> struct DigitCode<kSliceF16>
{
    static constexpr int kBeta = 9;
    static constexpr uint32_t kOff = 0x6500u;  // binary16 1280
    static constexpr uint32_t kBias = 0x6600u; // binary16 1536 = 1280 + 2^(beta-1)
    static __device__ __forceinline__ uint32_t sub(uint32_t w)
    {
        const __half2 r = __hsub2(*reinterpret_cast<const __half2 *>(&w), __halves2half2(__ushort_as_half((unsigned short)kBias), __ushort_as_half((unsigned short)kBias)));
        return *reinterpret_cast<const uint32_t *>(&r);
    }
};
template <> struct DigitCode<kSliceBF16>
{
    static constexpr int kBeta = 7;
    static constexpr uint32_t kOff = 0x4300u;  // bfloat16 128
    static constexpr uint32_t kBias = 0x4340u; // bfloat16 192 = 128 + 2^(beta-1)
    static __device__ __forceinline__ uint32_t sub(uint32_t w)
    {
        const __nv_bfloat162 r = __hsub2(*reinterpret_cast<const __nv_bfloat162 *>(&w),
                                         __halves2bfloat162(__ushort_as_bfloat16((unsigned short)kBias), __ushort_as_bfloat16((unsigned short)kBias)));
        return *reinterpret_cast<const uint32_t *>(&r);
    }
};

// sum over k < S of 2^(beta-1) 2^(beta k): adding it to X turns the balanced
// digits of X into the plain base-2^beta fields of the sum
template <int BETA, int S>
__host__ __device__ constexpr uint64_t half_digits()
{
    uint64_t h = 0;
    for (int k = 0; k < S; ++k)
        h += (uint64_t)1 << (BETA * k + BETA - 1);
    return h;
}

// Bits [lo, lo + width) of Y, moved to bit `up` (mask m = 2^width - 1);
// lo and up are compile-time constants after unrolling.
__device__ __forceinline__ uint32_t field_at(uint64_t Y, int lo, uint32_t m, int up)
{
    return lo >= up ? (uint32_t)(Y >> (lo - up)) & (m << up) : (uint32_t)(Y << (up - lo)) & (m << up);
}

// round(x 2^(BS - e)) + H as a uint64 (|x| 2^-e < 1/2, so the rounded value
// is at most 2^(BS-1) in magnitude and the sum is non-negative).  A normal x
// is a 53-bit integer m times 2^(be - 1075); its row exponent satisfies
// e >= be - 1021, so the left shift BS - e + be - 1075 is at most BS - 54 <= 9
// and one rounding right shift of m 2^10 suffices.  Zero, and subnormal x
// (rare; only rows whose maximum is tiny), take a slower exact path.
// round(x 2^(BS - e)) + H as a uint64.  x is an integer m < 2^53 times
// 2^(E - 1075) (E = the biased exponent, 1 for subnormals), so the value is
// m 2^sh with sh = E + BS - e - 1075.  With e = floor(log2 max) + G
// (G = 2 for the 16-bit digits, |x| 2^-e < 1/2 and BS <= 63; G = 3 for the
// int8 digits, |x| 2^-e < 1/4 and BS <= 64), a normal row maximum gives
// e >= E - 1023 + G and sh <= BS - 52 - G <= 9: one rounding (half away from
// zero) right shift of m 2^10 gives the value.  Only rows whose maximum is
// subnormal reach sh > 9, where the value is m 2^sh exactly.  The result
// stays below 2^(BS - G + 1) in magnitude; H makes it non-negative.
template <int BS>
__device__ __forceinline__ uint64_t offset_fixed(double x, int e, uint64_t H)
{
    static_assert(BS <= 64, "fixed-point image must fit in 64 bits");
    const uint64_t u = (uint64_t)__double_as_longlong(x);
    const int be = (int)(u >> 52) & 0x7FF;
    const uint64_t m = (u & 0xFFFFFFFFFFFFFull) | ((uint64_t)(be != 0) << 52);
    const int sh = (be ? be : 1) + BS - e - 1075;
    uint64_t a;
    if (sh <= 9)
    {
        const int rs = 9 - sh < 63 ? 9 - sh : 63;
        a = (((m << 10) >> rs) + 1) >> 1;
    }
    else
        a = m << (sh < 63 ? sh : 63);
    return ((u >> 63) ? (uint64_t)0 - a : a) + H;
}

// Split 32 values of one operand row (this thread's half of K) into S
// balanced base-2^beta digits and write digit p (1 = most significant) to
// tile_row(p).  Eight elements (one 16-byte chunk of each digit tile) at a
// time: Y = round(x 2^(beta S - e)) + H, then digit p is field S - p of Y
// minus 2^(beta-1) (the most significant field keeps its carry bit).
template <int SK, int S, class TileFn>
__device__ __forceinline__ void split_row(const double (&r)[32], int e, int half, TileFn tile_row)
{
    using Code = DigitCode<SK>;
    constexpr int BETA = Code::kBeta, BS = BETA * S;
    constexpr uint64_t H = half_digits<BETA, S>();
    constexpr uint32_t OFF2 = Code::kOff | (Code::kOff << 16);
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        uint64_t Y[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            Y[q] = offset_fixed<BS>(r[8 * c + q], e, H);
#pragma unroll
        for (int k = 0; k < S; ++k)
        {
            // the most significant field keeps its carry bit (f <= 2^beta)
            const uint32_t fm = k == S - 1 ? (2u << BETA) - 1u : (1u << BETA) - 1u;
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 8; q += 2)
                w[q >> 1] = Code::sub(field_at(Y[q], BETA * k, fm, 0) + field_at(Y[q + 1], BETA * k, fm, 16) + OFF2);
            uint8_t *base;
            int row;
            tile_row(S - k, base, row);
            *reinterpret_cast<uint4 *>(base + swz(row, half * 4 + c)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Load one row-half of an operand into r: `row` of A (is_b = false) or row
// `row` of the N x K view of B (column `row` of op(B)), K elements
// [32 half, 32 half + 32), zero outside the problem.  X / ld address the
// operand in global memory or its staged copy in shared memory (same
// layout, row stride ld).  Returns the maximum magnitude over the whole row
// (the two threads of a row are adjacent lanes; one shuffle).
__device__ __forceinline__ double load_row(const SplitParams &p, const double *X, int64_t ld, bool is_b, int row,
                                           int half, double (&r)[32])
{
    const int rows = is_b ? p.N : p.M;
    const bool strided = is_b && p.b_layout != KAMI_B_REF_NK;
    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < 32; i += 2)
    {
        const int k = half * 32 + i;
        double x0 = 0.0, x1 = 0.0;
        if (row < rows)
        {
            if (!strided)
            {
                const int64_t o = row * ld + k;
                if (k + 1 < p.K)
                {
                    const double2 v = *reinterpret_cast<const double2 *>(X + o);
                    x0 = v.x;
                    x1 = v.y;
                }
                else if (k < p.K)
                    x0 = X[o];
            }
            else
            {
                const int64_t o = (int64_t)k * ld + row;
                if (k < p.K)
                    x0 = X[o];
                if (k + 1 < p.K)
                    x1 = X[o + ld];
            }
        }
        r[i] = x0;
        r[i + 1] = x1;
        mx = fmax(mx, fmax(fabs(x0), fabs(x1)));
    }
    return fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
}

// Bytes of four 32-bit words transposed: out[p] = byte p of in[0..3] (in
// byte order).
__device__ __forceinline__ void byte_transpose4(const uint32_t (&in)[4], uint32_t (&out)[4])
{
    const uint32_t a = __byte_perm(in[0], in[1], 0x5140), b = __byte_perm(in[2], in[3], 0x5140);
    const uint32_t c = __byte_perm(in[0], in[1], 0x7362), d = __byte_perm(in[2], in[3], 0x7362);
    out[0] = __byte_perm(a, b, 0x5410);
    out[1] = __byte_perm(a, b, 0x7632);
    out[2] = __byte_perm(c, d, 0x5410);
    out[3] = __byte_perm(c, d, 0x7632);
}

// Int8 digits of 32 values of one row (this thread's half of K): with
// Y = round(x 2^(8S - e)) + H (H = 0x80 in each of the S-1 low bytes), the
// low S bytes of Y ^ H are the S balanced base-256 digits themselves, least
// significant first (low digits in [-128, 127], the top one within +-65).
// Digit p (1 = most significant) is byte S - p; eight values (8 bytes of one
// digit tile row) are transposed and stored at a time.
template <int S, class TileFn>
__device__ __forceinline__ void split_row_i8(const double (&r)[32], int e, int half, TileFn tile_row)
{
    constexpr uint64_t H = half_digits<8, S - 1>();
#pragma unroll
    for (int c8 = 0; c8 < 4; ++c8)
    {
        uint32_t lo[8], hi[8]; // digits 0-3 / 4-7 (from the least significant) of 8 values
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            const uint64_t D = offset_fixed<8 * S>(r[8 * c8 + q], e, H) ^ H;
            lo[q] = (uint32_t)D;
            hi[q] = (uint32_t)(D >> 32);
        }
        uint32_t t0[4], t1[4], u0[4], u1[4];
        byte_transpose4(*reinterpret_cast<const uint32_t(*)[4]>(&lo[0]), t0); // values 0-3, digits 0-3
        byte_transpose4(*reinterpret_cast<const uint32_t(*)[4]>(&lo[4]), t1); // values 4-7, digits 0-3
        if constexpr (S > 4)
        {
            byte_transpose4(*reinterpret_cast<const uint32_t(*)[4]>(&hi[0]), u0);
            byte_transpose4(*reinterpret_cast<const uint32_t(*)[4]>(&hi[4]), u1);
        }
        // K index of the first value: 32 half + 8 c8 -> 16-byte chunk and offset
        const int chunk = half * 2 + (c8 >> 1), off = (c8 & 1) * 8;
#pragma unroll
        for (int k = 0; k < S; ++k)
        {
            const uint32_t w0 = k < 4 ? t0[k & 3] : u0[k & 3], w1 = k < 4 ? t1[k & 3] : u1[k & 3];
            uint8_t *base;
            int row;
            tile_row(S - k, base, row);
            *reinterpret_cast<uint2 *>(base + swz(row, chunk) + off) = make_uint2(w0, w1);
        }
    }
}

// Scale and split one loaded row-half (row maximum mx).  Writes the row's
// exponent (half 0) and its S digits into the digit tiles at `dig` (A: digit
// p in stack (p-1)/2, row ((p-1)%2)*64 + row; B: digit p in tile p-1).
template <int SK, int S>
__device__ __forceinline__ void split_loaded(const double (&r)[32], double mx, int row, int half, uint8_t *dig,
                                             int *exps)
{
    // e = floor(log2 max) + G, so |x| 2^-e < 2^(1-G): G = 2 keeps every
    // 16-bit digit within 2^(beta-1); G = 3 keeps the top int8 digit within
    // +-65.  A zero row gets e = 0 (all digits zero).
    constexpr int G = SK == kSliceI8 ? 3 : 2;
    int e = 0;
    if (mx > 0.0)
    {
        const int be = (int)(((uint64_t)__double_as_longlong(mx) >> 52) & 0x7FF);
        if (be > 0)
            e = be - 1023 + G;
        else
        {
            frexp(mx, &e);
            e += G - 1;
        }
    }
    if (half == 0)
        exps[row] = e;
    // digit d of row `row`: A stack (d-1)/2 holds odd digits in rows 0..63 and
    // even digits in rows 64..127 (8 KB further), B tile d-1 holds digit d;
    // both place digit d at byte (d-1) * 8 KB + 128 row
    auto tile_row = [&](int d, uint8_t *&base, int &rr) {
        base = dig + (d - 1) * kSliceBytes;
        rr = row;
    };
    if constexpr (SK == kSliceI8)
        split_row_i8<S>(r, e, half, tile_row);
    else
        split_row<SK, S>(r, e, half, tile_row);
    if constexpr (S & 1)
    {
        // odd digit count: digit S+1 of the last pair is zero (int8 rows use
        // the first 64 bytes: two 16-byte chunks per row-half)
        uint8_t *base = dig + S * kSliceBytes;
        constexpr int nch = SK == kSliceI8 ? 2 : 4;
#pragma unroll
        for (int c = 0; c < nch; ++c)
            *reinterpret_cast<uint4 *>(base + swz(row, half * nch + c)) = make_uint4(0, 0, 0, 0);
    }
}

template <int SK, int S>
__device__ __forceinline__ void split_operand(const SplitParams &p, const double *X, bool is_b, int row, int half,
                                              uint8_t *dig, int *exps)
{
    double r[32];
    const double mx = load_row(p, X, is_b ? p.ldb : p.lda, is_b, row, half, r);
    split_loaded<SK, S>(r, mx, row, half, dig, exps);
}

// 2^n as a double for n >= -1074 (subnormal below -1022), 0 below
__device__ __forceinline__ double pow2(int n)
{
    if (n >= -1022)
        return __longlong_as_double((long long)(n + 1023) << 52);
    return n >= -1074 ? __longlong_as_double(1ll << (n + 1074)) : 0.0;
}

// v * 2^n for |v| < 2^64 and |n| < 2300.  Exact while the result is normal
// (a power-of-two factor); a result in the subnormal range may be rounded
// twice when n < -1022.
__device__ __forceinline__ double scale2(double v, int n)
{
    if (n >= -1022 && n <= 1023)
        return v * pow2(n);
    const int n1 = n < -1022 ? -1022 : 1023;
    return v * pow2(n1) * pow2(n - n1 > 1023 ? 1023 : n - n1);
}

// Row stride (doubles) of the recombination tile for chunks of W columns:
// W + 2 keeps rows 16-byte aligned and spreads 16-byte accesses of
// consecutive rows over all bank groups.
template <int W>
constexpr int xfer_ld()
{
    return W + 2;
}

// Partial sums of one TMEM lane for output columns j0..j0+W-1: column block
// b holds the left (columns j) and right (columns 64 + j) quadrants; lanes
// 0..63 (top, rows i) carry weights 2b+2 (left) and 2b+3 (right), lanes
// 64..127 (bottom, rows i - 64) 2b+3 and 2b+4, in units of 2^-beta.  Blocks
// are read smallest weight first, 16 columns at a time; the TMEM reads of
// the next 16 columns are in flight while the current ones are converted
// and accumulated.  taddr = lane quadrant + j0.
template <int BMAX, int W, int SK>
__device__ __forceinline__ void gather_chunk(uint32_t taddr, bool top, int beta, double (&acc)[W])
{
    constexpr int H = W / 16, NU = (BMAX + 1) * H; // units of 16 columns
    uint32_t vl[2][16], vr[2][16];
#pragma unroll
    for (int e = 0; e < W; ++e)
        acc[e] = 0.0;
    tc::tmem_ld16(taddr + (uint32_t)BMAX * 128, vl[0]);
    tc::tmem_ld16(taddr + (uint32_t)BMAX * 128 + 64, vr[0]);
#pragma unroll
    for (int u = 0; u < NU; ++u)
    {
        const int b = BMAX - u / H, h = u % H, cur = u & 1;
        tc::tmem_ld_wait();
        tc::tmem_regs_ready(vl[cur]);
        tc::tmem_regs_ready(vr[cur]);
        if (u + 1 < NU)
        {
            const int bn = BMAX - (u + 1) / H, hn = (u + 1) % H;
            tc::tmem_ld16(taddr + (uint32_t)bn * 128 + 16 * hn, vl[cur ^ 1]);
            tc::tmem_ld16(taddr + (uint32_t)bn * 128 + 64 + 16 * hn, vr[cur ^ 1]);
        }
        const int wl = top ? 2 * b + 2 : 2 * b + 3;
        if constexpr (SK == kSliceI8)
        {
            // INT32 quadrants: left * 2^8 + right is exact (|.| < 2^31, at most
            // four products of |d| <= 128 per quadrant and K = 64), converted
            // with the 2^52 + 2^51 bias (integer and FP64 add, no conversion
            // unit) and weighted as the right quadrant
            const double sr = pow2(-beta * (wl + 1));
            constexpr double kBias = 6755399441055744.0; // 2^52 + 2^51
#pragma unroll
            for (int e = 0; e < 16; ++e)
            {
                const int v = (int)(vl[cur][e] << 8) + (int)vr[cur][e];
                const double d = __hiloint2double(0x43380000 + (v >> 31), v) - kBias;
                acc[16 * h + e] = fma(d, sr, acc[16 * h + e]);
            }
        }
        else
        {
            const double sl = pow2(-beta * wl), sr = pow2(-beta * (wl + 1));
#pragma unroll
            for (int e = 0; e < 16; ++e)
                acc[16 * h + e] += (double)__uint_as_float(vr[cur][e]) * sr + (double)__uint_as_float(vl[cur][e]) * sl;
        }
    }
}

// Store the recombined 64 x W chunk j0..j0+W-1 of C.  The 128 calling
// threads (one per TMEM lane L) stage their partial sums of row L % 64 in
// xfer (tile L / 64, 64 x xfer_ld<W>() doubles each, 16-byte stores); then
// every thread finishes two adjacent columns of rows L / (W/2), ... : top +
// bottom partial, times 2^(eA[row] + eB[col]), alpha and beta, stored as one
// 16-byte pair, so a warp writes whole row segments of C.  Barrier 1 over
// the 128 threads orders xfer.
template <int W>
__device__ __forceinline__ void recombine_store(const SplitParams &p, double *Cp, const int *eA, const int *eB,
                                                double *xfer, const double (&part)[W], int L, int j0, bool valid)
{
    constexpr int LD = xfer_ld<W>(), TPR = W / 2, RSTEP = 128 / TPR; // threads per row, rows per pass
    double *mine = xfer + (L >> 6) * (64 * LD) + (L & 63) * LD;
    named_barrier(1, 128); // the previous chunk's stores are done with xfer
#pragma unroll
    for (int e = 0; e < W; e += 2)
        *reinterpret_cast<double2 *>(mine + e) = make_double2(part[e], part[e + 1]);
    named_barrier(1, 128);
    const int c = (L % TPR) * 2, jj = j0 + c;
    if (!valid || jj >= p.N)
        return;
    const bool two = jj + 1 < p.N;
    const int eb0 = eB[jj], eb1 = two ? eB[jj + 1] : 0;
    for (int r = L / TPR; r < p.M; r += RSTEP)
    {
        const double2 tp = *reinterpret_cast<const double2 *>(xfer + r * LD + c);
        const double2 bt = *reinterpret_cast<const double2 *>(xfer + (64 + r) * LD + c);
        const int ea = eA[r];
        double *dst = Cp + (int64_t)r * p.ldc + jj;
        double v0 = p.alpha * scale2(tp.x + bt.x, ea + eb0), v1 = p.alpha * scale2(tp.y + bt.y, ea + eb1);
        if (two && p.c_vec)
        {
            if (p.beta_c != 0.0)
            {
                const double2 o = *reinterpret_cast<const double2 *>(dst);
                v0 += p.beta_c * o.x;
                v1 += p.beta_c * o.y;
            }
            *reinterpret_cast<double2 *>(dst) = make_double2(v0, v1);
        }
        else
        {
            if (p.beta_c != 0.0)
                v0 += p.beta_c * dst[0];
            dst[0] = v0;
            if (two)
            {
                if (p.beta_c != 0.0)
                    v1 += p.beta_c * dst[1];
                dst[1] = v1;
            }
        }
    }
}

// One digit-pair product over K = 64: four kind::f16 MMAs of K = 16 (16-bit
// digits) or two kind::i8 MMAs of K = 32 (int8 digits); each K-step
// advances the descriptors by 32 bytes (2 in their 16-byte units).
template <int SK>
__device__ __forceinline__ void issue_pair(uint32_t col, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t first)
{
    if constexpr (SK == kSliceI8)
    {
        tc::mma_i8_ss(col, ad, bd, idesc, first);
        tc::mma_i8_ss(col, ad + 2, bd + 2, idesc, 1u);
    }
    else
    {
        tc::mma_f16_ss(col, ad, bd, idesc, first);
        tc::mma_f16_ss(col, ad + 2, bd + 2, idesc, 1u);
        tc::mma_f16_ss(col, ad + 4, bd + 4, idesc, 1u);
        tc::mma_f16_ss(col, ad + 6, bd + 6, idesc, 1u);
    }
}

template <int SK, int S>
__global__ void __launch_bounds__(128) split_f64_kernel(const SplitParams p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned base, derived from smem_raw by an offset so that the
    // compiler still knows every derived pointer addresses shared memory
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    constexpr int nstack = (S + 1) / 2;
    uint8_t *sA = smem;                           // nstack x 16 KB (A digit pairs)
    uint8_t *sB = sA + nstack * kStackBytes;      // nstack x 16 KB (B digit pairs)
    int *eA = reinterpret_cast<int *>(sB + nstack * kStackBytes);
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

    // ---- 1 + 2: scale and split A and B (two threads per row, 32 k each) ----
    const int row = t >> 1, half = t & 1;
#pragma unroll 1
    for (int op = 0; op < 2; ++op)
        split_operand<SK, S>(p, op ? B : A, op != 0, row, half, op ? sB : sA, op ? eB : eA);
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
        constexpr int bmax = (S - 1) / 2; // last column block kept
        const uint64_t ad0 = tc::desc_kmajor_sw128(tc::smem_u32(sA));
        const uint64_t bd0 = tc::desc_kmajor_sw128(tc::smem_u32(sB));
        const uint64_t pair16 = kStackBytes >> 4; // descriptor step between digit pairs
        for (int it = 0; it < p.num_iter; ++it)
            for (int st = 0; st < nstack; ++st)
                for (int u = 0; st + u <= bmax && u < nstack; ++u)
                {
                    const uint32_t col = tmem + (uint32_t)(st + u) * 128;
                    const uint64_t ad = ad0 + st * pair16, bd = bd0 + u * pair16;
                    // stack 0 opens every block; later stacks accumulate
                    const uint32_t first = (it == 0 && st == 0) ? 0u : 1u;
                    issue_pair<SK>(col, ad, bd, p.idesc, first);
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
    // bottom halves (rows i - 64); both stage their partial sums in shared
    // memory (the digit tiles are dead once the products are done).
    double *xfer = reinterpret_cast<double *>(smem); // 2 x 64 x xfer_ld<W>() doubles
    const int L = warp * 32 + lane;
    const bool top = L < 64;
    const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
    double *Cp = p.C + prob * p.sC;
    constexpr int bmax = (S - 1) / 2;
    constexpr int W = S >= 3 ? 32 : 16; // the 2-digit form has only 32 KB of dead digit tiles
    for (int j0 = 0; j0 < 64; j0 += W)
    {
        double acc[W];
        if (done)
            gather_chunk<bmax, W, SK>(tmem + lane_addr + j0, top, p.beta, acc);
        else
        {
#pragma unroll
            for (int e = 0; e < W; ++e)
                acc[e] = 0.0;
        }
        recombine_store<W>(p, Cp, eA, eB, xfer, acc, L, j0, done);
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
// Persistent form for the streamed regime (one launch over all problems, one
// CTA per SM, 12 warps), so the phases of consecutive problems overlap:
//   warps 0-7   split: 256 threads, one row-half of A or B each.  With
//               16-byte aligned rows the inputs of problem j are staged in
//               shared memory by bulk copies (TMA engine) that the split
//               warps issued for it while working on problem j-1; once all
//               eight warps have read problem j out of the stage they issue
//               the copies of problem j+1, then write the digits of problem
//               j into buffer j % nbuf once the MMAs of the problem that
//               last used it have completed;
//   warps 8-11  recombination of problem j from TMEM (lane quadrants 0-3).
//               After the last TMEM read of problem j, lane 0 of warp 8
//               issues the MMAs of problem j+1 (its digits complete), then
//               the four warps store the last columns of problem j.
// Row and column exponents live in a ring of four entries apart from the
// digit buffers.  Barriers: sfull (bulk copies, by bytes), dfull[b] (8 split
// warps), dempty[b] and tfull (MMA commits).
// Every mbarrier wait is bounded; each warp group agrees on the outcome of
// its waits with a barrier reduction before acting on it, so a timeout
// ends the whole group together.
// ---------------------------------------------------------------------------
constexpr int kStageLd = 66;                            // staged row stride (doubles): 528 bytes
constexpr int kStageBytes = 2 * 64 * kStageLd * 8;      // A rows, then B rows
constexpr int kExpRing = 4;

// Output columns per recombination chunk of the persistent form: 32, except
// where the 128 KB digit buffer of 7 or 8 digits leaves no room for it.
template <int S>
constexpr int persistent_chunk()
{
    return S <= 6 ? 32 : 16;
}

struct SplitStreamParams
{
    SplitParams p;
    int nbuf;      // digit buffers (1 or 2)
    int buf_bytes; // digits of A and B of one problem
    int staged;    // 1: inputs are staged by bulk copies (16-byte aligned rows)
};

// AND of `pred` over the `n` threads of named barrier `id` (whole warps)
__device__ __forceinline__ bool barrier_and(int id, int n, bool pred)
{
    uint32_t out;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}"
                 : "=r"(out)
                 : "r"((uint32_t)pred), "r"(id), "r"(n)
                 : "memory");
    return out != 0;
}

// Bulk copies of problem `prob`'s A rows (threads 0..63 of the split group)
// and B rows (threads 64..127) into the stage; thread 0 first announces the
// byte count on sfull.
__device__ __forceinline__ void stage_problem(const SplitParams &p, int64_t prob, int tt, uint8_t *stage,
                                              uint64_t *sfull)
{
    const bool refnk = p.b_layout == KAMI_B_REF_NK;
    const uint32_t a_bytes = (uint32_t)p.K * 8, b_bytes = (uint32_t)(refnk ? p.K : p.N) * 8;
    const int b_rows = refnk ? p.N : p.K;
    if (tt == 0)
        tc::mbar_expect_tx(sfull, (uint32_t)p.M * a_bytes + (uint32_t)b_rows * b_bytes);
    if (tt < 64 && tt < p.M)
        tc::bulk_g2s(stage + (size_t)tt * kStageLd * 8, p.A + prob * p.sA + tt * p.lda, a_bytes, sfull);
    else if (tt >= 64 && tt < 128 && tt - 64 < b_rows)
        tc::bulk_g2s(stage + (size_t)tt * kStageLd * 8, p.B + prob * p.sB + (tt - 64) * p.ldb, b_bytes, sfull);
}

template <int SK, int S>
__device__ __forceinline__ void issue_products(const SplitParams &p, uint32_t tmem, uint8_t *buf, uint64_t *dempty,
                                               uint64_t *tfull)
{
    constexpr int nstack = (S + 1) / 2, bmax = (S - 1) / 2;
    const uint64_t pair16 = kStackBytes >> 4;
    const uint64_t ad0 = tc::desc_kmajor_sw128(tc::smem_u32(buf));
    const uint64_t bd0 = tc::desc_kmajor_sw128(tc::smem_u32(buf + nstack * kStackBytes));
    for (int it = 0; it < p.num_iter; ++it)
        for (int st = 0; st < nstack; ++st)
            for (int u = 0; st + u <= bmax && u < nstack; ++u)
            {
                const uint32_t col = tmem + (uint32_t)(st + u) * 128;
                const uint64_t ad = ad0 + st * pair16, bd = bd0 + u * pair16;
                const uint32_t first = (it == 0 && st == 0) ? 0u : 1u;
                issue_pair<SK>(col, ad, bd, p.idesc, first);
            }
    tc::mma_commit(dempty);
    tc::mma_commit(tfull);
}

template <int SK, int S>
__global__ void __launch_bounds__(384, 1) split_f64_persistent(const SplitStreamParams sp)
{
    const SplitParams &p = sp.p;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned base, derived from smem_raw by an offset so that the
    // compiler still knows every derived pointer addresses shared memory
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    constexpr int nstack = (S + 1) / 2;
    uint8_t *stage = smem + (size_t)sp.nbuf * sp.buf_bytes;
    constexpr int W = persistent_chunk<S>();
    double *xfer = reinterpret_cast<double *>(stage + (sp.staged ? kStageBytes : 0)); // 2 x 64 x xfer_ld<W>()
    int *exps = reinterpret_cast<int *>(xfer + 2 * 64 * xfer_ld<W>());               // kExpRing x 128
    uint64_t *dfull = reinterpret_cast<uint64_t *>(exps + kExpRing * 128);
    uint64_t *dempty = dfull + 2;
    uint64_t *tfull = dempty + 2;
    uint64_t *sfull = tfull + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sfull + 1);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int64_t nprob = p.batch;
    const uint64_t limit = p.timeout_ns;
    if (t == 0)
    {
        for (int i = 0; i < 2; ++i)
        {
            tc::mbar_init(&dfull[i], 8);
            tc::mbar_init(&dempty[i], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(sfull, 1);
        tc::fence_mbar_init();
    }
    __syncwarp();
    if (warp == 8)
    {
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < 8)
    {
        // ---- split role (named barrier 2 over its 256 threads) ----
        const bool is_b = t >= 128;
        const int row = (t & 127) >> 1, half = t & 1;
        int issued = 0, consumed = 0; // stage phases started / completed and read
        if (sp.staged && blockIdx.x < nprob)
        {
            if (t < 128)
                stage_problem(p, blockIdx.x, t, stage, sfull);
            issued = 1;
        }
        int j = 0;
        for (int64_t prob = blockIdx.x; prob < nprob; prob += gridDim.x, ++j)
        {
            double r[32], mx;
            if (sp.staged)
            {
                if (!barrier_and(2, 256, tc::mbar_wait_bounded(sfull, j & 1, limit)))
                {
                    atomicExch(&g_split_error, 8);
                    break;
                }
                consumed = j + 1;
                mx = load_row(p, reinterpret_cast<const double *>(stage) + (is_b ? 64 * kStageLd : 0), kStageLd,
                              is_b, row, half, r);
                // all eight warps have read the stage: refill it with the next problem
                named_barrier(2, 256);
                if (prob + gridDim.x < nprob)
                {
                    if (t < 128)
                        stage_problem(p, prob + gridDim.x, t, stage, sfull);
                    issued = j + 2;
                }
            }
            else
                mx = load_row(p, is_b ? p.B + prob * p.sB : p.A + prob * p.sA, is_b ? p.ldb : p.lda, is_b, row,
                              half, r);
            const int b = j % sp.nbuf;
            if (!barrier_and(2, 256,
                             j < sp.nbuf || tc::mbar_wait_bounded(&dempty[b], ((j / sp.nbuf) - 1) & 1, limit)))
            {
                atomicExch(&g_split_error, 5);
                break;
            }
            uint8_t *buf = smem + (size_t)b * sp.buf_bytes;
            int *ex = exps + (j % kExpRing) * 128;
            split_loaded<SK, S>(r, mx, row, half, is_b ? buf + nstack * kStackBytes : buf, is_b ? ex + 64 : ex);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                tc::mbar_arrive(&dfull[b]);
        }
        // no bulk copy may still be landing when the CTA exits (possible only
        // after a failed wait): wait for the phase of the copies not yet read
        if (issued > consumed && !tc::mbar_wait_bounded(sfull, consumed & 1, limit))
            atomicExch(&g_split_error, 9);
    }
    else
    {
        // ---- recombination role: warps 8..11 = TMEM lane quadrants 0..3
        //      (named barrier 1 over its 128 threads); lane 0 of warp 8 also
        //      issues the MMAs ----
        const int quad = warp & 3;
        const int L = quad * 32 + lane;
        const bool top = L < 64;
        const bool issuer = warp == 8 && lane == 0;
        const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
        constexpr int bmax = (S - 1) / 2;
        if (issuer && blockIdx.x < nprob)
        {
            if (tc::mbar_wait_bounded(&dfull[0], 0, limit))
            {
                tc::tc_fence_after();
                issue_products<SK, S>(p, tmem, smem, &dempty[0], tfull);
            }
            else
                atomicExch(&g_split_error, 6);
        }
        __syncwarp();
        int j = 0;
        for (int64_t prob = blockIdx.x; prob < nprob; prob += gridDim.x, ++j)
        {
            if (!barrier_and(1, 128, tc::mbar_wait_bounded(tfull, j & 1, limit)))
            {
                atomicExch(&g_split_error, 7);
                break;
            }
            tc::tc_fence_after();
            const int *eA = exps + (j % kExpRing) * 128;
            const int *eB = eA + 64;
            double *Cp = p.C + prob * p.sC;
            for (int j0 = 0; j0 < 64; j0 += W)
            {
                double acc[W];
                gather_chunk<bmax, W, SK>(tmem + lane_addr + j0, top, p.beta, acc);
                if (j0 == 64 - W)
                {
                    // every TMEM read of problem j is done: start problem j+1
                    tc::tc_fence_before();
                    named_barrier(1, 128);
                    if (issuer && prob + gridDim.x < nprob)
                    {
                        const int jn = j + 1, bn = jn % sp.nbuf;
                        if (tc::mbar_wait_bounded(&dfull[bn], (jn / sp.nbuf) & 1, limit))
                        {
                            tc::tc_fence_after();
                            issue_products<SK, S>(p, tmem, smem + (size_t)bn * sp.buf_bytes, &dempty[bn], tfull);
                        }
                        else
                            atomicExch(&g_split_error, 6); // the next tfull wait then times out for all
                    }
                    __syncwarp();
                }
                recombine_store<W>(p, Cp, eA, eB, xfer, acc, L, j0, true);
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 8)
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

struct SplitFns
{
    const void *per_problem;
    const void *persistent;
};

template <int SK, int S>
SplitFns split_fns()
{
    return {(const void *)&split_f64_kernel<SK, S>, (const void *)&split_f64_persistent<SK, S>};
}

// kernels per (digit kind, digit count): FP16 digits 2..7, BF16 and int8
// digits 2..8
SplitFns split_lookup(int sk, int s)
{
#define KAMI_SPLIT_CASE(K, N) \
    case N: return split_fns<K, N>();
    if (sk == kSliceF16)
        switch (s)
        {
            KAMI_SPLIT_CASE(kSliceF16, 2) KAMI_SPLIT_CASE(kSliceF16, 3) KAMI_SPLIT_CASE(kSliceF16, 4)
            KAMI_SPLIT_CASE(kSliceF16, 5) KAMI_SPLIT_CASE(kSliceF16, 6) KAMI_SPLIT_CASE(kSliceF16, 7)
        default: break;
        }
    else if (sk == kSliceBF16)
        switch (s)
        {
            KAMI_SPLIT_CASE(kSliceBF16, 2) KAMI_SPLIT_CASE(kSliceBF16, 3) KAMI_SPLIT_CASE(kSliceBF16, 4)
            KAMI_SPLIT_CASE(kSliceBF16, 5) KAMI_SPLIT_CASE(kSliceBF16, 6) KAMI_SPLIT_CASE(kSliceBF16, 7)
            KAMI_SPLIT_CASE(kSliceBF16, 8)
        default: break;
        }
    else
        switch (s)
        {
            KAMI_SPLIT_CASE(kSliceI8, 2) KAMI_SPLIT_CASE(kSliceI8, 3) KAMI_SPLIT_CASE(kSliceI8, 4)
            KAMI_SPLIT_CASE(kSliceI8, 5) KAMI_SPLIT_CASE(kSliceI8, 6) KAMI_SPLIT_CASE(kSliceI8, 7)
            KAMI_SPLIT_CASE(kSliceI8, 8)
        default: break;
        }
#undef KAMI_SPLIT_CASE
    return {nullptr, nullptr};
}

// raise the dynamic shared memory limit of one kernel, once per process
cudaError_t allow_smem(const void *fn, int sk, int s, int which)
{
    static std::once_flag once[3][9][2];
    static cudaError_t err[3][9][2];
    std::call_once(once[sk][s][which], [&] {
        err[sk][s][which] = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    return err[sk][s][which];
}

size_t split_smem(int s) { return (size_t)((s + 1) / 2) * 2 * kStackBytes + 1024 + 1024; }

} // namespace
} // namespace kami

using namespace kami;

extern "C" int kami_split_f64_gemm_batched(int nslices, kami_dtype_t slice_type, int M, int N, int K, int64_t batch,
                                           const double *A, int64_t lda, int64_t strideA, const double *B,
                                           int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, double *C,
                                           int64_t ldc, int64_t strideC, double alpha, double beta, int num_iter,
                                           void *stream)
{
    if (slice_type != KAMI_F16 && slice_type != KAMI_BF16 && slice_type != KAMI_S8)
        return fail(KAMI_ERR_INVALID_VALUE, "split-FP64: slice_type must be KAMI_F16, KAMI_BF16 or KAMI_S8");
    const int sk = slice_type == KAMI_F16 ? kSliceF16 : (slice_type == KAMI_BF16 ? kSliceBF16 : kSliceI8);
    const int smax = sk == kSliceF16 ? 7 : 8;
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
    p.batch = batch;
    p.lda = lda;
    p.sA = strideA;
    p.ldb = ldb;
    p.sB = strideB;
    p.ldc = ldc;
    p.sC = strideC;
    p.b_layout = b_layout;
    p.c_vec = !(reinterpret_cast<uintptr_t>(C) & 15) && !(ldc & 1) && !(strideC & 1);
    p.s = nslices;
    p.beta = sk == kSliceF16 ? 9 : (sk == kSliceBF16 ? 7 : 8);
    p.alpha = alpha;
    p.beta_c = beta;
    p.num_iter = num_iter;
    p.idesc = sk == kSliceI8 ? tc::idesc_i8(128, 128) : tc::idesc_f16(sk == kSliceBF16, 128, 128);
    uint32_t cols = 32;
    while ((int)cols < ((nslices - 1) / 2 + 1) * 128)
        cols <<= 1;
    p.tmem_cols = cols;
    p.timeout_ns = (uint64_t)(5e8 + (double)num_iter * nslices * nslices * 4 * 2000.0);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const SplitFns fns = split_lookup(sk, nslices);
    if (!fns.per_problem)
        return fail(KAMI_ERR_UNSUPPORTED, "split-FP64: no kernel for %d slices", nslices);
    // persistent form: streamed products, and repeated products whenever the
    // per-problem form would hold one CTA per SM (four digit stacks: 7-8
    // digits) or the digits are int8 -- its warp groups then overlap the
    // splitting and recombination of neighbouring problems with the MMAs
    // (repeated 20x at 64^3: 8 int8 digits 1.20 ms vs 1.47 ms per problem CTA;
    // 6 FP16 digits stay per problem: 1.36 ms vs 1.44 ms)
    const int nstack_sel = (nslices + 1) / 2;
    if (num_iter <= 4 || nstack_sel >= 4 || sk == kSliceI8)
    {
        // streamed regime: the persistent, phase-overlapped form
        SplitStreamParams sp{};
        sp.p = p;
        const int nstack = (nslices + 1) / 2;
        sp.buf_bytes = 2 * nstack * kStackBytes;
        // bulk copies need 16-byte aligned rows whose length is a multiple of 16 bytes
        const bool a_ok = !(reinterpret_cast<uintptr_t>(A) & 15) && !(lda & 1) && !(strideA & 1) && !(K & 1);
        const bool b_ok = !(reinterpret_cast<uintptr_t>(B) & 15) && !(ldb & 1) && !(strideB & 1) &&
                          !((b_layout == KAMI_B_REF_NK ? K : N) & 1);
        sp.staged = a_ok && b_ok ? 1 : 0;
        const int xld = (nslices <= 6 ? 32 : 16) + 2; // xfer_ld<persistent_chunk<S>()>()
        const size_t fixed = (size_t)2 * 64 * xld * 8 + kExpRing * 128 * 4 + 128 + 1024 +
                             (sp.staged ? kStageBytes : 0);
        sp.nbuf = (size_t)2 * sp.buf_bytes + fixed <= 227 * 1024 ? 2 : 1;
        const size_t smem = (size_t)sp.nbuf * sp.buf_bytes + fixed;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const void *fn = fns.persistent;
        cudaError_t e2 = allow_smem(fn, sk, nslices, 1);
        if (e2 != cudaSuccess)
            return cuda_fail(e2, "cudaFuncSetAttribute(split_f64_persistent)");
        const int64_t grid = batch < sms ? batch : sms;
        void *args2[] = {&sp};
        e2 = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(384), args2, smem, st);
        if (e2 != cudaSuccess)
            return cuda_fail(e2, "cudaLaunchKernel(split_f64_persistent)");
        return KAMI_OK;
    }
    const size_t smem = split_smem(nslices);
    const void *fn = fns.per_problem;
    cudaError_t e = allow_smem(fn, sk, nslices, 0);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(split_f64_kernel)");
    void *args[] = {&p};
    e = cudaLaunchKernel(fn, dim3((unsigned)batch), dim3(128), args, smem, st);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(split_f64_kernel)");
    return KAMI_OK;
}
