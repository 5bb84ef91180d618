// split_f64.cu -- FP64-accurate batched GEMM on the FP16/BF16 tensor cores
// (tcgen05) by exact operand splitting (an Ozaki-type scheme).
//
// Per problem (one CTA, 128 threads), for C = A * op(B) with M, N, K <= 64:
//   1. scaling: row i of A is scaled by 2^-eA[i] and row j of B (column j of
//      op(B)) by 2^-eB[j], with eA/eB = floor(log2 of the row maximum) + 2
//      (read from the exponent bits), so every scaled value r satisfies
//      |r| < 1/2;
//   2. splitting: each scaled value is rounded to the integer
//      X = round(r * 2^(beta s)) (nearest, ties to even: an exact
//      power-of-two scaling and one conversion) and X is written in balanced base 2^beta, least significant
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
#include <cstring>
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

// Power-of-two factors of the fixed-point image: x 2^(BS - e) = (x s.lo) s.hi
// with s.lo = 2^min(BS - e, 1023) and s.hi = 2^(the rest).  Both products are
// exact: they only move the exponent, the result stays below 2^62 (no
// overflow), and a product that lands below the normal range is below 1/2,
// where any rounding of it still converts to 0.  BS - e >= -1010 (the row
// exponent is at most 1026), so only rows whose maximum is below about
// 2^-960 need s.hi != 1.
struct FixedScale
{
    double lo, hi;
};

template <int BS>
__device__ __forceinline__ FixedScale fixed_scale(int e)
{
    const int k = BS - e, k1 = k < 1023 ? k : 1023;
    return {__longlong_as_double((long long)(k1 + 1023) << 52), __longlong_as_double((long long)(k - k1 + 1023) << 52)};
}

// round(x 2^(BS - e)) + H as a uint64: the exact scaled value, rounded to the
// nearest integer (ties to even) by one conversion instruction.  With
// e = floor(log2 max) + G (G = 2 for the 16-bit digits, |x| 2^-e < 1/2 and
// BS <= 63; G = 3 for the int8 digits, |x| 2^-e < 1/4 and BS <= 64) the
// rounded value stays below 2^(BS - G + 1) <= 2^62 in magnitude; H makes it
// non-negative.
__device__ __forceinline__ uint64_t offset_fixed(double x, FixedScale s, uint64_t H)
{
    return (uint64_t)__double2ll_rn((x * s.lo) * s.hi) + H;
}

// Split 32 values of one operand row (this thread's half of K) into S
// balanced base-2^beta digits and write digit p (1 = most significant) to
// tile_row(p).  Values 8c..8c+7 of r belong to K group c ^ gx of the
// row-half (gx = 1 swaps the groups pairwise, as load_row_tiled leaves them).  Eight elements (one 16-byte chunk of each digit tile) at a
// time: Y = round(x 2^(beta S - e)) + H, then digit p is field S - p of Y
// minus 2^(beta-1) (the most significant field keeps its carry bit).
template <int SK, int S, class TileFn>
__device__ __forceinline__ void split_row(const double (&r)[32], int e, int half, int gx, TileFn tile_row)
{
    using Code = DigitCode<SK>;
    constexpr int BETA = Code::kBeta, BS = BETA * S;
    constexpr uint64_t H = half_digits<BETA, S>();
    constexpr uint32_t OFF2 = Code::kOff | (Code::kOff << 16);
    const FixedScale sc = fixed_scale<BS>(e);
#pragma unroll
    for (int c = 0; c < 4; ++c)
    {
        uint64_t Y[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            Y[q] = offset_fixed(r[8 * c + q], sc, H);
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
            *reinterpret_cast<uint4 *>(base + swz(row, half * 4 + (c ^ gx))) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Load one row-half of an operand into r: `row` of A (is_b = false) or row
// `row` of the N x K view of B (column `row` of op(B)), K elements
// [32 half, 32 half + 32), zero outside the problem.  X / ld address the
// operand in global memory (row stride ld).  Returns the maximum magnitude
// over the whole row (the two threads of a row are adjacent lanes; one
// shuffle).
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

// load_row for an operand staged by the tensor copies of the persistent
// form: its 64 x 64 tile as four boxes of 16 k x 64 rows (8 KB, 128-byte
// rows; 16-byte chunk c of row r lies at chunk c ^ (r % 8)).  Rows and k
// outside the problem were zero-filled by the copies, so nothing is checked.
//   !strided: `row` of the operand, k in [32 half, 32 half + 32): 16 double2
//             loads.  Half 1 visits its chunks in the order s ^ 4, so the two
//             threads of a row read different banks; its register pair s then
//             holds chunk s ^ 4, i.e. its groups of 8 values are swapped
//             pairwise (split with gx = half).
//   strided:  B stored K x N (row_kn), boxes of 16 n x 64 k: column `row`
//             of op(B) is a column of the tile, read in k order.
// The maximum is a tree of depth 5, not a chain of 16.
__device__ __forceinline__ double load_row_tiled(const uint8_t *tile, bool strided, int row, int half,
                                                 double (&r)[32])
{
    if (!strided)
    {
        const int x = (row & 7) ^ (4 * half);
        const uint8_t *rb = tile + half * 2 * 8192 + row * 128;
#pragma unroll
        for (int s = 0; s < 16; ++s)
        {
            const double2 v = *reinterpret_cast<const double2 *>(rb + (s >> 3) * 8192 + (((s & 7) ^ x) << 4));
            r[2 * s] = v.x;
            r[2 * s + 1] = v.y;
        }
    }
    else
    {
        const uint8_t *cb = tile + (row >> 4) * 8192 + half * 32 * 128 + (row & 1) * 8;
        const int cn = (row & 15) >> 1;
#pragma unroll
        for (int i = 0; i < 32; ++i)
            r[i] = *reinterpret_cast<const double *>(cb + i * 128 + ((cn ^ (i & 7)) << 4));
    }
    double m[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
        m[i] = fmax(fabs(r[2 * i]), fabs(r[2 * i + 1]));
#pragma unroll
    for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
        for (int i = 0; i < w; ++i)
            m[i] = fmax(m[i], m[i + w]);
    return fmax(m[0], __shfl_xor_sync(0xffffffffu, m[0], 1));
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
// digit tile row, K group c8 ^ gx of the row-half) are transposed and stored
// at a time.
template <int S, class TileFn>
__device__ __forceinline__ void split_row_i8(const double (&r)[32], int e, int half, int gx, TileFn tile_row)
{
    constexpr uint64_t H = half_digits<8, S - 1>();
    const FixedScale sc = fixed_scale<8 * S>(e);
#pragma unroll
    for (int c8 = 0; c8 < 4; ++c8)
    {
        uint32_t lo[8], hi[8]; // digits 0-3 / 4-7 (from the least significant) of 8 values
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            const uint64_t D = offset_fixed(r[8 * c8 + q], sc, H) ^ H;
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
        const int g = c8 ^ gx, chunk = half * 2 + (g >> 1), off = (g & 1) * 8;
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
// p in stack (p-1)/2, row ((p-1)%2)*64 + row; B: digit p in tile p-1); gx as
// for split_row.
template <int SK, int S>
__device__ __forceinline__ void split_loaded(const double (&r)[32], double mx, int row, int half, uint8_t *dig,
                                             int *exps, int gx = 0)
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
        split_row_i8<S>(r, e, half, gx, tile_row);
    else
        split_row<SK, S>(r, e, half, gx, tile_row);
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

// 2^n as a double for -1022 <= n <= 1023 (a normal power of two)
__device__ __forceinline__ double pow2n(int n) { return __longlong_as_double((long long)(n + 1023) << 52); }

// v * 2^n for |v| < 2^64 and |n| < 2300, without branches: v 2^n1 2^n2 with
// n1 = n clamped to the normal exponent range and n2 = the rest clamped the
// same way (a rest below -1022 arises only where the result is below 2^-1980
// and rounds to zero either way).  Exact while the result is normal; a result
// in the subnormal range may be rounded twice when n < -1022.
__device__ __forceinline__ double scale2(double v, int n)
{
    const int n1 = min(max(n, -1022), 1023);
    const int n2 = min(max(n - n1, -1022), 1023);
    return v * pow2n(n1) * pow2n(n2);
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
// CTA per SM), so the phases of consecutive problems overlap.  With P split
// warps (P = 8 or 4, split_warps below):
//   warps 0..P-1     split: one row-half of A or of B per thread (P = 8), or
//                    a row-half of A and then the same row-half of B (P = 4).
//                    With 16-byte aligned rows the inputs of problem j are
//                    staged in shared memory by eight tensor copies (TMA
//                    engine) that thread 0 issued once the split warps had
//                    read problem j-1 out of the stage; they write the digits
//                    of problem j into buffer j % nbuf once the MMAs of the
//                    problem that last used it have completed;
//   warps P..P+7     recombination of problem j from TMEM: warp w reads lane
//                    quadrant w % 4; warps P..P+3 finish output columns 0-31
//                    and warps P+4..P+7 columns 32-63 (two groups of 128
//                    threads, so two warps per scheduler hide each other's
//                    TMEM and FP64 latencies).  After the last TMEM read of
//                    problem j by both groups, lane 0 of warp P issues the
//                    MMAs of problem j+1 (its digits complete), then the
//                    groups store their last columns of problem j.
// Row and column exponents live in a ring of four entries apart from the
// digit buffers.  mbarriers: sfull (tensor copies, by bytes), dfull[b] (the
// P split warps), dempty[b] and tfull (MMA commits).  Named barriers: 2
// (split warps), 1 and 3 (one recombination group each), 4 (both groups).
// Every mbarrier wait is bounded; each warp group agrees on the outcome of
// its waits with a barrier reduction before acting on it, so a timeout
// ends the whole group together.
// ---------------------------------------------------------------------------
constexpr int kBoxBytes = 64 * 128;                     // one tensor-copy box: 16 doubles x 64 rows
constexpr int kStageBytes = 8 * kBoxBytes;              // A's four boxes, then B's
constexpr int kExpRing = 4;
// Split warps of the persistent form: eight (one row-half each, 16 warps of
// at most 128 registers) where the split's registers allow it -- int8 digits
// and up to four 16-bit digits; four (a row-half of A, then one of B; 12
// warps of up to 168 registers) for five to eight 16-bit digits, whose split
// would spill under the lower limit (measured at 64^3 x 8192: 7 int8 digits
// 0.263 vs 0.289 ms, 7 FP16 digits 0.420 vs 0.404 ms).
template <int SK, int S>
constexpr int split_warps()
{
    return SK == kSliceI8 || S <= 4 ? 8 : 4;
}

template <int SK, int S>
constexpr int persistent_threads()
{
    return split_warps<SK, S>() * 32 + 256; // + two recombination groups
}
constexpr int kPersistentW = 16;                        // output columns per recombination chunk
constexpr int kXferBytes = 2 * 64 * kPersistentW * 8;   // two groups' 64 x 16 FP64 tiles

struct SplitStreamParams
{
    SplitParams p;
    int nbuf;      // digit buffers (1 or 2)
    int buf_bytes; // digits of A and B of one problem
    int staged;    // 1: inputs are staged by tensor copies (maps tmA / tmB valid)
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

// Tensor copies of problem `prob` into the stage (one thread): A's 64 x 64
// tile as four boxes of 16 k, then B's (16 k of the N x K view, or 16 n of
// the K x N layout); the copies zero-fill rows and k beyond the problem, so
// every box carries its full 8 KB.
__device__ __forceinline__ void stage_problem(const CUtensorMap *tmA, const CUtensorMap *tmB, int64_t prob,
                                              uint8_t *stage, uint64_t *sfull)
{
    tc::mbar_expect_tx(sfull, kStageBytes);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        tc::tma_load_3d(stage + q * kBoxBytes, tmA, sfull, 16 * q, 0, (int)prob);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        tc::tma_load_3d(stage + (4 + q) * kBoxBytes, tmB, sfull, 16 * q, 0, (int)prob);
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

// 16-byte chunk c (columns 2c, 2c+1) of row r of a recombination group's
// 64 x 16 FP64 tile: 128-byte rows, chunk index XOR r % 8, so eight
// consecutive rows, or the eight chunks of one row, fall in distinct banks.
__device__ __forceinline__ double *tile_chunk(double *tile, int r, int c)
{
    return tile + r * 16 + ((c ^ (r & 7)) << 1);
}

// Finish the 64 x 16 chunk j0..j0+15 of C from the partial sums of one TMEM
// lane L (L < 64: the top partial of row L, L >= 64: the bottom partial of
// row L - 64).  The top thread of row r finishes columns j0..j0+7 and the
// bottom thread columns j0+8..j0+15: each leaves the half that it does not
// finish in the group's tile, adds the other thread's half to its own, scales
// by 2^(eA[r] + eB[col]) and alpha, and puts its eight results back into the
// tile; then the 128 threads copy the tile out row by row (8 threads per
// 128-byte row, beta applied there), so every warp store covers four whole
// row segments of C.  Named barrier `bar` over the group's 128 threads orders
// the tile.
template <int W>
__device__ __forceinline__ void finish_half_chunk(const SplitParams &p, double *Cp, const int *eA, const int *eB,
                                                  double *tile, const double (&part)[W], int L, int j0, int bar)
{
    static_assert(W == 16, "one 128-byte tile row per output row");
    constexpr int HW = W / 2;
    const bool top = L < 64;
    const int r = L & 63;
    const int mine = top ? 0 : 4; // first chunk this thread finishes
    named_barrier(bar, 128);      // the previous chunk's copy-out is done with the tile
#pragma unroll
    for (int c = 0; c < 4; ++c)
        *reinterpret_cast<double2 *>(tile_chunk(tile, r, 4 - mine + c)) =
            top ? make_double2(part[HW + 2 * c], part[HW + 2 * c + 1]) : make_double2(part[2 * c], part[2 * c + 1]);
    named_barrier(bar, 128);
    const int jb = j0 + 2 * mine; // first output column this thread finishes
    const int ea = eA[r];
    // HW exponents (16-byte aligned: jb is a multiple of 8) and the other
    // thread's HW partials
    int eb[HW];
#pragma unroll
    for (int e = 0; e < HW; e += 4)
        *reinterpret_cast<int4 *>(&eb[e]) = *reinterpret_cast<const int4 *>(eB + jb + e);
    double o[HW];
#pragma unroll
    for (int c = 0; c < 4; ++c)
        *reinterpret_cast<double2 *>(&o[2 * c]) = *reinterpret_cast<const double2 *>(tile_chunk(tile, r, mine + c));
    double v[HW];
#pragma unroll
    for (int e = 0; e < HW; ++e)
        v[e] = p.alpha * scale2((top ? part[e] : part[HW + e]) + o[e], ea + eb[e]);
    named_barrier(bar, 128); // every exchange read is done: the tile takes the results
#pragma unroll
    for (int c = 0; c < 4; ++c)
        *reinterpret_cast<double2 *>(tile_chunk(tile, r, mine + c)) = make_double2(v[2 * c], v[2 * c + 1]);
    named_barrier(bar, 128);
    // copy-out: thread L takes chunk L % 8 of rows L / 8, L / 8 + 16, ...
    const int cc = L & 7, col = j0 + 2 * cc;
    if (col >= p.N)
        return;
    const bool two = col + 1 < p.N;
#pragma unroll
    for (int pass = 0; pass < 4; ++pass)
    {
        const int row = (L >> 3) + 16 * pass;
        if (row >= p.M)
            break;
        const double2 val = *reinterpret_cast<const double2 *>(tile_chunk(tile, row, cc));
        double *dst = Cp + (int64_t)row * p.ldc + col;
        double v0 = val.x, v1 = val.y;
        if (two && p.c_vec)
        {
            if (p.beta_c != 0.0)
            {
                const double2 old = *reinterpret_cast<const double2 *>(dst);
                v0 += p.beta_c * old.x;
                v1 += p.beta_c * old.y;
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

template <int SK, int S>
__global__ void __launch_bounds__(persistent_threads<SK, S>(), 1) split_f64_persistent(const SplitStreamParams sp,
                                                               const __grid_constant__ CUtensorMap tmA,
                                                               const __grid_constant__ CUtensorMap tmB)
{
    const SplitParams &p = sp.p;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned base, derived from smem_raw by an offset so that the
    // compiler still knows every derived pointer addresses shared memory
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    constexpr int nstack = (S + 1) / 2;
    constexpr int W = kPersistentW;
    constexpr int kSplitWarps = split_warps<SK, S>();
    constexpr int kSplitThreads = kSplitWarps * 32;
    constexpr int kSplitPasses = 256 / kSplitThreads; // row-halves of A and B per split thread
    uint8_t *stage = smem + (size_t)sp.nbuf * sp.buf_bytes;
    double *xfer = reinterpret_cast<double *>(stage + (sp.staged ? kStageBytes : 0)); // kXferBytes
    int *exps = reinterpret_cast<int *>(xfer + kXferBytes / 8);                        // kExpRing x 128
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
            tc::mbar_init(&dfull[i], kSplitWarps);
            tc::mbar_init(&dempty[i], 1);
        }
        tc::mbar_init(tfull, 1);
        tc::mbar_init(sfull, 1);
        tc::fence_mbar_init();
    }
    __syncwarp();
    if (warp == kSplitWarps)
    {
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < kSplitWarps)
    {
        // ---- split role (named barrier 2 over its kSplitThreads threads) ----
        const int row = (t & 127) >> 1, half = t & 1;
        const bool strided_b = p.b_layout != KAMI_B_REF_NK;
        int issued = 0, consumed = 0; // stage phases started / completed and read
        if (sp.staged && blockIdx.x < nprob)
        {
            if (t == 0)
                stage_problem(&tmA, &tmB, blockIdx.x, stage, sfull);
            issued = 1;
        }
        int j = 0;
        for (int64_t prob = blockIdx.x; prob < nprob; prob += gridDim.x, ++j)
        {
            if (sp.staged)
            {
                if (!barrier_and(2, kSplitThreads, tc::mbar_wait_bounded(sfull, j & 1, limit)))
                {
                    atomicExch(&g_split_error, 8);
                    break;
                }
                consumed = j + 1;
            }
            const int b = j % sp.nbuf;
            uint8_t *buf = smem + (size_t)b * sp.buf_bytes;
            int *ex = exps + (j % kExpRing) * 128;
            bool ok = true;
#pragma unroll 1
            for (int pass = 0; pass < kSplitPasses; ++pass) // row-half of A, then of B
            {
                const bool is_b = kSplitPasses == 2 ? pass == 1 : t >= 128;
                double r[32];
                const bool strided = is_b && strided_b;
                const double mx =
                    sp.staged ? load_row_tiled(stage + (is_b ? 4 * kBoxBytes : 0), strided, row, half, r)
                              : load_row(p, is_b ? p.B + prob * p.sB : p.A + prob * p.sA, is_b ? p.ldb : p.lda, is_b,
                                         row, half, r);
                if (pass == kSplitPasses - 1 && sp.staged)
                {
                    // all split warps have read the stage: refill it with the next problem
                    named_barrier(2, kSplitThreads);
                    if (prob + gridDim.x < nprob)
                    {
                        if (t == 0)
                            stage_problem(&tmA, &tmB, prob + gridDim.x, stage, sfull);
                        issued = j + 2;
                    }
                }
                // the digit buffer is free once the MMAs of its last problem completed
                if (pass == 0 &&
                    !barrier_and(2, kSplitThreads,
                                 j < sp.nbuf || tc::mbar_wait_bounded(&dempty[b], ((j / sp.nbuf) - 1) & 1, limit)))
                {
                    ok = false;
                    break;
                }
                split_loaded<SK, S>(r, mx, row, half, is_b ? buf + nstack * kStackBytes : buf, is_b ? ex + 64 : ex,
                                    sp.staged && !strided ? half : 0);
            }
            if (!ok)
            {
                atomicExch(&g_split_error, 5);
                break;
            }
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
        // ---- recombination role: warps 4..11, lane quadrant warp % 4, column
        //      group (warp - 4) / 4; lane 0 of warp 4 also issues the MMAs ----
        const int quad = warp & 3, grp = (warp - kSplitWarps) >> 2;
        const int L = quad * 32 + lane;
        const bool top = L < 64;
        const bool issuer = warp == kSplitWarps && lane == 0;
        const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
        double *xg = xfer + grp * (64 * W);
        const int gbar = 1 + 2 * grp;
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
            if (!barrier_and(4, 256, tc::mbar_wait_bounded(tfull, j & 1, limit)))
            {
                atomicExch(&g_split_error, 7);
                break;
            }
            tc::tc_fence_after();
            const int *eA = exps + (j % kExpRing) * 128;
            const int *eB = eA + 64;
            double *Cp = p.C + prob * p.sC;
            for (int jc = 0; jc < 32; jc += W)
            {
                const int j0 = grp * 32 + jc;
                double acc[W];
                gather_chunk<bmax, W, SK>(tmem + lane_addr + j0, top, p.beta, acc);
                if (jc == 32 - W)
                {
                    // every TMEM read of problem j is done: start problem j+1
                    tc::tc_fence_before();
                    named_barrier(4, 256);
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
                finish_half_chunk<W>(p, Cp, eA, eB, xg, acc, L, j0, gbar);
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == kSplitWarps)
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
    int persistent_threads;
};

template <int SK, int S>
SplitFns split_fns()
{
    return {(const void *)&split_f64_kernel<SK, S>, (const void *)&split_f64_persistent<SK, S>,
            persistent_threads<SK, S>()};
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
    return {nullptr, nullptr, 0};
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

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn split_encode_fn()
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

// FP64 map {inner, rows, batch} with boxes of 16 x 64 x 1, 128-byte swizzle
// and zero fill outside the tensor (the stage layout of the persistent form).
// Needs a 16-byte aligned base and row / problem strides that are multiples
// of 16 bytes; false when the driver refuses the map.
bool make_stage_map(CUtensorMap *map, const double *base, int inner, int rows, int64_t batch, int64_t ld,
                    int64_t stride)
{
    EncodeTiledFn fn = split_encode_fn();
    if (!fn)
        return false;
    cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)rows, (cuuint64_t)batch};
    const int64_t s2 = batch > 1 ? stride : (int64_t)rows * ld;
    cuuint64_t strides[2] = {(cuuint64_t)(ld * 8), (cuuint64_t)((s2 > 0 ? s2 : ld * rows) * 8)};
    cuuint32_t box[3] = {16, 64, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

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
        // tensor copies need 16-byte aligned bases and row / problem strides
        // that are multiples of 16 bytes
        const bool a_ok = !(reinterpret_cast<uintptr_t>(A) & 15) && !(lda & 1) && (batch == 1 || !(strideA & 1));
        const bool b_ok = !(reinterpret_cast<uintptr_t>(B) & 15) && !(ldb & 1) && (batch == 1 || !(strideB & 1));
        CUtensorMap mapA, mapB;
        memset(&mapA, 0, sizeof(mapA));
        memset(&mapB, 0, sizeof(mapB));
        sp.staged = a_ok && b_ok && make_stage_map(&mapA, A, K, M, batch, lda, strideA) &&
                            (b_layout == KAMI_B_REF_NK ? make_stage_map(&mapB, B, K, N, batch, ldb, strideB)
                                                       : make_stage_map(&mapB, B, N, K, batch, ldb, strideB))
                        ? 1
                        : 0;
        const size_t fixed = (size_t)kXferBytes + kExpRing * 128 * 4 + 128 + 1024 + (sp.staged ? kStageBytes : 0);
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
        void *args2[] = {&sp, &mapA, &mapB};
        e2 = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)fns.persistent_threads), args2, smem, st);
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
