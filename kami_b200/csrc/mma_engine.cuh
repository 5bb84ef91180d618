// mma_engine.cuh -- the register-resident block GEMM on warp mma.sync.
//
// One CTA computes whole small GEMMs C = A * op(B) (one problem per group of
// warps; a CTA may hold several groups).  Each warp is a "rank": it loads its
// slices of A and B into registers once, and the warps exchange operand
// fragments through a small shared-memory buffer, one broadcast stage per
// rank, while C stays in registers -- the communication-avoiding block GEMM
// of KAMI, in its three partitionings:
//
//   1D (P warps)      warp w owns A rows w*M/P.. (all K) and B's N-slice w.
//                     Stage s: warp s publishes its B slice; every warp
//                     multiplies it into C columns of slice s.
//                     (block_gemm_1d_half_mma.cu:130-170)
//   2D (P x P warps)  warp (r,c) owns A(r, kslice c) and B(c, kslice r).
//                     Stage s: warps with c == s publish A, warps with r == s
//                     publish B; warp (r,c) accumulates C(r,c) (SUMMA).
//                     (block_gemm_2d_half_mma.cu:140-197)
//   3D (P^3 warps)    warp (r,c,d) owns A(r, kblock c*P+d), B(c, kblock r*P+d).
//                     Stage s publishes as in 2D per depth d; warp (r,c,d)
//                     accumulates a partial C(r,c) over kblocks s*P+d.  The
//                     P partials are reduced on the device through shared
//                     memory (each depth warp owns 1/P of the tile's
//                     fragments), where the reference reduced them on the
//                     host (block_gemm_3d_half_mma.cu:147-196, :291-300).
//
// Differences from the reference, all B200-motivated:
//   * FP16/BF16 inputs accumulate in FP32 (m16n8k16.f32); FP64 uses DMMA
//     m16n8k8.  One engine serves both through a traits class.
//   * The exchange buffer is double-buffered, so a stage needs one barrier
//     instead of two, and the barrier is a named barrier over the group's
//     warps only.
//   * Global loads are vectorised: within every MMA k-step the k index is
//     permuted identically for A and B (lane t holds 2 consecutive "units" at
//     k0 + 2t units), which leaves each dot product unchanged and turns the
//     reference's 32-bit loads into 64-bit (FP16) / 128-bit (FP64) loads.
//   * P == 1 keeps everything in registers (no shared-memory round trip).
//
// Two optional forms, compiled only where an instance asks for them:
//   * K split (RK >= 0, 1D): only the first RK k-steps of each rank's A and B
//     slices stay in registers; the remaining k-steps are written once to a
//     shared-memory cache (A per rank, B readable by every rank) and read
//     from there at every stage -- the register / shared-memory residency
//     trade-off of the reference's src/reg_smem/block_gemm_1d_half_mma.cu
//     (REG_K_SPLIT_BLOCK, :30-46).  It lets 1D 128^3 run with P = 4, whose
//     all-register form does not fit the register file.  RK = 0 caches
//     everything and needs no barrier after the first.
//   * TRACE: clock64 counts per warp of the cycles spent communicating
//     (publishing fragments and waiting at the stage barrier) and computing
//     (fragment reads and MMAs), written for problem 0 to GemmArgs::trace --
//     the measurement of the reference's src/usage_cycle/ kernels
//     (block_gemm_1d_half_mma_usage_cycle.cu:127-197), kept out of the
//     untraced instances.
#pragma once

#include "kami_common.cuh"

namespace kami {

// ---------------------------------------------------------------------------
// MMA traits.  A "unit" is what one MMA register holds along k: two 16-bit
// elements (FP16/BF16) or one double (FP64).  A k-step is 8 units.
// ---------------------------------------------------------------------------
template <bool BF16>
struct TrH16
{
    using Unit = uint32_t;
    using Acc = float;
    using Elem = uint16_t;
    static constexpr int EPU = 2;    // elements per unit
    static constexpr int KSTEP = 16; // elements per MMA k-step
    static constexpr int kInType = BF16 ? KAMI_BF16 : KAMI_F16;

    __device__ __forceinline__ static void mma(Acc (&d)[4], const Unit (&a)[4], Unit b0, Unit b1)
    {
        if constexpr (BF16)
            asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};"
                : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
        else
            asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};"
                : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
    // two units (4 contiguous elements, 8-byte aligned)
    __device__ __forceinline__ static void ld2(const Elem *p, Unit &lo, Unit &hi)
    {
        uint2 v = __ldg(reinterpret_cast<const uint2 *>(p));
        lo = v.x;
        hi = v.y;
    }
    // two units gathered from 4 elements at stride s
    __device__ __forceinline__ static void gather2(const Elem *p, int64_t s, Unit &lo, Unit &hi)
    {
        lo = (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + s) << 16);
        hi = (uint32_t)__ldg(p + 2 * s) | ((uint32_t)__ldg(p + 3 * s) << 16);
    }
    __device__ __forceinline__ static void st2(Unit *s, Unit x, Unit y)
    {
        *reinterpret_cast<uint2 *>(s) = make_uint2(x, y);
    }
    // two units (4 contiguous elements) from shared memory
    __device__ __forceinline__ static void ld2_smem(const Elem *p, Unit &lo, Unit &hi)
    {
        uint2 v = *reinterpret_cast<const uint2 *>(p);
        lo = v.x;
        hi = v.y;
    }
    __device__ __forceinline__ static void lds2(const Unit *s, Unit &x, Unit &y)
    {
        uint2 v = *reinterpret_cast<const uint2 *>(s);
        x = v.x;
        y = v.y;
    }
};

struct TrF64
{
    using Unit = double;
    using Acc = double;
    using Elem = double;
    static constexpr int EPU = 1;
    static constexpr int KSTEP = 8;
    static constexpr int kInType = KAMI_F64;

    __device__ __forceinline__ static void mma(Acc (&d)[4], const Unit (&a)[4], Unit b0, Unit b1)
    {
        asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
    }
    __device__ __forceinline__ static void ld2(const Elem *p, Unit &lo, Unit &hi)
    {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        lo = v.x;
        hi = v.y;
    }
    __device__ __forceinline__ static void gather2(const Elem *p, int64_t s, Unit &lo, Unit &hi)
    {
        lo = __ldg(p);
        hi = __ldg(p + s);
    }
    __device__ __forceinline__ static void st2(Unit *s, Unit x, Unit y)
    {
        *reinterpret_cast<double2 *>(s) = make_double2(x, y);
    }
    __device__ __forceinline__ static void ld2_smem(const Elem *p, Unit &lo, Unit &hi)
    {
        double2 v = *reinterpret_cast<const double2 *>(p);
        lo = v.x;
        hi = v.y;
    }
    __device__ __forceinline__ static void lds2(const Unit *s, Unit &x, Unit &y)
    {
        double2 v = *reinterpret_cast<const double2 *>(s);
        x = v.x;
        y = v.y;
    }
};

// ---------------------------------------------------------------------------
// Compile-time geometry of one (traits, BM, BN, BK, P, partition) instance.
// ---------------------------------------------------------------------------
template <class Tr, int BM, int BN, int BK, int P, int PART, int RK = -1>
struct BlockGeom
{
    static constexpr int NW = PART == 1 ? P : PART == 2 ? P * P : P * P * P;
    static constexpr int SUB_M = BM / P;
    static constexpr int SUB_N = BN / P;
    static constexpr int SUB_K = PART == 1 ? BK : PART == 2 ? BK / P : BK / (P * P);
    static constexpr int TM = SUB_M / 16;
    static constexpr int TN = SUB_N / 8;
    static constexpr int TK = SUB_K / Tr::KSTEP;
    static constexpr int CN = PART == 1 ? BN / 8 : TN; // C n-tiles per warp
    static_assert(PART >= 1 && PART <= 3, "partition");
    static_assert(TM * 16 * P == BM && TN * 8 * P == BN, "M/P must be a multiple of 16, N/P of 8");
    static_assert(TK >= 1 && TK * Tr::KSTEP == SUB_K, "per-rank K slice must be a multiple of the MMA k-step");
    static_assert(NW <= 32, "at most 32 warps per problem");

    // K split: k-steps of a rank's slices held in registers (RKE) and in the
    // shared-memory cache (SKE)
    static constexpr int RKE = RK < 0 ? TK : RK;
    static constexpr int SKE = TK - RKE;
    static_assert(RK < 0 || (PART == 1 && P > 1 && RK <= TK), "the K split is a 1D form with P > 1");

    static constexpr bool EXCHANGE = P > 1 && RKE > 0;
    static constexpr int A_FRAG_U = 4 * 32; // units per published A fragment
    static constexpr int B_FRAG_U = 2 * 32;
    static constexpr int XA_SLOTS = PART == 1 ? 0 : PART == 2 ? P : P * P;
    static constexpr int XB_SLOTS = PART == 1 ? 1 : PART == 2 ? P : P * P;
    static constexpr int XA_SLOT_U = TM * TK * A_FRAG_U;
    static constexpr int XB_SLOT_U = TN * RKE * B_FRAG_U;
    static constexpr int XBUF_U = XA_SLOTS * XA_SLOT_U + XB_SLOTS * XB_SLOT_U;
    static constexpr size_t XBYTES = EXCHANGE ? 2ull * XBUF_U * sizeof(typename Tr::Unit) : 0;
    static constexpr int F = TM * TN;
    static constexpr int FO = (F + P - 1) / P;
    static constexpr size_t RBYTES =
        (PART == 3 && P > 1) ? (size_t)P * P * P * (P - 1) * FO * 32 * 4 * sizeof(typename Tr::Acc) : 0;
    // K-split caches, per rank: A fragments (read by the rank itself) then B
    // fragments (read by every rank at the rank's stage)
    static constexpr int AC_U = TM * SKE * A_FRAG_U;
    static constexpr int BC_U = TN * SKE * B_FRAG_U;
    static constexpr size_t XR = XBYTES > RBYTES ? XBYTES : RBYTES;
    static constexpr size_t CBYTES = (size_t)NW * (AC_U + BC_U) * sizeof(typename Tr::Unit);
    static constexpr size_t SMEM = XR + CBYTES; // per problem group
};

template <class Tr>
__device__ __forceinline__ void load_a_frag(const GemmArgs &g, const typename Tr::Elem *A, int r, int kk,
                                            typename Tr::Unit (&a)[4])
{
    using Unit = typename Tr::Unit;
    const bool kin = kk < g.K;
    Unit lo0 = Unit(0), hi0 = Unit(0), lo1 = Unit(0), hi1 = Unit(0);
    if (g.a_layout == KAMI_A_ROW_MK)
    {
        if (kin && r < g.M)
            Tr::ld2(A + (int64_t)r * g.lda + kk, lo0, hi0);
        if (kin && r + 8 < g.M)
            Tr::ld2(A + (int64_t)(r + 8) * g.lda + kk, lo1, hi1);
    }
    else
    {
        if (kin && r < g.M)
            Tr::gather2(A + (int64_t)kk * g.lda + r, g.lda, lo0, hi0);
        if (kin && r + 8 < g.M)
            Tr::gather2(A + (int64_t)kk * g.lda + r + 8, g.lda, lo1, hi1);
    }
    a[0] = lo0;
    a[1] = lo1;
    a[2] = hi0;
    a[3] = hi1;
}

template <class Tr>
__device__ __forceinline__ void load_b_frag(const GemmArgs &g, const typename Tr::Elem *B, int n, int kk,
                                            typename Tr::Unit (&b)[2])
{
    using Unit = typename Tr::Unit;
    Unit lo = Unit(0), hi = Unit(0);
    if (kk < g.K && n < g.N)
    {
        if (g.b_layout == KAMI_B_REF_NK)
            Tr::ld2(B + (int64_t)n * g.ldb + kk, lo, hi);
        else
            Tr::gather2(B + (int64_t)kk * g.ldb + n, g.ldb, lo, hi);
    }
    b[0] = lo;
    b[1] = hi;
}

template <class Tr, int BM, int BN, int BK, int P, int PART, int RK = -1, bool TRACE = false>
__global__ void block_mma_kernel(const GemmArgs g)
{
    using G = BlockGeom<Tr, BM, BN, BK, P, PART, RK>;
    using Unit = typename Tr::Unit;
    using Acc = typename Tr::Acc;
    using Elem = typename Tr::Elem;
    constexpr int TM = G::TM, TN = G::TN, TK = G::TK, CN = G::CN;
    constexpr int KU = Tr::KSTEP; // elements per k-step

    extern __shared__ __align__(16) unsigned char smem_raw[];

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int group = warp / G::NW;
    const int w = warp % G::NW;
    if (group >= g.problems_per_cta)
        return; // warps beyond the partition (NUM_ALLOC_RANK_BLOCK extras) leave
    const int64_t prob = (int64_t)blockIdx.x * g.problems_per_cta + group;
    if (prob >= g.batch)
        return; // the whole group leaves together; its barrier is its own

    const int bar_id = 1 + group;
    constexpr int bar_n = G::NW * 32;
    Unit *xbuf = reinterpret_cast<Unit *>(smem_raw + (size_t)group * G::SMEM);

    int wr, wc, wd;
    if constexpr (PART == 1)
    {
        wr = w;
        wc = 0;
        wd = 0;
    }
    else if constexpr (PART == 2)
    {
        wr = w / P;
        wc = w % P;
        wd = 0;
    }
    else
    {
        wr = w / (P * P);
        wc = (w / P) % P;
        wd = w % P;
    }

    const Elem *A = reinterpret_cast<const Elem *>(g.A) + prob * g.sA;
    const Elem *B = reinterpret_cast<const Elem *>(g.B) + prob * g.sB;
    const int gq = lane >> 2, tq = lane & 3;

    // origins of the rank-owned slices
    const int a_row0 = wr * G::SUB_M;
    const int a_k0 = PART == 1 ? 0 : PART == 2 ? wc * G::SUB_K : (wc * P + wd) * G::SUB_K;
    const int b_n0 = PART == 1 ? wr * G::SUB_N : wc * G::SUB_N;
    const int b_k0 = PART == 1 ? 0 : PART == 2 ? wr * G::SUB_K : (wr * P + wd) * G::SUB_K;
    const int lane_k = tq * 2 * Tr::EPU; // permuted k offset of this lane inside a k-step

    constexpr int RKE = G::RKE, SKE = G::SKE, RKA = RKE > 0 ? RKE : 1;
    Unit a[TM][RKA][4];
    Unit b[TN][RKA][2];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int k = 0; k < RKE; ++k)
            load_a_frag<Tr>(g, A, a_row0 + 16 * i + gq, a_k0 + k * KU + lane_k, a[i][k]);
#pragma unroll
    for (int j = 0; j < TN; ++j)
#pragma unroll
        for (int k = 0; k < RKE; ++k)
            load_b_frag<Tr>(g, B, b_n0 + 8 * j + gq, b_k0 + k * KU + lane_k, b[j][k]);
    // K split: the k-steps past RKE go to this rank's shared-memory cache
    Unit *cache = reinterpret_cast<Unit *>(smem_raw + (size_t)group * G::SMEM + G::XR);
    if constexpr (SKE > 0)
    {
        Unit *ac = cache + w * (G::AC_U + G::BC_U), *bc = ac + G::AC_U;
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int k = 0; k < SKE; ++k)
            {
                Unit f[4];
                load_a_frag<Tr>(g, A, a_row0 + 16 * i + gq, a_k0 + (RKE + k) * KU + lane_k, f);
                Unit *d = ac + (i * SKE + k) * G::A_FRAG_U;
                Tr::st2(d + lane * 2, f[0], f[1]);
                Tr::st2(d + 64 + lane * 2, f[2], f[3]);
            }
#pragma unroll
        for (int j = 0; j < TN; ++j)
#pragma unroll
            for (int k = 0; k < SKE; ++k)
            {
                Unit f[2];
                load_b_frag<Tr>(g, B, b_n0 + 8 * j + gq, b_k0 + (RKE + k) * KU + lane_k, f);
                Tr::st2(bc + (j * SKE + k) * G::B_FRAG_U + lane * 2, f[0], f[1]);
            }
    }
    long long t_comm = 0, t_comp = 0; // TRACE instances only

    Acc acc[TM][CN][4];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < CN; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                acc[i][j][e] = Acc(0);

    if constexpr (P == 1)
    {
        // P == 1: one rank holds everything; no exchange.
        const long long t0 = TRACE ? clock64() : 0;
        for (int it = 0; it < g.num_iter; ++it)
        {
#pragma unroll
            for (int k = 0; k < TK; ++k)
#pragma unroll
                for (int j = 0; j < TN; ++j)
#pragma unroll
                    for (int i = 0; i < TM; ++i)
                        Tr::mma(acc[i][j], a[i][k], b[j][k][0], b[j][k][1]);
        }
        if constexpr (TRACE)
            t_comp += clock64() - t0;
    }
    else
    {
        for (int it = 0; it < g.num_iter; ++it)
        {
#pragma unroll
            for (int s = 0; s < P; ++s)
            {
                const int parity = (it * P + s) & 1;
                Unit *xa = xbuf + parity * G::XBUF_U;
                Unit *xb = xa + G::XA_SLOTS * G::XA_SLOT_U;
                const long long t0 = TRACE ? clock64() : 0;
                // ---- publish ----
                if constexpr (PART == 1)
                {
                    if (RKE > 0 && wr == s)
                    {
#pragma unroll
                        for (int j = 0; j < TN; ++j)
#pragma unroll
                            for (int k = 0; k < RKE; ++k)
                                Tr::st2(xb + (j * RKE + k) * G::B_FRAG_U + lane * 2, b[j][k][0], b[j][k][1]);
                    }
                }
                else
                {
                    const int a_slot = PART == 2 ? wr : wr * P + wd;
                    const int b_slot = PART == 2 ? wc : wc * P + wd;
                    if (wc == s)
                    {
                        Unit *dst = xa + a_slot * G::XA_SLOT_U;
#pragma unroll
                        for (int i = 0; i < TM; ++i)
#pragma unroll
                            for (int k = 0; k < TK; ++k)
                            {
                                Unit *f = dst + (i * TK + k) * G::A_FRAG_U;
                                Tr::st2(f + lane * 2, a[i][k][0], a[i][k][1]);
                                Tr::st2(f + 64 + lane * 2, a[i][k][2], a[i][k][3]);
                            }
                    }
                    if (wr == s)
                    {
                        Unit *dst = xb + b_slot * G::XB_SLOT_U;
#pragma unroll
                        for (int j = 0; j < TN; ++j)
#pragma unroll
                            for (int k = 0; k < TK; ++k)
                                Tr::st2(dst + (j * TK + k) * G::B_FRAG_U + lane * 2, b[j][k][0], b[j][k][1]);
                    }
                }
                // the exchange needs a barrier per stage; an all-cached K split
                // only one, before the caches are first read
                if (RKE > 0 || (it == 0 && s == 0))
                    named_barrier(bar_id, bar_n);
                long long t1 = 0;
                if constexpr (TRACE)
                {
                    t1 = clock64();
                    t_comm += t1 - t0;
                }
                // ---- compute ----
                if constexpr (PART == 1)
                {
#pragma unroll
                    for (int j = 0; j < TN; ++j)
#pragma unroll
                        for (int k = 0; k < RKE; ++k)
                        {
                            Unit b0, b1;
                            Tr::lds2(xb + (j * RKE + k) * G::B_FRAG_U + lane * 2, b0, b1);
#pragma unroll
                            for (int i = 0; i < TM; ++i)
                                Tr::mma(acc[i][s * TN + j], a[i][k], b0, b1);
                        }
                    if constexpr (SKE > 0)
                    {
                        const Unit *ac = cache + w * (G::AC_U + G::BC_U);
                        const Unit *bc = cache + s * (G::AC_U + G::BC_U) + G::AC_U; // rank s's B
#pragma unroll
                        for (int k = 0; k < SKE; ++k)
                        {
                            Unit af[TM][4];
#pragma unroll
                            for (int i = 0; i < TM; ++i)
                            {
                                const Unit *f = ac + (i * SKE + k) * G::A_FRAG_U;
                                Tr::lds2(f + lane * 2, af[i][0], af[i][1]);
                                Tr::lds2(f + 64 + lane * 2, af[i][2], af[i][3]);
                            }
#pragma unroll
                            for (int j = 0; j < TN; ++j)
                            {
                                Unit b0, b1;
                                Tr::lds2(bc + (j * SKE + k) * G::B_FRAG_U + lane * 2, b0, b1);
#pragma unroll
                                for (int i = 0; i < TM; ++i)
                                    Tr::mma(acc[i][s * TN + j], af[i], b0, b1);
                            }
                        }
                    }
                }
                else
                {
                    const Unit *sa = xa + (PART == 2 ? wr : wr * P + wd) * G::XA_SLOT_U;
                    const Unit *sb = xb + (PART == 2 ? wc : wc * P + wd) * G::XB_SLOT_U;
#pragma unroll
                    for (int k = 0; k < TK; ++k)
                    {
                        Unit af[TM][4];
#pragma unroll
                        for (int i = 0; i < TM; ++i)
                        {
                            const Unit *f = sa + (i * TK + k) * G::A_FRAG_U;
                            Tr::lds2(f + lane * 2, af[i][0], af[i][1]);
                            Tr::lds2(f + 64 + lane * 2, af[i][2], af[i][3]);
                        }
#pragma unroll
                        for (int j = 0; j < TN; ++j)
                        {
                            Unit b0, b1;
                            Tr::lds2(sb + (j * TK + k) * G::B_FRAG_U + lane * 2, b0, b1);
#pragma unroll
                            for (int i = 0; i < TM; ++i)
                                Tr::mma(acc[i][j], af[i], b0, b1);
                        }
                    }
                }
                if constexpr (TRACE)
                    t_comp += clock64() - t1;
            }
        }
    }
    if constexpr (TRACE)
    {
        if (lane == 0 && prob == 0 && g.trace)
        {
            g.trace[2 * w] = (unsigned long long)t_comm;
            g.trace[2 * w + 1] = (unsigned long long)t_comp;
        }
    }

    void *Cb = reinterpret_cast<char *>(g.C) +
               prob * g.sC * (g.out_type == KAMI_F64 ? 8 : g.out_type == KAMI_F32 ? 4 : 2);
    const int c_row0 = wr * G::SUB_M;
    const int c_col0 = PART == 1 ? 0 : wc * G::SUB_N;

    if constexpr (PART == 3 && P > 1)
    {
        // ---- on-device reduction of the P depth partials ----
        // fragment f = i*TN + j of tile (wr,wc) is owned by depth f % P; every
        // other depth leaves its partial of f in shared memory.
        named_barrier(bar_id, bar_n); // everyone is done with the exchange buffers
        Acc *red = reinterpret_cast<Acc *>(xbuf);
        const int tile = wr * P + wc;
#pragma unroll
        for (int f = 0; f < G::F; ++f)
        {
            const int o = f % P;
            if (o != wd)
            {
                const int slot = wd < o ? wd : wd - 1;
                Acc *dst = red + ((((size_t)tile * P + o) * (P - 1) + slot) * G::FO + f / P) * 128 + lane * 4;
                const int i = f / TN, j = f % TN;
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    dst[e] = acc[i][j][e];
            }
        }
        named_barrier(bar_id, bar_n);
#pragma unroll
        for (int f = 0; f < G::F; ++f)
        {
            if (f % P == wd)
            {
                const int i = f / TN, j = f % TN;
#pragma unroll
                for (int slot = 0; slot < P - 1; ++slot)
                {
                    const Acc *src = red + ((((size_t)tile * P + wd) * (P - 1) + slot) * G::FO + f / P) * 128 + lane * 4;
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        acc[i][j][e] += src[e];
                }
                const int r = c_row0 + 16 * i + gq;
                const int c = c_col0 + 8 * j + 2 * tq;
                store_pair<Acc>(g, Cb, r, c, acc[i][j][0], acc[i][j][1]);
                store_pair<Acc>(g, Cb, r + 8, c, acc[i][j][2], acc[i][j][3]);
            }
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < CN; ++j)
            {
                const int r = c_row0 + 16 * i + gq;
                const int c = c_col0 + 8 * j + 2 * tq;
                store_pair<Acc>(g, Cb, r, c, acc[i][j][0], acc[i][j][1]);
                store_pair<Acc>(g, Cb, r + 8, c, acc[i][j][2], acc[i][j][3]);
            }
    }
}

// ---------------------------------------------------------------------------
// Registry of compiled instances, filled by the instantiation files.
// ---------------------------------------------------------------------------
struct MmaInstance
{
    int in_type; // KAMI_F16 / KAMI_BF16 / KAMI_F64
    int part;
    int BM, BN, BK, P;
    int nwarps;
    size_t smem_per_group;
    const void *fn; // __global__ function
};

// Each instantiation .cu file defines one of these; kami_abi.cu concatenates.
const MmaInstance *mma_instances_f16(int *count);
const MmaInstance *mma_instances_bf16(int *count);
const MmaInstance *mma_instances_f64(int *count);

#define KAMI_MMA_INSTANCE(TR, INTYPE, BM, BN, BK, P, PART)                                                      \
    MmaInstance                                                                                                  \
    {                                                                                                            \
        INTYPE, PART, BM, BN, BK, P, BlockGeom<TR, BM, BN, BK, P, PART>::NW,                                     \
            BlockGeom<TR, BM, BN, BK, P, PART>::SMEM, (const void *)&block_mma_kernel<TR, BM, BN, BK, P, PART> \
    }

} // namespace kami
