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
#include <algorithm>
#include <cstring>
#include <mutex>

#include "kami_common.cuh"
#include "tc05_epi.cuh"
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
    int store_slots;    // per-problem kernel: staging boxes per warp for bulk C stores (0: per-thread stores)
};

__device__ __forceinline__ void tc05_flag(int code) { atomicExch(&g_tc05_error, code); }

// The MMA issue loop of one problem (one thread).  Operand descriptors
// advance by addition (16-byte units of the start-address field: +32 B per
// k-step along a K-major row, +2 KB down an MN-major box, a jump to the next
// 64-element K box every 4 k-steps).  The single issuing thread has to keep
// pace with 64-cycle MMAs, so the common single-accumulator case hoists every
// invariant out of the repeat loop and unrolls the k-steps exactly when their
// count is a small compile-time constant (1, 2, 4, 8); other counts take a
// runtime loop.  Repeated products (batch 592, 1000 repeats): a runtime loop
// rebuilding the descriptors every repeat measured 1708 / 1784 / 1151 / 700
// TFLOP/s at 128^3 / 128x128x32 / 128x128x16 / 64^3, this form 1899 / 1846 /
// 1677 / 1000; a fully unrolled loop predicated on the count was slower than
// either.
__device__ __forceinline__ uint64_t kdesc(uint32_t base, int box, int mn, int ks)
{
    const uint32_t addr = base + (uint32_t)((ks >> 2) * box + (ks & 3) * (mn ? 2048 : 32));
    return mn ? tc::desc_mnmajor_sw128(addr, 8192) : tc::desc_kmajor_sw128(addr);
}

template <bool TS, int KS>
__device__ __forceinline__ void repeat_mmas(const Tc05Params &p, uint32_t tmem, uint64_t ad0, uint64_t bd0,
                                            uint32_t at0, uint64_t a_in, uint64_t b_in, uint64_t a_wrap,
                                            uint64_t b_wrap, int ks_n)
{
    for (int it = 0; it < p.g.num_iter; ++it)
    {
        uint64_t ad = ad0, bd = bd0;
        uint32_t at = at0;
#pragma unroll
        for (int ks = 0; ks < (KS ? KS : ks_n); ++ks)
        {
            const uint32_t acc = (it > 0 || ks > 0) ? 1u : 0u;
            if (TS)
                tc::mma_f16_ts(tmem, at, bd, p.idesc, acc);
            else
                tc::mma_f16_ss(tmem, ad, bd, p.idesc, acc);
            const bool wrap = (ks & 3) == 3;
            ad += wrap ? a_wrap : a_in;
            bd += wrap ? b_wrap : b_in;
            at += 8;
        }
    }
}

template <bool TS>
__device__ __forceinline__ void issue_mmas(const Tc05Params &p, uint32_t tmem, uint32_t a0, uint32_t b0, int a_box,
                                           int b_box)
{
    const int depth = p.part == 3 ? p.P : 1;
    const int panels = p.part == 2 ? p.P : 1;
    const int pn = p.bn / panels;
    const uint64_t a_in = p.a_mn ? 128 : 2, b_in = p.b_mn ? 128 : 2;
    const uint64_t a_wrap = (uint64_t)(a_box >> 4) - 3 * a_in, b_wrap = (uint64_t)(b_box >> 4) - 3 * b_in;
    // descriptor step between B panels (2D), in 16-byte units
    const uint64_t qstep = p.b_mn ? (uint64_t)(pn / 64) * (8192 >> 4) : (uint64_t)pn * (128 >> 4);
    if (depth == 1 && panels == 1)
    {
        const uint64_t ad0 = TS ? 0 : kdesc(a0, a_box, p.a_mn, 0), bd0 = kdesc(b0, b_box, p.b_mn, 0);
        const uint32_t at0 = tmem + p.a_col;
        switch (p.ksteps)
        {
        case 1: repeat_mmas<TS, 1>(p, tmem, ad0, bd0, at0, a_in, b_in, a_wrap, b_wrap, 1); return;
        case 2: repeat_mmas<TS, 2>(p, tmem, ad0, bd0, at0, a_in, b_in, a_wrap, b_wrap, 2); return;
        case 4: repeat_mmas<TS, 4>(p, tmem, ad0, bd0, at0, a_in, b_in, a_wrap, b_wrap, 4); return;
        case 8: repeat_mmas<TS, 8>(p, tmem, ad0, bd0, at0, a_in, b_in, a_wrap, b_wrap, 8); return;
        default: repeat_mmas<TS, 0>(p, tmem, ad0, bd0, at0, a_in, b_in, a_wrap, b_wrap, p.ksteps); return;
        }
    }
    for (int it = 0; it < p.g.num_iter; ++it)
    {
        for (int d = 0; d < depth; ++d)
        {
            const int k_lo = p.ksteps * d / depth, k_hi = p.ksteps * (d + 1) / depth;
            const uint32_t dcol = tmem + (uint32_t)(d * p.bn);
            uint64_t ad = TS ? 0 : kdesc(a0, a_box, p.a_mn, k_lo);
            uint64_t bd = kdesc(b0, b_box, p.b_mn, k_lo);
            uint32_t at = tmem + p.a_col + (uint32_t)k_lo * 8;
            for (int ks = k_lo; ks < k_hi; ++ks)
            {
                const uint32_t acc = (it > 0 || ks > k_lo) ? 1u : 0u;
                if (panels == 1)
                {
                    if (TS)
                        tc::mma_f16_ts(dcol, at, bd, p.idesc, acc);
                    else
                        tc::mma_f16_ss(dcol, ad, bd, p.idesc, acc);
                }
                else
                {
                    for (int q = 0; q < panels; ++q)
                    {
                        if (TS)
                            tc::mma_f16_ts(dcol + q * pn, at, bd + q * qstep, p.idesc, acc);
                        else
                            tc::mma_f16_ss(dcol + q * pn, ad, bd + q * qstep, p.idesc, acc);
                    }
                }
                const bool wrap = (ks & 3) == 3;
                ad += wrap ? a_wrap : a_in;
                bd += wrap ? b_wrap : b_in;
                at += 8;
            }
        }
    }
}


// C through bulk tensor stores: each warp packs 128 bytes of each of its rows
// (32 FP32 or 64 16-bit columns, the sum of the depth accumulators) into a
// 128B-swizzled staging box and one lane stores the box.  The boxes live in
// the operand tiles, dead once the MMAs have completed; with fewer slots than
// boxes a slot is rewritten after the bulk stores have read it.
struct BulkOut
{
    int out_type;
    int rows, cols;   // valid extent of the output tile (M x N)
    int bm;           // accumulator rows (MMA M: 64 -> 16 rows per warp, 128 -> 32)
    int bn;           // accumulator columns read (a whole number of boxes)
    int depth;        // accumulators summed, bn columns apart
    int slots;        // staging boxes per warp
};

__device__ __forceinline__ void epilogue_bulk(const BulkOut &o, const CUtensorMap *tmC, uint32_t tcol, uint8_t *stg,
                                              int row_base, int prob)
{
    const int lane = threadIdx.x & 31;
    const bool f32 = o.out_type == KAMI_F32, bf = o.out_type == KAMI_BF16;
    const int rows = o.bm == 128 ? 32 : 16;
    const int bcols = f32 ? 32 : 64;
    const int box_bytes = rows * 128;
    int nb = 0;
    for (int c0 = 0; c0 < o.bn; c0 += bcols, ++nb)
    {
        uint8_t *box = stg + (nb % o.slots) * box_bytes;
        if (nb >= o.slots)
        {
            if (lane == 0)
                tc::bulk_wait_read<0>();
            __syncwarp();
        }
        uint8_t *row = box + lane * 128;
        // 16 columns at a time: 64 bytes (FP32) or 32 bytes (16-bit) of the row
#pragma unroll
        for (int h = 0; h < 4; ++h)
        {
            if (h >= bcols / 16)
                break;
            uint32_t v[16];
            tc::tmem_ld16(tcol + c0 + 16 * h, v);
            tc::tmem_ld_wait();
            float f[16];
#pragma unroll
            for (int e = 0; e < 16; ++e)
                f[e] = __uint_as_float(v[e]);
            for (int d = 1; d < o.depth; ++d)
            {
                uint32_t u[16];
                tc::tmem_ld16(tcol + d * o.bn + c0 + 16 * h, u);
                tc::tmem_ld_wait();
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    f[e] += __uint_as_float(u[e]);
            }
            if (lane < rows)
            {
                if (f32)
                {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        *reinterpret_cast<uint4 *>(row + (((4 * h + q) ^ (lane & 7)) << 4)) =
                            make_uint4(__float_as_uint(f[4 * q]), __float_as_uint(f[4 * q + 1]),
                                       __float_as_uint(f[4 * q + 2]), __float_as_uint(f[4 * q + 3]));
                }
                else
                {
#pragma unroll
                    for (int q = 0; q < 2; ++q)
                        *reinterpret_cast<uint4 *>(row + (((2 * h + q) ^ (lane & 7)) << 4)) =
                            make_uint4(pack2(f[8 * q], f[8 * q + 1], bf), pack2(f[8 * q + 2], f[8 * q + 3], bf),
                                       pack2(f[8 * q + 4], f[8 * q + 5], bf), pack2(f[8 * q + 6], f[8 * q + 7], bf));
                }
            }
        }
        tc::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0)
        {
            if (row_base < o.rows && c0 < o.cols)
                tc::tma_store_3d(tmC, box, c0, row_base, prob);
            tc::bulk_commit();
        }
    }
    if (lane == 0)
        tc::bulk_wait_read<0>();
    __syncwarp();
}

template <bool BF16>
__global__ void __launch_bounds__(128) tc05_block_kernel(const __grid_constant__ CUtensorMap tmA,
                                                         const __grid_constant__ CUtensorMap tmB,
                                                         const __grid_constant__ CUtensorMap tmC,
                                                         const Tc05Params p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment of the swizzle atoms
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_box = p.a_tmem ? 0 : p.bm * 128, b_box = p.bn * 128;
    uint8_t *sA = smem;
    uint8_t *sB = sA + p.nkb * a_box;
    float *epi = reinterpret_cast<float *>(sB + p.nkb * b_box);            // 4 x kEpiTileBytes
    uint64_t *bars = reinterpret_cast<uint64_t *>(sB + p.nkb * b_box + 4 * kEpiTileBytes); // [0] loads, [1] MMAs
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
        // loaded after the TMEM allocation and the block barrier: issuing them
        // first measured slower (BF16 64^3 x 4096: 37.8 against 31.6 us)
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
            if (p.a_tmem)
                issue_mmas<true>(p, tmem, tc::smem_u32(sA), tc::smem_u32(sB), a_box, b_box);
            else
                issue_mmas<false>(p, tmem, tc::smem_u32(sA), tc::smem_u32(sB), a_box, b_box);
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
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        const int depth = p.part == 3 ? p.P : 1;
        const int osz = g.out_type == KAMI_F32 ? 4 : 2;
        void *Cb = reinterpret_cast<char *>(g.C) + (int64_t)prob * g.sC * osz;
        const int row_base = p.bm == 128 ? warp * 32 : warp * 16;
        float *T = epi + warp * (kEpiTileBytes / 4);
        if (p.store_slots > 0)
        {
            const BulkOut o{g.out_type, g.M, g.N, p.bm, p.bn, depth, p.store_slots};
            epilogue_bulk(o, &tmC, tmem + lane_addr, smem + (size_t)warp * p.store_slots * (p.bm == 128 ? 32 : 16) * 128,
                          row_base, prob);
        }
        else
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
            store_chunk(g, Cb, f, row_base, p.bm == 128 ? 32 : 16, c0, T);
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
// Persistent streaming form (1D mapping) for the streamed regime: a fixed
// grid of CTAs (one per SM; two per SM for 64-90 KB problems, each with one
// slot) walks problems blockIdx.x, blockIdx.x + grid, ...
// with three warp roles so that loads, MMAs and the epilogue of different
// problems overlap:
//   warp 0 (one lane)  TMA producer: a ring of `stages` shared-memory slots,
//                      each holding one problem's A and B;
//   warp 1 (one lane)  MMA issuer: a ring of `naccs` TMEM accumulators (as
//                      many as 512 columns hold, at most 8), commits free the
//                      slot and publish the accumulator; for problems of
//                      16-32 KB of operands a second issuer (the last warp)
//                      takes the odd problems, because one thread's issue,
//                      commit and barrier work (~1k cycles per 64^3 problem)
//                      bounds the rate -- only with an even number of slots
//                      and of accumulators, so that every slot and
//                      accumulator belongs to one issuer, which consumes its
//                      phases in order (shared ones let an issuer wait for a
//                      phase two ahead of the last one completed, which
//                      parity-based waits cannot tell apart);
//   warps 2..          epilogue, `groups` groups of four (two, or four when
//                      shared memory leaves room for their transpose tiles
//                      and naccs >= 4 -- never more groups than accumulators):
//                      group g drains the accumulator of every problem j with
//                      j % groups == g (tcgen05.ld of its TMEM lane quadrant,
//                      coalesced C stores), then releases it -- the epilogue
//                      is the longest phase of a small problem, so several
//                      drain at once.
// Plain stores (alpha 1, beta 0, 16-byte aligned C rows and problems) leave
// through the tensor-store unit: each epilogue warp packs 128 bytes of each of
// its rows into a 128B-swizzled staging box (32 FP32 or 64 16-bit columns)
// and one thread issues the box as a bulk tensor store, so C goes out as
// whole lines while the warp reads the next columns from tensor memory; the
// accumulator is released as soon as its last columns are in registers.
// Every wait is bounded like the per-problem kernel's.
// ---------------------------------------------------------------------------
struct Tc05StreamParams
{
    Tc05Params t;
    int stages;
    int stage_bytes; // A + B of one problem (1024-byte multiple)
    int groups;      // epilogue groups of four warps (2 or 4)
    int naccs;       // TMEM accumulators (2..8)
    int tma_store;   // C written by bulk tensor stores (plain stores only)
    int store_bufs;  // staging boxes per epilogue warp (1 or 2)
    int issuers;     // MMA-issuing threads (2 only with even stages and naccs)
    int pair;        // 64 x 64 problems two per unit: A rows and B rows of problems 2u, 2u + 1
                     // stacked in one 128 x 128 MMA tile, C on the accumulator's diagonal
};

constexpr int kStoreBoxBytes = 4096; // one staging box: up to 32 rows x 128 bytes

constexpr int kStreamMaxGroups = 4;

template <bool BF16>
__global__ void __launch_bounds__(96 + 128 * kStreamMaxGroups, 1) tc05_stream_kernel(const __grid_constant__ CUtensorMap tmA,
                                                             const __grid_constant__ CUtensorMap tmB,
                                                             const __grid_constant__ CUtensorMap tmC,
                                                             const Tc05StreamParams sp)
{
    const Tc05Params &p = sp.t;
    const GemmArgs &g = p.g;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = sp.stages;
    const int a_box = p.bm * 128, b_box = p.bn * 128;
    const int G = sp.groups, NA = sp.naccs;
    // per epilogue warp: a transpose tile (kEpiTileBytes) or store_bufs staging boxes
    const int epi_warp_bytes = sp.tma_store ? sp.store_bufs * kStoreBoxBytes : kEpiTileBytes;
    uint8_t *epi_base = smem + (size_t)S * sp.stage_bytes;
    float *epi = reinterpret_cast<float *>(epi_base);
    uint64_t *full = reinterpret_cast<uint64_t *>(epi_base + 4 * G * epi_warp_bytes);
    uint64_t *empty = full + S;
    uint64_t *tfull = empty + S;   // [NA]
    uint64_t *tempty = tfull + NA; // [NA]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + NA);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // work units: problems, or with sp.pair problem pairs (2u, 2u + 1)
    const int64_t nprob = g.batch;
    const int64_t nunit = sp.pair ? (nprob + 1) / 2 : nprob;
    // one unit's A and B into slot st (the producer thread)
    auto load_slot = [&](int st, int64_t prob) {
        uint8_t *sA = smem + (size_t)st * sp.stage_bytes;
        uint8_t *sB = sA + p.nkb * a_box;
        if (sp.pair)
        {
            // problem 2u + q: its 64 A rows (or MN chunk) and 64 B rows (or MN
            // chunk) at +q * 8 KB inside every 64-element K box
            const int nq = 2 * prob + 1 < nprob ? 2 : 1;
            tc::mbar_expect_tx(&full[st], (uint32_t)(sp.stage_bytes / 2 * nq));
            for (int q = 0; q < nq; ++q)
                for (int kb = 0; kb < p.nkb; ++kb)
                {
                    const int pr = (int)(2 * prob + q);
                    tc::tma_load_3d(sA + kb * a_box + q * 8192, &tmA, &full[st], p.a_mn ? 0 : kb * 64,
                                    p.a_mn ? kb * 64 : 0, pr);
                    tc::tma_load_3d(sB + kb * b_box + q * 8192, &tmB, &full[st], p.b_mn ? 0 : kb * 64,
                                    p.b_mn ? kb * 64 : 0, pr);
                }
            return;
        }
        tc::mbar_expect_tx(&full[st], (uint32_t)sp.stage_bytes);
        for (int kb = 0; kb < p.nkb; ++kb)
        {
            if (p.a_mn)
                for (int mc = 0; mc < p.bm / 64; ++mc)
                    tc::tma_load_3d(sA + kb * a_box + mc * 8192, &tmA, &full[st], mc * 64, kb * 64, (int)prob);
            else
                tc::tma_load_3d(sA + kb * a_box, &tmA, &full[st], kb * 64, 0, (int)prob);
            if (p.b_mn)
                for (int nc = 0; nc < p.bn / 64; ++nc)
                    tc::tma_load_3d(sB + kb * b_box + nc * 8192, &tmB, &full[st], nc * 64, kb * 64, (int)prob);
            else
                tc::tma_load_3d(sB + kb * b_box, &tmB, &full[st], kb * 64, 0, (int)prob);
        }
    };
    int j0 = 0; // problems whose loads thread 0 issued during setup
    if (threadIdx.x == 0)
    {
        for (int i = 0; i < S; ++i)
        {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < NA; ++i)
        {
            tc::mbar_init(&tfull[i], 1);
            tc::mbar_init(&tempty[i], 4);
        }
        tc::fence_mbar_init();
        // every slot is free: the first loads start before the TMEM
        // allocation and the block barrier
        for (int64_t prob = blockIdx.x; prob < nunit && j0 < S; prob += gridDim.x, ++j0)
            load_slot(j0, prob);
    }
    __syncwarp();
    if (warp == 1)
    {
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint64_t limit = p.timeout_ns;

    if (warp == 0)
    {
        if (lane == 0)
        {
            int j = j0;
            for (int64_t prob = blockIdx.x + (int64_t)j0 * gridDim.x; prob < nunit; prob += gridDim.x, ++j)
            {
                const int st = j % S;
                if (j >= S && !tc::mbar_wait_bounded(&empty[st], ((j / S) - 1) & 1, limit))
                {
                    tc05_flag(5);
                    break;
                }
                load_slot(st, prob);
            }
            // copies of the last slots still in flight complete before exit
            const int jn = j;
            for (int k = (jn > S ? jn - S : 0); k < jn; ++k)
                tc::mbar_wait_bounded(&full[k % S], (k / S) & 1, limit);
        }
    }
    else if (warp == 1 || (sp.issuers == 2 && warp == 2 + 4 * G))
    {
        // issuer t takes the problems j with j % issuers == t
        const int t = warp == 1 ? 0 : 1;
        if (lane == 0)
        {
            int j = t;
            for (int64_t prob = blockIdx.x + (int64_t)t * gridDim.x; prob < nunit;
                 prob += (int64_t)sp.issuers * gridDim.x, j += sp.issuers)
            {
                const int st = j % S, b = j % NA;
                if (!tc::mbar_wait_bounded(&full[st], (j / S) & 1, limit))
                {
                    tc05_flag(6);
                    break;
                }
                if (j >= NA && !tc::mbar_wait_bounded(&tempty[b], ((j / NA) - 1) & 1, limit))
                {
                    tc05_flag(7);
                    break;
                }
                tc::tc_fence_after();
                const uint32_t a0 = tc::smem_u32(smem + (size_t)st * sp.stage_bytes);
                const uint32_t b0 = a0 + p.nkb * a_box;
                const uint32_t acc_base = tmem + (uint32_t)(b * p.bn);
                const uint64_t a_in = p.a_mn ? 128 : 2, b_in = p.b_mn ? 128 : 2;
                const uint64_t a_wrap = (uint64_t)(a_box >> 4) - 3 * a_in, b_wrap = (uint64_t)(b_box >> 4) - 3 * b_in;
                for (int it = 0; it < g.num_iter; ++it)
                {
                    uint64_t ad = kdesc(a0, a_box, p.a_mn, 0), bd = kdesc(b0, b_box, p.b_mn, 0);
                    for (int ks = 0; ks < p.ksteps; ++ks)
                    {
                        tc::mma_f16_ss(acc_base, ad, bd, p.idesc, (it > 0 || ks > 0) ? 1u : 0u);
                        const bool wrap = (ks & 3) == 3;
                        ad += wrap ? a_wrap : a_in;
                        bd += wrap ? b_wrap : b_in;
                    }
                }
                tc::mma_commit(&empty[st]);
                tc::mma_commit(&tfull[b]);
            }
        }
    }
    else if (warp < 2 + 4 * G)
    {
        // epilogue group g = warps 2+4g .. 5+4g, covering TMEM lane quadrants
        // 2, 3, 0, 1
        const int quad = warp & 3;
        const int grp = (warp - 2) >> 2;
        // with pairs, quadrants 0-1 hold problem 2u's rows, 2-3 problem 2u + 1's,
        // whose columns are the accumulator's 64..127
        const int pq = sp.pair ? quad >> 1 : 0;
        const int row_base = sp.pair ? (quad & 1) * 32 : p.bm == 128 ? quad * 32 : quad * 16;
        const int ucols = sp.pair ? 64 : p.bn;     // accumulator columns of this warp's problem
        const uint32_t ucol0 = (uint32_t)(pq * 64); // and the first of them
        const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
        const int osz = g.out_type == KAMI_F32 ? 4 : 2;
        float *T = epi + (warp - 2) * (kEpiTileBytes / 4);
        int j = grp;
        if (sp.tma_store)
        {
            const int rows = p.bm == 128 ? 32 : 16;   // accumulator rows this warp holds
            const int bcols = 128 / osz;              // columns of one staging box
            const bool f32 = g.out_type == KAMI_F32, bf = g.out_type == KAMI_BF16;
            uint8_t *stg = epi_base + (size_t)(warp - 2) * sp.store_bufs * kStoreBoxBytes;
            int nb = 0;
            for (int64_t unit = blockIdx.x + (int64_t)grp * gridDim.x; unit < nunit;
                 unit += (int64_t)G * gridDim.x, j += G)
            {
                const int64_t prob = sp.pair ? 2 * unit + pq : unit;
                const int b = j % NA;
                const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&tfull[b], (j / NA) & 1, limit));
                if (!ok)
                {
                    tc05_flag(8);
                    break;
                }
                tc::tc_fence_after();
                for (int c0 = 0; c0 < ucols; c0 += bcols)
                {
                    // this thread's 128 bytes of row (row_base + lane), columns c0..c0+bcols-1
                    uint32_t w[32];
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                    {
                        uint32_t v[16], u[16];
                        const uint32_t col = tmem + lane_addr + (uint32_t)(b * p.bn + c0) + ucol0;
                        if (f32)
                        {
                            tc::tmem_ld16(col + 16 * h, v);
                            tc::tmem_ld_wait();
#pragma unroll
                            for (int e = 0; e < 16; ++e)
                                w[16 * h + e] = v[e];
                        }
                        else
                        {
                            tc::tmem_ld16(col + 32 * h, v);
                            tc::tmem_ld16(col + 32 * h + 16, u);
                            tc::tmem_ld_wait();
#pragma unroll
                            for (int e = 0; e < 8; ++e)
                            {
                                w[16 * h + e] = pack2(__uint_as_float(v[2 * e]), __uint_as_float(v[2 * e + 1]), bf);
                                w[16 * h + 8 + e] = pack2(__uint_as_float(u[2 * e]), __uint_as_float(u[2 * e + 1]), bf);
                            }
                        }
                    }
                    if (c0 + bcols >= ucols)
                    {
                        // the accumulator's last columns are in registers: free it
                        tc::tc_fence_before();
                        __syncwarp();
                        if (lane == 0)
                            tc::mbar_arrive(&tempty[b]);
                    }
                    uint8_t *box = stg + (nb % sp.store_bufs) * kStoreBoxBytes;
                    // the box's previous bulk store has finished reading it
                    if (lane == 0)
                    {
                        if (sp.store_bufs == 2)
                            tc::bulk_wait_read<1>();
                        else
                            tc::bulk_wait_read<0>();
                    }
                    __syncwarp();
                    if (lane < rows)
                    {
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            *reinterpret_cast<uint4 *>(box + lane * 128 + ((q ^ (lane & 7)) << 4)) =
                                make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
                    }
                    tc::fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0)
                    {
                        if (row_base < g.M && c0 < g.N && prob < nprob)
                            tc::tma_store_3d(&tmC, box, c0, row_base, (int)prob);
                        tc::bulk_commit();
                    }
                    ++nb;
                }
            }
            if (lane == 0)
                tc::bulk_wait_all();
        }
        else
        for (int64_t unit = blockIdx.x + (int64_t)grp * gridDim.x; unit < nunit;
             unit += (int64_t)G * gridDim.x, j += G)
        {
            const int64_t prob = sp.pair ? 2 * unit + pq : unit;
            const int b = j % NA;
            const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&tfull[b], (j / NA) & 1, limit));
            if (!ok)
            {
                tc05_flag(8);
                break;
            }
            tc::tc_fence_after();
            void *Cb = reinterpret_cast<char *>(g.C) + prob * g.sC * osz;
            for (int c0 = 0; c0 < ucols; c0 += 16)
            {
                uint32_t v[16];
                tc::tmem_ld16(tmem + lane_addr + (uint32_t)(b * p.bn + c0) + ucol0, v);
                tc::tmem_ld_wait();
                float f[16];
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    f[e] = __uint_as_float(v[e]);
                if (prob < nprob)
                    store_chunk(g, Cb, f, row_base, p.bm == 128 ? 32 : 16, c0, T);
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0)
                tc::mbar_arrive(&tempty[b]);
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1)
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

// Encoded maps of the last few requests, per host thread: a training loop
// asks for the same maps call after call (the caching allocator hands back
// the same buffers), and a hit skips the driver's encoding.
struct MapKey
{
    const void *base;
    cuuint64_t dims[3], strides[2];
    cuuint32_t box[3];
    int dt, rank, swizzle, l2, oob;
};

static CUresult encode_cached(CUtensorMap *map, CUtensorMapDataType dt, cuuint32_t rank, void *base,
                              const cuuint64_t *dims, const cuuint64_t *strides, const cuuint32_t *box,
                              CUtensorMapSwizzle swizzle, CUtensorMapL2promotion l2, CUtensorMapFloatOOBfill oob)
{
    struct Entry
    {
        MapKey k;
        CUtensorMap m;
        bool used;
    };
    thread_local Entry cache[8];
    thread_local int next = 0;
    if (rank > 3)
        return CUDA_ERROR_INVALID_VALUE;
    MapKey k;
    memset(&k, 0, sizeof(k));
    k.base = base;
    for (cuuint32_t i = 0; i < rank; ++i)
    {
        k.dims[i] = dims[i];
        k.box[i] = box[i];
        if (i + 1 < rank)
            k.strides[i] = strides[i];
    }
    k.dt = (int)dt;
    k.rank = (int)rank;
    k.swizzle = (int)swizzle;
    k.l2 = (int)l2;
    k.oob = (int)oob;
    for (int i = 0; i < 8; ++i)
        if (cache[i].used && memcmp(&cache[i].k, &k, sizeof(k)) == 0)
        {
            *map = cache[i].m;
            return CUDA_SUCCESS;
        }
    EncodeTiledFn fn = encode_fn();
    if (!fn)
        return CUDA_ERROR_NOT_SUPPORTED;
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = fn(map, dt, rank, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, l2, oob);
    if (r == CUDA_SUCCESS)
    {
        cache[next].k = k;
        cache[next].m = *map;
        cache[next].used = true;
        next = (next + 1) & 7;
    }
    return r;
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
        CUresult r = encode_cached(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                                   const_cast<void *>(base), dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
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
    CUresult r = encode_cached(map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                               const_cast<void *>(base), dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
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

static size_t smem_bytes(int bm, int bn, int nkb)
{
    return (size_t)nkb * (bm + bn) * 128 + 4 * kEpiTileBytes + 1024 + 64;
}

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
    Tc05Shape s{};
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

// Tensor map of an output for the bulk-store epilogue: boxes of 128 bytes x
// box_rows rows of one problem, 128B-swizzled.  False when the output does not
// qualify (plain stores of FP32 / FP16 / BF16 with 16-byte aligned rows and
// problems, the accumulator width bn a whole number of boxes) or the encoding
// fails.
static bool make_store_map(CUtensorMap *map, int out_type, void *C, int N, int M, int64_t batch, int64_t ldc,
                           int64_t sC, int bn, int box_rows)
{
    if (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return false;
    const int osz = out_type == KAMI_F32 ? 4 : 2;
    const int64_t s2 = batch > 1 ? sC : (int64_t)M * ldc;
    if ((reinterpret_cast<uintptr_t>(C) & 15) || (ldc * osz) % 16 || s2 <= 0 || (s2 * osz) % 16 || bn % (128 / osz))
        return false;
    cuuint64_t dims[3] = {(cuuint64_t)N, (cuuint64_t)M, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)(ldc * osz), (cuuint64_t)(s2 * osz)};
    cuuint32_t box[3] = {(cuuint32_t)(128 / osz), (cuuint32_t)box_rows, 1};
    const CUtensorMapDataType dt = out_type == KAMI_F32    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : out_type == KAMI_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                           : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    return encode_cached(map, dt, 3, C, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C of a batched GEMM: bulk stores only for alpha 1, beta 0
static bool make_c_map(CUtensorMap *map, const GemmArgs &g, int bn, int box_rows)
{
    if (g.alpha != 1.0 || g.beta != 0.0)
        return false;
    return make_store_map(map, g.out_type, g.C, g.N, g.M, g.batch, g.ldc, g.sC, bn, box_rows);
}

// Launch the persistent streaming form: one CTA per SM, as many ring slots
// as shared memory holds (2..6), and as many TMEM accumulators as 512
// columns hold (at most 8) -- except for 64-90 KB problems with bulk-store
// epilogues: two CTAs per SM, each with one slot, one epilogue group, one
// staging box per warp and two accumulators.  With bulk tensor stores: two epilogue groups,
// two staging boxes per warp when three slots still fit beside them (else
// one).  Otherwise four epilogue groups when at least three slots still fit
// beside their transpose tiles and there are at least four accumulators
// (else two).  A second MMA issuer for problems under 32 KB when slots and
// accumulators are both even; need_two: launch nothing (KAMI_ERR_UNSUPPORTED,
// no message) when that layout is not possible.
static int stream_launch(CUtensorMap &ma, CUtensorMap &mb, Tc05Params &p, bool bf16, cudaStream_t stream,
                         bool need_two, bool pair = false)
{
    Tc05StreamParams sp{};
    if (pair)
    {
        // two 64 x 64 problems per unit: one M = 128, N = 128 MMA chain whose
        // diagonal 64 x 64 blocks are the two C (the off-diagonal blocks cost
        // tensor time the streamed regime has to spare and are never read)
        p.bm = 128;
        p.bn = 128;
        p.idesc = tc::idesc_f16(bf16, 128, 128, p.a_mn, p.b_mn);
        sp.pair = 1;
    }
    sp.t = p;
    sp.stage_bytes = p.nkb * (p.bm + p.bn) * 128;
    CUtensorMap mc = ma;
    sp.tma_store = make_c_map(&mc, p.g, p.bn, p.bm == 128 ? 32 : 16);
    // accumulators: at least as many as epilogue groups.  Group j % groups
    // drains problem j from accumulator j % naccs; with fewer accumulators the
    // next user of an accumulator belongs to a group whose previous problem
    // is older, which can reach its wait while the accumulator's current phase
    // is still open -- a parity wait for the phase after it passes at once.
    sp.naccs = std::min(8, 512 / p.bn);
    int budget;
    if (sp.tma_store)
    {
        sp.groups = 2;
        sp.store_bufs = 2;
        budget = 227 * 1024 - 1024 - 512 - 4 * sp.groups * sp.store_bufs * kStoreBoxBytes;
        if (budget / sp.stage_bytes < 3)
        {
            sp.store_bufs = 1;
            budget = 227 * 1024 - 1024 - 512 - 4 * sp.groups * sp.store_bufs * kStoreBoxBytes;
        }
    }
    else
    {
        sp.groups = kStreamMaxGroups;
        budget = 227 * 1024 - 1024 - 512 - 4 * sp.groups * kEpiTileBytes;
        if (budget / sp.stage_bytes < 3 || sp.naccs < sp.groups)
        {
            sp.groups = 2;
            budget = 227 * 1024 - 1024 - 512 - 4 * sp.groups * kEpiTileBytes;
        }
    }
    sp.stages = std::min(6, budget / sp.stage_bytes);
    // problems of 64-90 KB (128 x 128 x 128 in 16-bit types) with bulk-store
    // epilogues: two CTAs per SM, each with one stage, one epilogue group and
    // two accumulators (256 TMEM columns), rather than one CTA with three
    // stages -- two independent load -> MMA -> epilogue chains per SM
    // (FP16 128^3 x 592, FP32 C: 16.2 against 17.2 us; BF16 x 2048: 32.6
    // against 33.7 us)
    int per_sm = 1;
    if (sp.tma_store && !pair && sp.stage_bytes >= 65536 && sp.stage_bytes <= 90 * 1024)
    {
        sp.stages = 1;
        sp.groups = 1;
        sp.store_bufs = 1;
        sp.naccs = 2;
        per_sm = 2;
    }
    else if (sp.stages < 2)
        return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 streaming form: a problem needs %d bytes of shared memory",
                    sp.stage_bytes);
    uint32_t cols = 32;
    while ((int)cols < sp.naccs * p.bn)
        cols <<= 1;
    sp.t.tmem_cols = cols;
    sp.t.timeout_ns = p.timeout_ns + 500000000ull;
    const size_t epi = sp.tma_store ? (size_t)4 * sp.groups * sp.store_bufs * kStoreBoxBytes
                                    : (size_t)4 * sp.groups * kEpiTileBytes;
    const size_t smem = (size_t)sp.stages * sp.stage_bytes + epi + 1024 + 512;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void *fn = bf16 ? (const void *)&tc05_stream_kernel<true> : (const void *)&tc05_stream_kernel<false>;
    static std::once_flag once[2];
    cudaError_t e = cudaSuccess;
    std::call_once(once[bf16 ? 1 : 0],
                   [&] { e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024); });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(tc05_stream_kernel)");
    const int64_t grid = std::min<int64_t>(pair ? (p.g.batch + 1) / 2 : p.g.batch, (int64_t)sms * per_sm);
    sp.issuers = sp.stage_bytes < 32768 && sp.stages % 2 == 0 && sp.naccs % 2 == 0 ? 2 : 1;
    if (need_two && sp.issuers != 2)
        return KAMI_ERR_UNSUPPORTED; // nothing launched: the caller runs one CTA per problem
    void *args[] = {&ma, &mb, &mc, &sp};
    e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(64 + 128 * sp.groups + 32 * (sp.issuers - 1)), args, smem,
                         stream);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(tc05_stream_kernel)");
    return KAMI_OK;
}

int tc05_launch(const GemmArgs &g, int in_type, int partition, int P, void *, size_t, cudaStream_t stream,
                int a_tmem)
{
    Tc05Shape s{};
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

    // Streamed regime: the persistent form for problems of >= 32 KB of operands
    // (measured on B200: 128^3 x 592 121 vs 105 TFLOP/s, x 8192 190 vs 150),
    // and for 16-32 KB when it runs two MMA issuers (an even number of
    // accumulators; the six slots it gets are even): BF16 64^3 x 4096 28.7
    // against 31.6 us one CTA per problem, FP16 64^3 x 8192 with FP32 C 51.3
    // against 52.2 us (with one issuer 32.6 and 55.3).
    const int stage_bytes = s.nkb * (s.bm + s.bn) * 128;
    // 64 x 64 problems stream two to a unit (one 128 x 128 MMA chain, half the
    // issue, commit and hand-off work per problem)
    if (s.part == KAMI_PARTITION_1D && !s.a_tmem && g.num_iter <= 4 && s.bm == 64 && s.bn == 64 && g.M == 64 &&
        g.N == 64 && g.batch >= 2 && 4 * stage_bytes <= 227 * 1024 - 1024 - 512 - 8 * kEpiTileBytes)
        return stream_launch(ma, mb, p, bf16, stream, false, true);
    if (s.part == KAMI_PARTITION_1D && !s.a_tmem && g.num_iter <= 4 && stage_bytes >= 16384 &&
        2 * stage_bytes <= 227 * 1024 - 1024 - 512 - 8 * kEpiTileBytes)
    {
        const bool small = stage_bytes < 32768;
        st = stream_launch(ma, mb, p, bf16, stream, small);
        if (!small || st != KAMI_ERR_UNSUPPORTED)
            return st;
    }

    // bulk C stores staged in the operand tiles and transpose tiles (dead
    // after the MMAs): as many boxes per warp as they hold, up to all of them
    CUtensorMap mc = ma;
    const int rows = s.bm == 128 ? 32 : 16;
    if (make_c_map(&mc, g, s.bn, rows))
    {
        const int boxes = s.bn / (g.out_type == KAMI_F32 ? 32 : 64);
        const int region = s.nkb * ((s.a_tmem ? 0 : s.bm) + s.bn) * 128 + 4 * kEpiTileBytes;
        p.store_slots = std::min(boxes, region / (4 * rows * 128));
    }
    const void *fn = bf16 ? (const void *)&tc05_block_kernel<true> : (const void *)&tc05_block_kernel<false>;
    static std::once_flag once[2];
    cudaError_t e = cudaSuccess;
    std::call_once(once[bf16 ? 1 : 0], [&] {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(tc05_block_kernel)");
    // one CTA per SM on request: more than half of the SM's shared memory
    int smem = (int)s.smem;
    if (g.one_per_sm)
    {
        static int per_sm = 0;
        if (!per_sm)
        {
            int dev = 0;
            cudaGetDevice(&dev);
            if (cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
                per_sm = 228 * 1024;
        }
        smem = std::max(smem, std::min(per_sm / 2 + 1024, 227 * 1024));
    }
    void *args[] = {&ma, &mb, &mc, &p};
    e = cudaLaunchKernel(fn, dim3((unsigned)g.batch), dim3(128), args, smem, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(tc05_block_kernel)");
    return KAMI_OK;
}

// ---------------------------------------------------------------------------
// Fused backward of C = A B (A: M x K, B: K x N, C: M x N, row-major -- the
// torch.bmm layout) for M, N, K in {64, 128}: one CTA per problem loads dC,
// A and B once by TMA (64-column boxes, 128-byte swizzle) and runs both
// gradients from the same shared-memory tiles:
//   dA = dC B^T   (M x K): dC as the K-major A operand (rows m, K = n) and B
//                  as the K-major B operand (rows k, K = n);
//   dB = A^T dC   (K x N): A as the MN-major A operand (K = m rows of 64
//                  k-elements) and dC as the MN-major B operand (K = m rows
//                  of 64 n-elements) -- a row-major tile with 64-column boxes
//                  is both the K-major view of one product and the MN-major
//                  view of the other.
// The two accumulators sit side by side in TMEM (columns 0..K-1 and
// K..K+N-1); the four warps drain dA, then dB.  Waits are bounded as in the
// forward kernels.
// ---------------------------------------------------------------------------
struct Tc05BwdParams
{
    int M, N, K;
    int64_t batch;
    void *dA, *dB; // either may be null
    int out_type;
    uint32_t idesc_a, idesc_b; // dA: M x K (K-major, K-major); dB: K x N (MN-major, MN-major)
    uint32_t tmem_cols;
    uint64_t timeout_ns;
    int slots_a, slots_b;      // staging boxes per warp for bulk stores of dA / dB (0: per-thread stores)
    int pair;                  // M = N = K = 64: problems 2c, 2c + 1 in CTA c, stacked in 128-row tiles
};

template <bool BF16>
__global__ void __launch_bounds__(128) tc05_bwd_kernel(const __grid_constant__ CUtensorMap tmG,
                                                       const __grid_constant__ CUtensorMap tmA,
                                                       const __grid_constant__ CUtensorMap tmB,
                                                       const __grid_constant__ CUtensorMap tmDA,
                                                       const __grid_constant__ CUtensorMap tmDB,
                                                       const Tc05BwdParams p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int M = p.M, N = p.N, K = p.K;
    // with p.pair (64^3): two problems, each region holding problem 0's box
    // then problem 1's, i.e. 128-row tiles of the stacked problems
    const int np = p.pair ? 2 : 1;
    uint8_t *sG = smem;                               // dC: N / 64 boxes of M rows x 128 B (x np)
    uint8_t *sA = sG + (size_t)np * M * N * 2;        // A:  K / 64 boxes of M rows (x np)
    uint8_t *sB = sA + (size_t)np * M * K * 2;        // B:  N / 64 boxes of K rows (x np)
    float *epi = reinterpret_cast<float *>(sB + (size_t)np * K * N * 2);
    uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<uint8_t *>(epi) + 4 * kEpiTileBytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
    int *ok_slot = reinterpret_cast<int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5;
    // this warp's problem: with pairs, warps 0-1 hold problem 2c's rows and
    // warps 2-3 problem 2c + 1's (M = 128 accumulator rows)
    const int wq = p.pair ? warp >> 1 : 0;
    const int prob = p.pair ? 2 * blockIdx.x + wq : blockIdx.x;
    const int nq = p.pair && 2 * (int64_t)blockIdx.x + 1 < p.batch ? 2 : 1; // problems present

    if (threadIdx.x == 0)
    {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
        tc::fence_mbar_init();
        *ok_slot = 1;
        tc::prefetch_tmap(&tmG);
        tc::prefetch_tmap(&tmA);
        tc::prefetch_tmap(&tmB);
        tc::mbar_expect_tx(&bars[0], (uint32_t)((M * N + M * K + K * N) * 2 * nq));
        for (int q = 0; q < nq; ++q)
        {
            const int pr = (p.pair ? 2 * blockIdx.x : blockIdx.x) + q;
            const size_t o = (size_t)q * 64 * 128; // pairs: 64^3, one box per operand per problem
            for (int b = 0; b < N / 64; ++b)
                tc::tma_load_3d(sG + o + (size_t)b * M * 128, &tmG, &bars[0], b * 64, 0, pr);
            for (int b = 0; b < K / 64; ++b)
                tc::tma_load_3d(sA + o + (size_t)b * M * 128, &tmA, &bars[0], b * 64, 0, pr);
            for (int b = 0; b < N / 64; ++b)
                tc::tma_load_3d(sB + o + (size_t)b * K * 128, &tmB, &bars[0], b * 64, 0, pr);
        }
    }
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
            const uint32_t g0 = tc::smem_u32(sG), a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            if (p.dA)
            {
                // dA = dC B^T: K-major operands, k-step of 16 n = +32 B, next
                // 64-column box after 4 steps
                for (int ks = 0; ks < N / 16; ++ks)
                {
                    const uint32_t ga = g0 + (uint32_t)((ks >> 2) * M * 128 + (ks & 3) * 32);
                    const uint32_t bb = b0 + (uint32_t)((ks >> 2) * K * 128 + (ks & 3) * 32);
                    tc::mma_f16_ss(tmem, tc::desc_kmajor_sw128(ga), tc::desc_kmajor_sw128(bb), p.idesc_a,
                                   ks > 0 ? 1u : 0u);
                }
            }
            if (p.dB)
            {
                // dB = A^T dC: MN-major operands, k-step of 16 m-rows = +2 KB,
                // the next 64-element MN chunk one box (M rows) away (with
                // pairs: the other problem's chunk, its own m rows)
                for (int ks = 0; ks < M / 16; ++ks)
                    tc::mma_f16_ss(tmem + (uint32_t)(np * K), tc::desc_mnmajor_sw128(a0 + ks * 2048, (uint32_t)M * 128),
                                   tc::desc_mnmajor_sw128(g0 + ks * 2048, (uint32_t)M * 128), p.idesc_b,
                                   ks > 0 ? 1u : 0u);
            }
            tc::mma_commit(&bars[1]);
        }
    }
    __syncwarp();

    const bool done_w = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&bars[1], 0, p.timeout_ns));
    tc::tc_fence_after();
    if (!done_w)
        tc05_flag(2);
    // block-uniform outcome: the epilogue below holds a block barrier
    const bool done = __syncthreads_and(done_w);
    const bool ok = done && *reinterpret_cast<volatile int *>(ok_slot);
    if (ok)
    {
        const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
        const int osz = p.out_type == KAMI_F32 ? 4 : 2;
        float *T = epi + warp * (kEpiTileBytes / 4);
        for (int which = 0; which < 2; ++which)
        {
            void *out = which == 0 ? p.dA : p.dB;
            if (!out)
                continue;
            const int rows = which == 0 ? M : K, cols = which == 0 ? K : N;
            // accumulator columns of this warp's problem: dA then dB, each np
            // problems wide (a pair's diagonal blocks)
            const uint32_t col0 = (which == 0 ? 0u : (uint32_t)(np * K)) + (uint32_t)(wq * cols);
            const bool here = wq < nq; // a pair's second problem may be absent
            GemmArgs g{};
            g.M = here ? rows : 0;
            g.N = cols;
            g.ldc = cols;
            g.out_type = p.out_type;
            g.c_vec = 1;
            g.c_vec4 = 1;
            g.alpha = 1.0;
            g.beta = 0.0;
            void *Cb = reinterpret_cast<char *>(out) + (int64_t)(here ? prob : 0) * rows * cols * osz;
            const int row_base = p.pair ? (warp & 1) * 32 : rows == 128 ? warp * 32 : warp * 16;
            const int wrows = p.pair || rows == 128 ? 32 : 16; // accumulator rows this warp holds
            const int slots = which == 0 ? p.slots_a : p.slots_b;
            // dB's staging (or transpose tiles) may overlap boxes of another
            // warp's dA stores: every warp's dA boxes have been read first
            // (each warp waits for its own stores at the end of its pass)
            if (which == 1 && p.dA && p.slots_a > 0)
                __syncthreads();
            if (slots > 0)
            {
                // staged in the dC / A / B tiles, dead after the MMAs (an absent
                // problem stages nothing out: rows 0)
                const BulkOut o{p.out_type, here ? rows : 0, cols, wrows == 32 ? 128 : 64, cols, 1, slots};
                epilogue_bulk(o, which == 0 ? &tmDA : &tmDB, tmem + lane_addr + col0,
                              smem + (size_t)warp * slots * wrows * 128, row_base, here ? prob : 0);
                continue;
            }
            for (int c0 = 0; c0 < cols; c0 += 16)
            {
                uint32_t v[16];
                tc::tmem_ld16(tmem + lane_addr + col0 + c0, v);
                tc::tmem_ld_wait();
                float f[16];
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    f[e] = __uint_as_float(v[e]);
                store_chunk(g, Cb, f, row_base, wrows, c0, T);
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

// Launch the fused backward; KAMI_ERR_UNSUPPORTED (nothing launched) outside
// FP16 / BF16 with M, N, K in {64, 128}, packed problems and 16-byte aligned
// buffers.
int tc05_backward_launch(int in_type, int out_type, int M, int N, int K, int64_t batch, const void *A, const void *B,
                         const void *dC, void *dA, void *dB, cudaStream_t stream)
{
    auto dim_ok = [](int x) { return x == 64 || x == 128; };
    if ((in_type != KAMI_F16 && in_type != KAMI_BF16) || !dim_ok(M) || !dim_ok(N) || !dim_ok(K) ||
        (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16) || batch < 1 || batch > 0x7fffffff)
        return KAMI_ERR_UNSUPPORTED;
    auto al = [](const void *q) { return q == nullptr || (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    if (!al(A) || !al(B) || !al(dC) || !al(dA) || !al(dB))
        return KAMI_ERR_UNSUPPORTED;
    const bool bf16 = in_type == KAMI_BF16;
    CUtensorMap mg, ma, mb;
    int st;
    // row-major tiles as {columns, rows, batch} maps with 64-column boxes of all rows
    if ((st = make_map(&mg, bf16, dC, N, M, batch, N, (int64_t)M * N, M)) ||
        (st = make_map(&ma, bf16, A, K, M, batch, K, (int64_t)M * K, M)) ||
        (st = make_map(&mb, bf16, B, N, K, batch, N, (int64_t)K * N, K)))
        return st;
    Tc05BwdParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.batch = batch;
    p.dA = dA;
    p.dB = dB;
    p.out_type = out_type;
    // 64^3 problems two per CTA: both gradients as one 128 x 128 MMA chain each
    // over the stacked problems, the two C on the accumulators' diagonals (the
    // off-diagonal blocks cost tensor time this memory-bound pass has to spare)
    p.pair = M == 64 && N == 64 && K == 64 && batch >= 2;
    const int np = p.pair ? 2 : 1;
    p.idesc_a = tc::idesc_f16(bf16, np * M, np * K, 0, 0);
    p.idesc_b = tc::idesc_f16(bf16, np * K, np * N, 1, 1);
    uint32_t cols = 32;
    while ((int)cols < np * (K + N))
        cols <<= 1;
    p.tmem_cols = cols;
    p.timeout_ns = (uint64_t)(5e8 + (double)(M + N) * 4000.0);
    const size_t smem = (size_t)np * (M * N + M * K + K * N) * 2 + 4 * kEpiTileBytes + 64 + 1024;
    // bulk stores of each gradient, staged in the operand and transpose tiles
    CUtensorMap mda = mg, mdb = mg;
    const int region = np * (M * N + M * K + K * N) * 2 + 4 * kEpiTileBytes;
    const int bcols = out_type == KAMI_F32 ? 32 : 64;
    const int wra = p.pair || M == 128 ? 32 : 16, wrb = p.pair || K == 128 ? 32 : 16; // rows per warp
    if (dA && make_store_map(&mda, out_type, dA, K, M, batch, K, (int64_t)M * K, K, wra))
        p.slots_a = std::min(K / bcols, region / (4 * wra * 128));
    if (dB && make_store_map(&mdb, out_type, dB, N, K, batch, N, (int64_t)K * N, N, wrb))
        p.slots_b = std::min(N / bcols, region / (4 * wrb * 128));
    const void *fn = bf16 ? (const void *)&tc05_bwd_kernel<true> : (const void *)&tc05_bwd_kernel<false>;
    static std::once_flag once[2];
    cudaError_t e = cudaSuccess;
    std::call_once(once[bf16 ? 1 : 0], [&] {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(tc05_bwd_kernel)");
    void *args[] = {&mg, &ma, &mb, &mda, &mdb, &p};
    e = cudaLaunchKernel(fn, dim3((unsigned)(p.pair ? (batch + 1) / 2 : batch)), dim3(128), args, smem, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(tc05_bwd_kernel)");
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
