// grouped.cu -- thousands of independent block GEMMs of uneven M/N/K in ONE
// persistent launch (graph-capturable), with the warp partition chosen per
// problem shape by a measuring autotuner.
//
// The reference launches one kernel per compile-time shape, one problem per
// CTA (batched_gemm_{1d,2d,3d}_double_mma.cu: blockIdx.x = problem, :83-86).
// Here every problem carries its own (M, N, K) and partition, and a fixed
// grid of persistent CTAs (8 warps each) walks a host-built schedule
// (longest-processing-time-first over the CTAs).  Each CTA streams its
// problems through a multi-stage cp.async pipeline of K chunks staged in
// shared memory, so the loads of the next chunk (or the next problem)
// overlap the MMAs of the current one.
//
// Partitions of the 8 warps (R x C x D warp grids, R*C*D = 8), the KAMI
// 1D / 2D / 3D ideas applied to a runtime-sized tile:
//   cfg 0  8x1x1  1D: warps split M (16-row strips), each owns all of N
//   cfg 1  4x2x1  2D
//   cfg 2  2x4x1  2D
//   cfg 3  2x2x2  3D: K steps interleaved over 2 depth ranks (M, N <= 64)
//   cfg 4  1x1x8  3D: 8 depth ranks (M, N <= 32)
//   cfg 5  2x1x4  3D (M <= 64, N <= 32)
//   cfg 6  1x2x4  3D (M <= 32, N <= 64)
//   cfg 7  one warp owns the whole problem (M, N <= 32): after its CTA's
//          share of the larger problems, every warp of the grid takes small
//          problems round-robin and runs them from registers -- all loads of
//          a K chunk issued before its MMAs, no shared memory, no CTA
//          barrier -- so hundreds of tiny problems per SM stream in parallel.
// Depth partials are reduced on the device through shared memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <tuple>
#include <vector>

#include "grouped.cuh"
#include "kami_common.cuh"
#include "mma_engine.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kCfgs = 8; // cfg 7 = single-warp problems
__host__ __device__ constexpr int cfg_R(int c) { return c == 0 ? 8 : c == 1 ? 4 : c == 2 ? 2 : c == 3 ? 2 : c == 4 ? 1 : c == 5 ? 2 : 1; }
__host__ __device__ constexpr int cfg_C(int c) { return c == 0 ? 1 : c == 1 ? 2 : c == 2 ? 4 : c == 3 ? 2 : c == 4 ? 1 : c == 5 ? 1 : 2; }
__host__ __device__ constexpr int cfg_D(int c) { return c <= 2 ? 1 : c == 3 ? 2 : c == 4 ? 8 : 4; }
// register tile (fragment rows x fragment cols) a warp can hold per cfg
__host__ __device__ constexpr int cfg_MI(int c) { return c == 0 ? 1 : c == 1 ? 2 : c == 2 ? 4 : 2; }
__host__ __device__ constexpr int cfg_MJ(int c) { return c == 0 ? 16 : c == 1 ? 8 : c == 2 ? 4 : 4; }

// per-precision pipeline geometry
template <class Tr>
struct GGeom
{
    static constexpr int ES = sizeof(typename Tr::Elem);
    static constexpr int KCH = ES == 2 ? 64 : 32; // K elements per chunk
    static constexpr int PAD = ES == 2 ? 16 : 8;  // row padding (elements) for conflict-free fragment loads
    static constexpr int LD = KCH + PAD;          // smem row stride (elements)
    static constexpr int ROW = LD * ES;           // bytes of one staged row
    static constexpr int RED = kWarps * 8 * 128 * (int)sizeof(typename Tr::Acc); // depth partials
    // byte ring of staged K chunks, each sized by its problem (the largest,
    // 128 + 128 rows, is 40 KB for FP16 and 80 KB for FP64)
    static constexpr int RING = ES == 2 ? 192 * 1024 : 160 * 1024;
    static constexpr int SMEM = RING + RED;
    static constexpr int MAXF = 8; // K chunks in flight at most (cp.async groups)
    // ring bytes of one K chunk of a problem: A rows to a multiple of 16 and B
    // rows to a multiple of 8, the rows the fragment loads touch
    static __host__ __device__ int chunk_bytes(int M, int N) { return (((M + 15) & ~15) + ((N + 7) & ~7)) * ROW; }
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    const int n = valid ? 16 : 0; // src-size 0: zero-fill
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// wait until at most n (< 8) cp.async groups of this thread are pending
__device__ __forceinline__ void cp_async_wait_dyn(int n)
{
    switch (n)
    {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    case 3: cp_async_wait<3>(); break;
    case 4: cp_async_wait<4>(); break;
    case 5: cp_async_wait<5>(); break;
    case 6: cp_async_wait<6>(); break;
    default: cp_async_wait<7>(); break;
    }
}

template <class Tr>
__device__ __forceinline__ void load_chunk(const GroupedParams &p, const GroupedDesc &d, int k0, uint8_t *stage)
{
    using G = GGeom<Tr>;
    using Elem = typename Tr::Elem;
    constexpr int CPR = G::KCH * G::ES / 16; // 16-byte chunks per staged row
    const Elem *A = reinterpret_cast<const Elem *>(p.A) + d.a_off;
    const Elem *B = reinterpret_cast<const Elem *>(p.B) + d.b_off;
    Elem *sA = reinterpret_cast<Elem *>(stage);
    Elem *sB = reinterpret_cast<Elem *>(stage + ((d.M + 15) & ~15) * G::ROW);
    const int epc = 16 / G::ES; // elements per 16-byte chunk
    for (int c = threadIdx.x; c < d.M * CPR; c += kThreads)
    {
        const int r = c / CPR, q = c % CPR;
        const int k = k0 + q * epc;
        const bool v = k < d.K;
        cp_async16(sA + r * G::LD + q * epc, v ? (const void *)(A + (int64_t)r * d.lda + k) : (const void *)A, v);
    }
    for (int c = threadIdx.x; c < d.N * CPR; c += kThreads)
    {
        const int r = c / CPR, q = c % CPR;
        const int k = k0 + q * epc;
        const bool v = k < d.K;
        cp_async16(sB + r * G::LD + q * epc, v ? (const void *)(B + (int64_t)r * d.ldb + k) : (const void *)B, v);
    }
}

struct Tile
{
    int i0, ni, j0, nj, d, D;
};

__device__ __forceinline__ Tile warp_tile(const GroupedDesc &d, int warp)
{
    const int cfg = d.cfg;
    const int R = cfg_R(cfg), C = cfg_C(cfg), D = cfg_D(cfg);
    const int MF = (d.M + 15) >> 4, NF = (d.N + 7) >> 3;
    const int dr = warp % D, c = (warp / D) % C, r = warp / (D * C);
    const int mi = (MF + R - 1) / R, mj = (NF + C - 1) / C;
    Tile t;
    t.i0 = r * mi;
    t.ni = max(0, min(mi, MF - t.i0));
    t.j0 = c * mj;
    t.nj = max(0, min(mj, NF - t.j0));
    t.d = dr;
    t.D = D;
    return t;
}

template <class Tr, int MI, int MJ>
__device__ __forceinline__ void compute_chunk(const GroupedDesc &d, const Tile &t, int k0, const uint8_t *stage,
                                              int num_iter, typename Tr::Acc (&acc)[16][4])
{
    using G = GGeom<Tr>;
    using Unit = typename Tr::Unit;
    using Elem = typename Tr::Elem;
    const Elem *sA = reinterpret_cast<const Elem *>(stage);
    const Elem *sB = reinterpret_cast<const Elem *>(stage + ((d.M + 15) & ~15) * G::ROW);
    const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
    const int kin = min(G::KCH, d.K - k0);
    const int ksteps = (kin + Tr::KSTEP - 1) / Tr::KSTEP;
    const int lane_k = tq * 2 * Tr::EPU;
    if (t.ni <= 0 || t.nj <= 0)
        return;
    for (int it = 0; it < num_iter; ++it)
        for (int ks = t.d; ks < ksteps; ks += t.D)
        {
            const int kk = ks * Tr::KSTEP + lane_k;
            Unit a[MI][4];
#pragma unroll
            for (int ii = 0; ii < MI; ++ii)
                if (ii < t.ni)
                {
                    const int r = (t.i0 + ii) * 16 + gq;
                    Tr::ld2_smem(sA + r * G::LD + kk, a[ii][0], a[ii][2]);
                    Tr::ld2_smem(sA + (r + 8) * G::LD + kk, a[ii][1], a[ii][3]);
                }
            // B fragments one at a time: only the A fragments and one B
            // fragment are live next to the accumulators
#pragma unroll
            for (int jj = 0; jj < MJ; ++jj)
                if (jj < t.nj)
                {
                    Unit b0, b1;
                    const int n = (t.j0 + jj) * 8 + gq;
                    Tr::ld2_smem(sB + n * G::LD + kk, b0, b1);
#pragma unroll
                    for (int ii = 0; ii < MI; ++ii)
                        if (ii < t.ni)
                            Tr::mma(acc[ii * MJ + jj], a[ii], b0, b1);
                }
        }
}

template <class Acc>
__device__ __forceinline__ void gstore_pair(const GroupedParams &p, const GroupedDesc &d, int r, int c, Acc v0,
                                            Acc v1)
{
    GemmArgs g{};
    g.M = d.M;
    g.N = d.N;
    g.ldc = d.ldc;
    g.out_type = p.out_type;
    g.c_vec = ((d.ldc & 1) == 0) && ((d.c_off & 1) == 0); // the C base is 16-byte aligned (host-checked)
    g.alpha = p.alpha;
    g.beta = p.beta;
    const int osz = p.out_type == KAMI_F64 ? 8 : p.out_type == KAMI_F32 ? 4 : 2;
    void *Cb = reinterpret_cast<char *>(p.C) + d.c_off * osz;
    store_pair<Acc>(g, Cb, r, c, v0, v1);
}

template <class Tr, int MI, int MJ>
__device__ __forceinline__ void finish_problem(const GroupedParams &p, const GroupedDesc &d, const Tile &t,
                                               uint8_t *red_raw, typename Tr::Acc (&acc)[16][4])
{
    using Acc = typename Tr::Acc;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (t.D > 1)
    {
        // depth ranks d > 0 leave their partials; rank 0 of each (r, c) sums
        Acc *red = reinterpret_cast<Acc *>(red_raw);
        if (t.d > 0)
        {
            Acc *dst = red + (size_t)warp * (MI * MJ * 128) + lane * 4;
#pragma unroll
            for (int ii = 0; ii < MI; ++ii)
#pragma unroll
                for (int jj = 0; jj < MJ; ++jj)
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        dst[(ii * MJ + jj) * 128 + e] = acc[ii * MJ + jj][e];
        }
        __syncthreads();
        if (t.d == 0)
        {
            for (int dd = 1; dd < t.D; ++dd)
            {
                const Acc *src = red + (size_t)(warp + dd) * (MI * MJ * 128) + lane * 4;
#pragma unroll
                for (int ii = 0; ii < MI; ++ii)
#pragma unroll
                    for (int jj = 0; jj < MJ; ++jj)
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            acc[ii * MJ + jj][e] += src[(ii * MJ + jj) * 128 + e];
            }
        }
    }
    if (t.d == 0)
    {
        const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
        for (int ii = 0; ii < MI; ++ii)
#pragma unroll
            for (int jj = 0; jj < MJ; ++jj)
                if (ii < t.ni && jj < t.nj)
                {
                    const int r = (t.i0 + ii) * 16 + gq, c = (t.j0 + jj) * 8 + 2 * tq;
                    gstore_pair<Acc>(p, d, r, c, acc[ii * MJ + jj][0], acc[ii * MJ + jj][1]);
                    gstore_pair<Acc>(p, d, r + 8, c, acc[ii * MJ + jj][2], acc[ii * MJ + jj][3]);
                }
    }
}

template <class Tr, int MI, int MJ>
__device__ __forceinline__ void run_chunk(const GroupedParams &p, const GroupedDesc &d, int k0, bool first,
                                          bool last, const uint8_t *stage, uint8_t *red,
                                          typename Tr::Acc (&acc)[16][4])
{
    static_assert(MI * MJ <= 16, "register tile");
    const Tile t = warp_tile(d, threadIdx.x >> 5);
    if (first)
    {
#pragma unroll
        for (int f = 0; f < 16; ++f)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                acc[f][e] = 0;
    }
    compute_chunk<Tr, MI, MJ>(d, t, k0, stage, p.num_iter, acc);
    if (last)
        finish_problem<Tr, MI, MJ>(p, d, t, red, acc);
}

// One warp computes one small problem (M, N <= 32) from registers.
template <class Tr>
__device__ __forceinline__ void warp_problem(const GroupedParams &p, const GroupedDesc &d)
{
    using Unit = typename Tr::Unit;
    using Acc = typename Tr::Acc;
    using Elem = typename Tr::Elem;
    constexpr int KC = Tr::EPU == 2 ? 8 : 4; // resident k-steps per chunk (K <= 128 in one chunk for FP16)
    const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
    GemmArgs g{};
    g.M = d.M;
    g.N = d.N;
    g.K = d.K;
    g.lda = d.lda;
    g.ldb = d.ldb;
    g.a_layout = KAMI_A_ROW_MK;
    g.b_layout = KAMI_B_REF_NK;
    const Elem *A = reinterpret_cast<const Elem *>(p.A) + d.a_off;
    const Elem *B = reinterpret_cast<const Elem *>(p.B) + d.b_off;
    const int MF = (d.M + 15) >> 4, NF = (d.N + 7) >> 3;
    const int lane_k = tq * 2 * Tr::EPU;
    Acc acc[2][4][4];
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                acc[ii][jj][e] = Acc(0);
    for (int k0 = 0; k0 < d.K; k0 += KC * Tr::KSTEP)
    {
        Unit a[2][KC][4], b[4][KC][2];
#pragma unroll
        for (int ii = 0; ii < 2; ++ii)
#pragma unroll
            for (int kk = 0; kk < KC; ++kk)
                load_a_frag<Tr>(g, A, (ii < MF ? ii * 16 : 1 << 20) + gq, k0 + kk * Tr::KSTEP + lane_k, a[ii][kk]);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
#pragma unroll
            for (int kk = 0; kk < KC; ++kk)
                load_b_frag<Tr>(g, B, (jj < NF ? jj * 8 : 1 << 20) + gq, k0 + kk * Tr::KSTEP + lane_k, b[jj][kk]);
        for (int it = 0; it < p.num_iter; ++it)
#pragma unroll
            for (int kk = 0; kk < KC; ++kk)
                if (k0 + kk * Tr::KSTEP < d.K)
#pragma unroll
                    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj)
                            if (ii < MF && jj < NF)
                                Tr::mma(acc[ii][jj], a[ii][kk], b[jj][kk][0], b[jj][kk][1]);
    }
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
            if (ii < MF && jj < NF)
            {
                const int r = ii * 16 + gq, c = jj * 8 + 2 * tq;
                gstore_pair<Acc>(p, d, r, c, acc[ii][jj][0], acc[ii][jj][1]);
                gstore_pair<Acc>(p, d, r + 8, c, acc[ii][jj][2], acc[ii][jj][3]);
            }
}

// The CTA-wide pipeline over this CTA's larger problems.  K chunks are staged
// in a byte ring, each at the size its problem needs, so that many small
// chunks are in flight at once (up to MAXF cp.async groups): the loads are
// latency-bound, not bandwidth-bound, per SM.  Every thread runs the same
// allocator over the same chunk sequence, so producer and consumer agree on
// where chunk u lives without any shared state: the producer side places
// chunk after chunk at `head` (wrapping to 0 when the rest of the ring is too
// short, the skipped bytes counted as part of that chunk), the consumer side
// replays the same placement to find chunk u and frees it after its MMAs.
template <class Tr>
__device__ __forceinline__ void cta_problems(const GroupedParams &p, int begin, int end, uint8_t *smem)
{
    using G = GGeom<Tr>;
    uint8_t *red = smem + G::RING;
    // producer cursor: problem, chunk start, ring head, chunks issued
    int lp = begin, lk = 0, head = 0, issued = 0;
    int used = 0; // ring bytes held by chunks issued and not yet freed
    // consumer cursor: problem, chunk start, ring position, chunks consumed
    int cp = begin, ck = 0, chead = 0, u = 0;
    GroupedDesc ld_desc = p.desc[begin];
    // accumulators (up to 16 fragments per warp), live across K chunks; each
    // register-tile shape indexes them as [ii * MJ + jj]
    typename Tr::Acc acc[16][4];
    while (cp < end)
    {
        // issue every chunk that fits, up to MAXF in flight
        while (lp < end && issued - u < G::MAXF)
        {
            const int sz = G::chunk_bytes(ld_desc.M, ld_desc.N);
            const bool wrap = head + sz > G::RING; // (head may equal RING: wrap with nothing skipped)
            const int skip = wrap ? G::RING - head : 0;
            if (used + skip + sz > G::RING)
                break;
            const int at = wrap ? 0 : head;
            load_chunk<Tr>(p, ld_desc, lk, smem + at);
            cp_async_commit();
            head = at + sz;
            used += skip + sz;
            ++issued;
            lk += GGeom<Tr>::KCH;
            if (lk >= ld_desc.K)
            {
                lk = 0;
                if (++lp < end)
                    ld_desc = p.desc[lp];
            }
        }
        cp_async_wait_dyn(issued - u - 1);
        __syncthreads();
        const GroupedDesc d = p.desc[cp];
        const int sz = G::chunk_bytes(d.M, d.N);
        const bool wrap = chead + sz > G::RING;
        const int skip = wrap ? G::RING - chead : 0;
        const int at = wrap ? 0 : chead;
        const uint8_t *stage = smem + at;
        const bool first = ck == 0, last = ck + G::KCH >= d.K;
        switch (d.cfg)
        {
        case 0:
            run_chunk<Tr, 1, 16>(p, d, ck, first, last, stage, red, acc);
            break;
        case 1:
            run_chunk<Tr, 2, 8>(p, d, ck, first, last, stage, red, acc);
            break;
        case 2:
            run_chunk<Tr, 4, 4>(p, d, ck, first, last, stage, red, acc);
            break;
        default:
            run_chunk<Tr, 2, 4>(p, d, ck, first, last, stage, red, acc);
            break;
        }
        __syncthreads(); // every warp is done with chunk u: its bytes are free
        chead = at + sz;
        used -= skip + sz;
        ck += G::KCH;
        if (last)
        {
            ck = 0;
            ++cp;
        }
        ++u;
    }
    cp_async_wait<0>();
}

template <class Tr>
__global__ void __launch_bounds__(kThreads, 1) grouped_kernel(const GroupedParams p)
{
    extern __shared__ __align__(128) uint8_t smem[];
    const int begin = p.cta_begin[blockIdx.x], end = p.cta_begin[blockIdx.x + 1];
    if (begin < end)
        cta_problems<Tr>(p, begin, end, smem);
    // then every warp of the grid takes single-warp problems round-robin
    const int gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
    const int nw = gridDim.x * kWarps;
    for (int i = p.small_begin + gw; i < p.small_end; i += nw)
        warp_problem<Tr>(p, p.desc[i]);
}


} // namespace
} // namespace kami

// ---------------------------------------------------------------------------
// host side: plan = descriptors + schedule (+ autotuned partitions)
// ---------------------------------------------------------------------------
using namespace kami;

struct kami_grouped_plan
{
    int in_type, out_type, count, ctas, smem;
    int kernel = 0; // 0: mma.sync warp grids (grouped_kernel), 1: tcgen05 (grouped_tc05_kernel),
                    // 2: staged FP64 DMMA (grouped_f64_kernel)
    int tc_m64 = 0, tc_m128 = 0; // tcgen05 plans: problems on M = 64 / M = 128 MMAs
    bool packed = false;         // tcgen05 plans: some work item holds several problems
    int small_begin = 0, small_end = 0; // desc range of single-warp problems
    GroupedDesc *d_desc = nullptr;
    int *d_begin = nullptr;
    int cfg_hist[kCfgs] = {0};
    int64_t flops = 0, bytes = 0;
};

namespace kami {
namespace {

bool cfg_valid(int cfg, int M, int N)
{
    if (cfg == 7)
        return M <= 32 && N <= 32;
    const int MF = (M + 15) / 16, NF = (N + 7) / 8;
    return (MF + cfg_R(cfg) - 1) / cfg_R(cfg) <= cfg_MI(cfg) && (NF + cfg_C(cfg) - 1) / cfg_C(cfg) <= cfg_MJ(cfg);
}

// static choice: fewest MMA steps on the busiest warp, then fewer depth ranks
int cfg_heuristic(int in_type, int M, int N, int K)
{
    const int kstep = in_type == KAMI_F64 ? 8 : 16;
    const int MF = (M + 15) / 16, NF = (N + 7) / 8, KS = (K + kstep - 1) / kstep;
    if (M <= 32 && N <= 32)
        return 7; // single-warp problem
    int best = -1;
    double bc = 0;
    for (int c = 0; c < 7; ++c)
    {
        if (!cfg_valid(c, M, N))
            continue;
        const int mi = (MF + cfg_R(c) - 1) / cfg_R(c), mj = (NF + cfg_C(c) - 1) / cfg_C(c);
        const int kd = (KS + cfg_D(c) - 1) / cfg_D(c);
        const double cost = (double)mi * mj * kd + 0.5 * (mi + mj) * kd + (cfg_D(c) > 1 ? 4.0 * mi * mj : 0.0);
        if (best < 0 || cost < bc)
        {
            best = c;
            bc = cost;
        }
    }
    return best;
}

// autotune cache: (in_type, M/8, N/8, K/8) -> cfg, measured on this device
std::mutex g_tune_mu;
struct TuneKey
{
    int dev, in_type, M, N, K;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(dev, in_type, M, N, K) < std::tie(o.dev, o.in_type, o.M, o.N, o.K);
    }
};
std::map<TuneKey, int> g_tune;

} // namespace
} // namespace kami

static const void *grouped_fn(int in_type)
{
    return in_type == KAMI_F64    ? (const void *)&grouped_kernel<TrF64>
           : in_type == KAMI_BF16 ? (const void *)&grouped_kernel<TrH16<true>>
                                  : (const void *)&grouped_kernel<TrH16<false>>;
}

static int grouped_smem(int in_type)
{
    return in_type == KAMI_F64 ? GGeom<TrF64>::SMEM : GGeom<TrH16<false>>::SMEM;
}

static int launch_grouped(const kami_grouped_plan *plan, const void *A, const void *B, void *C, double alpha,
                          double beta, int num_iter, cudaStream_t s)
{
    GroupedParams p{};
    p.desc = plan->d_desc;
    p.cta_begin = plan->d_begin;
    p.A = A;
    p.B = B;
    p.C = C;
    p.out_type = plan->out_type;
    p.alpha = alpha;
    p.beta = beta;
    p.num_iter = num_iter;
    p.small_begin = plan->small_begin;
    p.small_end = plan->small_end;
    if (plan->kernel == 1)
        return grouped_tc05_launch(p, plan->in_type == KAMI_BF16, plan->packed, plan->ctas, s);
    if (plan->kernel == 2)
        return grouped_f64s_launch(p, plan->ctas, s);
    void *args[] = {&p};
    cudaError_t e = cudaLaunchKernel(grouped_fn(plan->in_type), dim3(plan->ctas), dim3(kThreads), args,
                                     (size_t)plan->smem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(grouped_kernel)");
    return KAMI_OK;
}

static int free_plan(kami_grouped_plan *pl)
{
    if (!pl)
        return KAMI_OK;
    if (pl->d_desc)
        cudaFree(pl->d_desc);
    if (pl->d_begin)
        cudaFree(pl->d_begin);
    delete pl;
    return KAMI_OK;
}

// Build descriptors + LPT schedule for `count` problems (host arrays) with
// the given partitions and upload them.  kernel 1 (FP16 / BF16 only) is the
// tcgen05 kernel, kernel 2 (FP64 only) the staged DMMA kernel: every problem
// goes through their CTA pipelines (no single-warp problems); the tcgen05
// kernel's cost model is its bytes plus a fixed per-problem latency.
static int build_plan(int in_type, int out_type, int count, const int *M, const int *N, const int *K,
                      const int64_t *ao, const int64_t *bo, const int64_t *co, const int *cfg,
                      kami_grouped_plan **out, const int *lda = nullptr, const int *ldb = nullptr,
                      const int *ldc = nullptr, int kernel = 0, bool pack = false)
{
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return cuda_fail(e, "cudaDeviceGetAttribute");
    const bool tc = kernel == 1, staged = kernel == 2;
    const void *fn = tc ? grouped_tc05_fn(in_type == KAMI_BF16, false) : staged ? grouped_f64s_fn() : grouped_fn(in_type);
    const int smem = tc ? grouped_tc05_smem() : staged ? grouped_f64s_smem() : grouped_smem(in_type);
    const int threads = tc ? grouped_tc05_threads() : staged ? grouped_f64s_threads() : kThreads;
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(grouped kernel)");
    if (tc && (e = cudaFuncSetAttribute(grouped_tc05_fn(in_type == KAMI_BF16, true),
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(grouped kernel)");
    // all of the SM's unified L1 / shared memory as shared memory, so the
    // occupancy below counts every CTA that fits
    for (int pk = 0; tc && pk < 2; ++pk)
        if ((e = cudaFuncSetAttribute(grouped_tc05_fn(in_type == KAMI_BF16, pk == 1),
                                      cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(grouped kernel carveout)");
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (tc)
        occ = grouped_tc05_ctas_per_sm(); // sized for two per SM; the query reports one
    occ = std::max(occ, 1);
    const int ctas = std::max(1, std::min(count, sms * occ));
    const int esz = in_type == KAMI_F64 ? 8 : 2;
    const int osz = out_type == KAMI_F64 ? 8 : out_type == KAMI_F32 ? 4 : 2;
    // FLOP per byte where compute and HBM meet (the tcgen05 kernel's MMAs
    // are never the bound at these sizes)
    const double balance = in_type == KAMI_F64 ? 6.0 : tc ? 1e9 : 150.0;

    auto *pl = new kami_grouped_plan();
    pl->in_type = in_type;
    pl->out_type = out_type;
    pl->count = count;
    pl->ctas = ctas;
    pl->smem = smem;
    pl->kernel = kernel;
    std::vector<double> cost(count);
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i)
    {
        const double fl = 2.0 * M[i] * N[i] * K[i];
        const double by = (double)(M[i] + N[i]) * K[i] * esz + (double)M[i] * N[i] * osz;
        cost[i] = std::max(fl / balance, by) + 2048.0; // + fixed per-problem latency
        order[i] = i;
        pl->flops += (int64_t)fl;
        pl->bytes += (int64_t)by;
        if (!tc && !staged)
            pl->cfg_hist[cfg[i]]++;
    }
    // Work items.  tcgen05 plans put several small problems in one item: their
    // A rows stacked in the item's 128-row A tile, their B rows (each problem's
    // rounded up to 16) in its 128-row B tile, so that one chain of MMAs computes
    // every problem's C block on the accumulator's diagonal (the off-diagonal
    // blocks are computed and never read) and the issuing thread, the loaders
    // and the epilogue pay their fixed per-item costs once for all of them.
    // pk[i]: row offset | column offset << 8 | problems in the item << 16.
    std::vector<std::vector<int>> items;
    std::vector<int> pk(count, 0);
    if (tc && pack)
    {
        std::vector<int> small;
        for (int i = 0; i < count; ++i)
        {
            if (M[i] <= 64 && ((N[i] + 15) & ~15) <= 64)
                small.push_back(i);
            else
                items.push_back({i});
        }
        // similar K together (an item runs to its largest K), then tall first
        std::stable_sort(small.begin(), small.end(), [&](int a, int b) {
            return K[a] != K[b] ? K[a] > K[b] : M[a] > M[b];
        });
        struct Bin
        {
            int item, m, n, k0;
        };
        std::vector<Bin> open; // the most recent bins, first fit
        for (int i : small)
        {
            const int n16 = (N[i] + 15) & ~15;
            bool placed = false;
            for (Bin &b : open)
                if (b.m + M[i] <= 128 && b.n + n16 <= 128 && (int)items[b.item].size() < 4 && b.k0 - K[i] <= 32)
                {
                    pk[i] = b.m | (b.n << 8);
                    items[b.item].push_back(i);
                    b.m += M[i];
                    b.n += n16;
                    placed = true;
                    break;
                }
            if (!placed)
            {
                items.push_back({i});
                open.push_back(Bin{(int)items.size() - 1, M[i], n16, K[i]});
                if (open.size() > 16)
                    open.erase(open.begin());
            }
        }
        for (const auto &it : items)
        {
            for (int i : it)
                pk[i] |= (int)it.size() << 16;
            pl->packed = pl->packed || it.size() > 1;
        }
    }
    else
        for (int i : order)
            items.push_back({i});
    if (tc)
        for (const auto &it : items)
        {
            int mt = 0;
            for (int i : it)
                mt += M[i];
            (mt <= 64 ? pl->tc_m64 : pl->tc_m128) += (int)it.size();
        }
    std::vector<double> icost(items.size(), 2048.0);
    std::vector<int> iorder(items.size());
    for (size_t t = 0; t < items.size(); ++t)
    {
        for (int i : items[t])
            icost[t] += cost[i] - 2048.0;
        iorder[t] = (int)t;
    }
    std::stable_sort(iorder.begin(), iorder.end(), [&](int a, int b) { return icost[a] > icost[b]; });
    typedef std::pair<double, int> Load;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int c = 0; c < ctas; ++c)
        heap.push(Load(0.0, c));
    std::vector<std::vector<int>> lists(ctas); // work items per CTA
    std::vector<int> smalls;
    for (int t : iorder)
    {
        const int i = items[t][0];
        if (cfg[i] == 7 && kernel == 0)
        {
            smalls.push_back(i); // longest first, spread over all warps round-robin
            continue;
        }
        Load l = heap.top();
        heap.pop();
        lists[l.second].push_back(t);
        heap.push(Load(l.first + icost[t], l.second));
    }
    std::vector<GroupedDesc> desc;
    desc.reserve(count);
    std::vector<int> begin(ctas + 1, 0);
    for (int c = 0; c < ctas; ++c)
    {
        begin[c] = (int)desc.size();
        for (int t : lists[c])
        {
            // tcgen05 plans: the item's extent in every member (see item_at in
            // grouped_tc05.cu): count | Mt << 3 | (Nt / 16) << 11 | Kt << 15
            int mt = 0, nt = 0, kt = 0;
            for (int i : items[t])
            {
                mt = std::max(mt, (pk[i] & 0xff) + M[i]);
                nt = std::max(nt, ((pk[i] >> 8) & 0xff) + ((N[i] + 15) & ~15));
                kt = std::max(kt, K[i]);
            }
            const int ext = tc ? (int)items[t].size() | (mt << 3) | ((nt / 16) << 11) | (kt << 15) : 0;
            for (int i : items[t])
                desc.push_back(GroupedDesc{M[i], N[i], K[i], tc ? pk[i] : cfg[i], ao[i], bo[i], co[i],
                                           lda ? lda[i] : K[i], ldb ? ldb[i] : K[i], ldc ? ldc[i] : N[i], ext});
        }
    }
    begin[ctas] = (int)desc.size();
    pl->small_begin = (int)desc.size();
    for (int i : smalls)
        desc.push_back(GroupedDesc{M[i], N[i], K[i], cfg[i], ao[i], bo[i], co[i], lda ? lda[i] : K[i],
                                   ldb ? ldb[i] : K[i], ldc ? ldc[i] : N[i], 0});
    pl->small_end = (int)desc.size();
    if ((e = cudaMalloc(&pl->d_desc, sizeof(GroupedDesc) * std::max(count, 1))) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_begin, sizeof(int) * (ctas + 1))) != cudaSuccess)
    {
        free_plan(pl);
        return cuda_fail(e, "cudaMalloc(grouped plan)");
    }
    if ((e = cudaMemcpy(pl->d_desc, desc.data(), sizeof(GroupedDesc) * count, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(pl->d_begin, begin.data(), sizeof(int) * (ctas + 1), cudaMemcpyHostToDevice)) != cudaSuccess)
    {
        free_plan(pl);
        return cuda_fail(e, "cudaMemcpy(grouped plan)");
    }
    *out = pl;
    return KAMI_OK;
}

// Measure every valid partition on a batch of problems of one shape and
// return the fastest.  Scratch buffers are the caller's.
static int tune_shape(int in_type, int out_type, int M, int N, int K, void *A, void *B, void *C, int reps_problems,
                      int *best_cfg)
{
    std::vector<int> vm(reps_problems, M), vn(reps_problems, N), vk(reps_problems, K), vc(reps_problems);
    std::vector<int64_t> ao(reps_problems), bo(reps_problems), co(reps_problems);
    for (int i = 0; i < reps_problems; ++i)
    {
        ao[i] = (int64_t)i * M * K;
        bo[i] = (int64_t)i * N * K;
        co[i] = (int64_t)i * M * N;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bc = cfg_heuristic(in_type, M, N, K);
    for (int c = 0; c < kCfgs; ++c)
    {
        if (!cfg_valid(c, M, N))
            continue;
        std::fill(vc.begin(), vc.end(), c);
        kami_grouped_plan *pl = nullptr;
        int st = build_plan(in_type, out_type, reps_problems, vm.data(), vn.data(), vk.data(), ao.data(), bo.data(),
                            co.data(), vc.data(), &pl);
        if (st)
        {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return st;
        }
        launch_grouped(pl, A, B, C, 1.0, 0.0, 1, 0);
        cudaEventRecord(e0, 0);
        for (int r = 0; r < 3; ++r)
            launch_grouped(pl, A, B, C, 1.0, 0.0, 1, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        free_plan(pl);
        if (ms < best)
        {
            best = ms;
            bc = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(e, "grouped autotune");
    *best_cfg = bc;
    return KAMI_OK;
}

namespace kami {

// Serve a batched request that no compiled block instance covers (e.g. FP64
// above 64^3) with the grouped kernel: one plan per distinct request shape,
// cached (descriptors hold offsets, not pointers, so a plan serves any
// buffers).
int grouped_fallback(const GemmArgs &g, int in_type, cudaStream_t stream)
{
    if (g.a_layout != KAMI_A_ROW_MK || g.b_layout != KAMI_B_REF_NK)
        return fail(KAMI_ERR_UNSUPPORTED, "no kernel for this shape with these layouts");
    const int q = in_type == KAMI_F64 ? 2 : 8;
    if (g.M > 128 || g.N > 128 || g.K > 128 || g.K % q || g.lda % q || g.ldb % q || g.sA % q || g.sB % q ||
        g.batch > 1000000)
        return fail(KAMI_ERR_UNSUPPORTED, "no kernel for M=%d N=%d K=%d (lda=%lld ldb=%lld)", g.M, g.N, g.K,
                    (long long)g.lda, (long long)g.ldb);
    if ((reinterpret_cast<uintptr_t>(g.A) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15) ||
        (reinterpret_cast<uintptr_t>(g.C) & 15))
        return fail(KAMI_ERR_UNSUPPORTED, "no kernel for this shape with unaligned buffers");
    static std::mutex mu;
    static std::map<std::vector<int64_t>, kami_grouped_plan *> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<int64_t> key = {dev, in_type, g.out_type, g.M, g.N, g.K, g.batch, g.lda, g.ldb, g.ldc, g.sA, g.sB, g.sC};
    kami_grouped_plan *pl = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end())
            pl = it->second;
    }
    if (!pl)
    {
        const int n = (int)g.batch;
        std::vector<int> vm(n, g.M), vn(n, g.N), vk(n, g.K), vc(n, cfg_heuristic(in_type, g.M, g.N, g.K));
        std::vector<int> la(n, (int)g.lda), lb(n, (int)g.ldb), lc(n, (int)g.ldc);
        std::vector<int64_t> ao(n), bo(n), co(n);
        for (int i = 0; i < n; ++i)
        {
            ao[i] = (int64_t)i * g.sA;
            bo[i] = (int64_t)i * g.sB;
            co[i] = (int64_t)i * g.sC;
        }
        int st = build_plan(in_type, g.out_type, n, vm.data(), vn.data(), vk.data(), ao.data(), bo.data(), co.data(),
                            vc.data(), &pl, la.data(), lb.data(), lc.data(), in_type == KAMI_F64 ? 2 : 1);
        if (st)
            return st;
        std::lock_guard<std::mutex> lk(mu);
        if (cache.size() < 256)
            cache[key] = pl;
    }
    return launch_grouped(pl, g.A, g.B, g.C, g.alpha, g.beta, g.num_iter, stream);
}

} // namespace kami

extern "C" {

int kami_gemm_grouped_plan_create(kami_dtype_t in_type, kami_dtype_t out_type, int count, const int *M, const int *N,
                                  const int *K, const int64_t *a_offsets, const int64_t *b_offsets,
                                  const int64_t *c_offsets, int flags, kami_grouped_plan **plan)
{
    if (!plan)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: plan is NULL");
    *plan = nullptr;
    if (in_type != KAMI_F16 && in_type != KAMI_BF16 && in_type != KAMI_F64)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: in_type must be KAMI_F16, KAMI_BF16 or KAMI_F64");
    if ((in_type == KAMI_F64) != (out_type == KAMI_F64) ||
        (out_type != KAMI_F64 && out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16))
        return fail(KAMI_ERR_UNSUPPORTED, "grouped: output type does not match the input type");
    if (count < 0 || (count > 0 && (!M || !N || !K || !a_offsets || !b_offsets || !c_offsets)))
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: bad count or null shape/offset arrays");
    const bool force_mma = (flags & KAMI_PLAN_MMA_SYNC) != 0, force_tc = (flags & KAMI_PLAN_TCGEN05) != 0,
               force_st = (flags & KAMI_PLAN_STAGED) != 0, pack = (flags & KAMI_PLAN_PACK) != 0;
    if ((int)force_mma + (int)force_tc + (int)force_st > 1)
        return fail(KAMI_ERR_INVALID_VALUE,
                    "grouped: KAMI_PLAN_MMA_SYNC, KAMI_PLAN_TCGEN05 and KAMI_PLAN_STAGED are exclusive");
    if (force_tc && in_type == KAMI_F64)
        return fail(KAMI_ERR_UNSUPPORTED, "grouped: the tcgen05 kernel takes FP16 / BF16 inputs");
    if (force_st && in_type != KAMI_F64)
        return fail(KAMI_ERR_UNSUPPORTED, "grouped: the staged DMMA kernel takes FP64 inputs");
    const int kq = in_type == KAMI_F64 ? 2 : 8;
    for (int i = 0; i < count; ++i)
    {
        if (M[i] < 1 || N[i] < 1 || K[i] < 1 || M[i] > 128 || N[i] > 128 || K[i] > 128)
            return fail(KAMI_ERR_UNSUPPORTED, "grouped: problem %d has M, N, K = %d, %d, %d (each must be 1..128)",
                        i, M[i], N[i], K[i]);
        if (K[i] % kq)
            return fail(KAMI_ERR_UNSUPPORTED, "grouped: problem %d: K must be a multiple of %d", i, kq);
        if (a_offsets[i] % kq || b_offsets[i] % kq || a_offsets[i] < 0 || b_offsets[i] < 0 || c_offsets[i] < 0)
            return fail(KAMI_ERR_MISALIGNED, "grouped: problem %d: A/B offsets must be multiples of %d", i, kq);
    }
    std::vector<int> cfg(count);
    const bool tune = (flags & 1) != 0;
    if (!tune)
    {
        for (int i = 0; i < count; ++i)
            cfg[i] = cfg_heuristic(in_type, M[i], N[i], K[i]);
    }
    else
    {
        int dev = 0;
        cudaGetDevice(&dev);
        // tune per 16-rounded shape bucket, measured at the bucket's largest shape
        std::map<TuneKey, int> need;
        for (int i = 0; i < count; ++i)
        {
            TuneKey k{dev, in_type, (M[i] + 15) / 16, (N[i] + 15) / 16, (K[i] + 15) / 16};
            need[k] = -1;
        }
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            for (auto &kv : need)
            {
                auto it = g_tune.find(kv.first);
                if (it != g_tune.end())
                    kv.second = it->second;
            }
        }
        const int reps = 1024;
        const int esz = in_type == KAMI_F64 ? 8 : 2, osz = out_type == KAMI_F64 ? 8 : out_type == KAMI_F32 ? 4 : 2;
        void *tA = nullptr, *tB = nullptr, *tC = nullptr;
        bool missing = false;
        for (auto &kv : need)
            missing |= kv.second < 0;
        if (missing)
        {
            cudaError_t e;
            if ((e = cudaMalloc(&tA, (size_t)reps * 128 * 128 * esz)) != cudaSuccess ||
                (e = cudaMalloc(&tB, (size_t)reps * 128 * 128 * esz)) != cudaSuccess ||
                (e = cudaMalloc(&tC, (size_t)reps * 128 * 128 * osz)) != cudaSuccess)
            {
                cudaFree(tA);
                cudaFree(tB);
                return cuda_fail(e, "cudaMalloc(grouped autotune scratch)");
            }
            cudaMemset(tA, 0, (size_t)reps * 128 * 128 * esz);
            cudaMemset(tB, 0, (size_t)reps * 128 * 128 * esz);
            for (auto &kv : need)
            {
                if (kv.second >= 0)
                    continue;
                const int m = std::min(128, kv.first.M * 16), n = std::min(128, kv.first.N * 16),
                          k = std::min(128, kv.first.K * 16);
                int best = 0;
                int st = tune_shape(in_type, out_type, m, n, k, tA, tB, tC, reps, &best);
                if (st)
                {
                    cudaFree(tA);
                    cudaFree(tB);
                    cudaFree(tC);
                    return st;
                }
                kv.second = best;
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune[kv.first] = best;
            }
            cudaFree(tA);
            cudaFree(tB);
            cudaFree(tC);
        }
        for (int i = 0; i < count; ++i)
        {
            TuneKey k{dev, in_type, (M[i] + 15) / 16, (N[i] + 15) / 16, (K[i] + 15) / 16};
            int c = need[k];
            cfg[i] = cfg_valid(c, M[i], N[i]) ? c : cfg_heuristic(in_type, M[i], N[i], K[i]);
        }
    }
    // the kernel besides the warp-grid one: tcgen05 for 16-bit inputs, the
    // staged DMMA kernel for FP64
    const int alt = in_type == KAMI_F64 ? 2 : 1;
    // FP64 without a measurement: the staged kernel, unless problems of at
    // most 32 x 32 carry most of the bytes -- its fourteen compute warps pay
    // a fixed cost per problem that the warp-grid kernel's one-warp path for
    // such problems does not (20000 problems of 32^3: 0.21 ms staged, 0.15
    // warp grids; the uneven 8..128 mix: 0.36 against 0.81)
    bool tiny_mix = false;
    if (in_type == KAMI_F64 && !force_st && !tune)
    {
        double tiny = 0.0, all = 0.0;
        for (int i = 0; i < count; ++i)
        {
            const double by = (double)(M[i] + N[i]) * K[i] + (double)M[i] * N[i];
            all += by;
            if (M[i] <= 32 && N[i] <= 32)
                tiny += by;
        }
        tiny_mix = tiny > 0.6 * all;
    }
    if (force_mma || tiny_mix)
        return build_plan(in_type, out_type, count, M, N, K, a_offsets, b_offsets, c_offsets, cfg.data(), plan);
    if (force_tc || force_st || !tune || count == 0)
        return build_plan(in_type, out_type, count, M, N, K, a_offsets, b_offsets, c_offsets, cfg.data(), plan,
                          nullptr, nullptr, nullptr, alt, pack);
    // autotuned, kernel not forced: build both kernels' plans, time each on
    // scratch buffers of the plan's extent, keep the faster
    kami_grouped_plan *pl[2] = {nullptr, nullptr};
    for (int k = 0; k < 2; ++k)
    {
        int st = build_plan(in_type, out_type, count, M, N, K, a_offsets, b_offsets, c_offsets, cfg.data(), &pl[k],
                            nullptr, nullptr, nullptr, k == 0 ? 0 : alt, pack);
        if (st)
        {
            free_plan(pl[0]);
            return st;
        }
    }
    int64_t na = 0, nb = 0, nc = 0;
    for (int i = 0; i < count; ++i)
    {
        na = std::max(na, a_offsets[i] + (int64_t)M[i] * K[i]);
        nb = std::max(nb, b_offsets[i] + (int64_t)N[i] * K[i]);
        nc = std::max(nc, c_offsets[i] + (int64_t)M[i] * N[i]);
    }
    const int isz = in_type == KAMI_F64 ? 8 : 2, osz = out_type == KAMI_F64 ? 8 : out_type == KAMI_F32 ? 4 : 2;
    void *tA = nullptr, *tB = nullptr, *tC = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&tA, (size_t)na * isz)) != cudaSuccess ||
        (e = cudaMalloc(&tB, (size_t)nb * isz)) != cudaSuccess || (e = cudaMalloc(&tC, (size_t)nc * osz)) != cudaSuccess)
    {
        cudaFree(tA);
        cudaFree(tB);
        free_plan(pl[0]);
        free_plan(pl[1]);
        return cuda_fail(e, "cudaMalloc(grouped kernel choice scratch)");
    }
    cudaMemset(tA, 0, (size_t)na * isz);
    cudaMemset(tB, 0, (size_t)nb * isz);
    float ms[2] = {0.f, 0.f};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = KAMI_OK;
    for (int k = 0; k < 2 && st == KAMI_OK; ++k)
    {
        st = launch_grouped(pl[k], tA, tB, tC, 1.0, 0.0, 1, 0);
        cudaEventRecord(e0, 0);
        for (int r = 0; r < 3 && st == KAMI_OK; ++r)
            st = launch_grouped(pl[k], tA, tB, tC, 1.0, 0.0, 1, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[k], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st == KAMI_OK && (e = cudaGetLastError()) != cudaSuccess)
        st = cuda_fail(e, "grouped kernel choice");
    cudaFree(tA);
    cudaFree(tB);
    cudaFree(tC);
    if (st)
    {
        free_plan(pl[0]);
        free_plan(pl[1]);
        return st;
    }
    const int keep = ms[1] <= ms[0] ? 1 : 0;
    free_plan(pl[1 - keep]);
    *plan = pl[keep];
    return KAMI_OK;
}

int kami_gemm_grouped_run(const kami_grouped_plan *plan, const void *A, const void *B, void *C, double alpha,
                          double beta, int num_iter, void *stream)
{
    if (!plan)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: plan is NULL");
    if (num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: num_iter must be >= 1");
    if (plan->count == 0)
        return KAMI_OK;
    if (!A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: null buffer");
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15) ||
        (reinterpret_cast<uintptr_t>(C) & 15))
        return fail(KAMI_ERR_MISALIGNED, "grouped: A, B, C must be 16-byte aligned");
    return launch_grouped(plan, A, B, C, alpha, beta, num_iter, reinterpret_cast<cudaStream_t>(stream));
}

int kami_gemm_grouped_plan_info(const kami_grouped_plan *plan, int64_t out[16])
{
    if (!plan || !out)
        return fail(KAMI_ERR_INVALID_VALUE, "grouped: null plan or out");
    out[0] = plan->count;
    out[1] = plan->ctas;
    out[2] = plan->smem;
    out[3] = plan->flops;
    out[4] = plan->bytes;
    for (int c = 0; c < kCfgs; ++c)
        out[5 + c] = plan->cfg_hist[c];
    out[13] = plan->kernel;
    out[14] = plan->tc_m64;
    out[15] = plan->tc_m128;
    return KAMI_OK;
}

int kami_gemm_grouped_plan_destroy(kami_grouped_plan *plan) { return free_plan(plan); }

} // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of the grouped launch.
//
// Callers that cannot allocate device memory -- hosts whose own allocator
// carves up device memory once at start-up and treats any later cudaMalloc
// as a fault (serving processes, real-time and embedded controllers), and
// plug-ins running inside such hosts -- cannot create a plan, because a plan
// keeps its problem descriptors and schedule in cudaMalloc'd memory.  This
// entry point keeps them instead in one fixed array of device memory that
// belongs to the library (a file-scope __device__ array,
// KAMI_NOALLOC_MAX_PROBLEMS descriptors plus the CTA schedule, about 0.45 MB
// on every GPU that loads the library, held until the process exits).  Each
// call rebuilds the schedule on the host (static staging arrays, no heap),
// copies it into that array with cudaMemcpyAsync on the caller's stream and
// launches the mma.sync grouped kernel (warp grids chosen by the static cost
// model).  Every call shares the array and leaves its own contents behind.
// Calls on one stream are ordered by that stream and are safe; calls on
// different streams (or from host threads using different streams) whose
// work overlaps on the GPU race on the array.
// ---------------------------------------------------------------------------
namespace kami {
namespace {

constexpr int kNoAllocMaxProblems = 8192; // KAMI_NOALLOC_MAX_PROBLEMS in kami.h
constexpr int kNoAllocMaxCtas = 1024;
constexpr size_t kNoAllocDescBytes = (size_t)kNoAllocMaxProblems * sizeof(GroupedDesc);
constexpr size_t kNoAllocBytes = kNoAllocDescBytes + (size_t)(kNoAllocMaxCtas + 1) * sizeof(int);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocDevice
{
    bool ready = false;
    void *scratch = nullptr; // device address of g_noalloc_scratch on this device
    int ctas_max = 0;        // persistent CTAs the kernel can keep resident
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64][3]; // [device][precision class]

// host staging (no heap allocation on this path)
GroupedDesc g_na_desc[kNoAllocMaxProblems];
int g_na_begin[kNoAllocMaxCtas + 1];
int g_na_order[kNoAllocMaxProblems];
int g_na_cta[kNoAllocMaxProblems];
double g_na_cost[kNoAllocMaxProblems];
double g_na_load[kNoAllocMaxCtas];
int g_na_heap[kNoAllocMaxCtas];

int noalloc_class(int in_type) { return in_type == KAMI_F64 ? 2 : in_type == KAMI_BF16 ? 1 : 0; }

// once per device (with that device current): the device address of the
// scratch array, the kernel's shared-memory limit and its resident CTAs
int noalloc_setup(int in_type, NoAllocDevice **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return fail(KAMI_ERR_UNSUPPORTED, "no-alloc grouped GEMM: device ordinal %d above 63", dev);
    NoAllocDevice &d = g_noalloc_dev[dev][noalloc_class(in_type)];
    if (!d.ready)
    {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        const void *fn = grouped_fn(in_type);
        const int smem = grouped_smem(in_type);
        if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(grouped_kernel)");
        int sms = 0, occ = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
            return cuda_fail(e, "cudaDeviceGetAttribute");
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kThreads, smem)) != cudaSuccess)
            return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        d.scratch = ptr;
        d.ctas_max = std::min(kNoAllocMaxCtas, sms * std::max(occ, 1));
        d.ready = true;
    }
    *out = &d;
    return KAMI_OK;
}

void heap_sift_down(int n, int i)
{
    while (true)
    {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && g_na_load[g_na_heap[l]] < g_na_load[g_na_heap[m]])
            m = l;
        if (r < n && g_na_load[g_na_heap[r]] < g_na_load[g_na_heap[m]])
            m = r;
        if (m == i)
            return;
        std::swap(g_na_heap[i], g_na_heap[m]);
        i = m;
    }
}

} // namespace
} // namespace kami

extern "C" int kami_gemm_grouped_noalloc(kami_dtype_t in_type, kami_dtype_t out_type, int count, const int *M,
                                         const int *N, const int *K, const int64_t *a_offsets,
                                         const int64_t *b_offsets, const int64_t *c_offsets, const void *A,
                                         const void *B, void *C, double alpha, double beta, int num_iter,
                                         void *stream)
{
    if (in_type != KAMI_F16 && in_type != KAMI_BF16 && in_type != KAMI_F64)
        return fail(KAMI_ERR_INVALID_VALUE, "no-alloc grouped GEMM: in_type must be KAMI_F16, KAMI_BF16 or KAMI_F64");
    if ((in_type == KAMI_F64) != (out_type == KAMI_F64) ||
        (out_type != KAMI_F64 && out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16))
        return fail(KAMI_ERR_UNSUPPORTED, "no-alloc grouped GEMM: output type does not match the input type");
    if (count < 0 || num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "no-alloc grouped GEMM: bad count or num_iter");
    if (count > kNoAllocMaxProblems)
        return fail(KAMI_ERR_UNSUPPORTED,
                    "no-alloc grouped GEMM: %d problems exceed the fixed device array of %d descriptors "
                    "(KAMI_NOALLOC_MAX_PROBLEMS); split the call or use kami_gemm_grouped_plan_create",
                    count, kNoAllocMaxProblems);
    if (count == 0)
        return KAMI_OK;
    if (!M || !N || !K || !a_offsets || !b_offsets || !c_offsets || !A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "no-alloc grouped GEMM: null array or buffer");
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15) ||
        (reinterpret_cast<uintptr_t>(C) & 15))
        return fail(KAMI_ERR_MISALIGNED, "no-alloc grouped GEMM: A, B, C must be 16-byte aligned");
    const int kq = in_type == KAMI_F64 ? 2 : 8;
    for (int i = 0; i < count; ++i)
    {
        if (M[i] < 1 || N[i] < 1 || K[i] < 1 || M[i] > 128 || N[i] > 128 || K[i] > 128 || K[i] % kq)
            return fail(KAMI_ERR_UNSUPPORTED, "no-alloc grouped GEMM: problem %d has M, N, K = %d, %d, %d", i, M[i],
                        N[i], K[i]);
        if (a_offsets[i] % kq || b_offsets[i] % kq || a_offsets[i] < 0 || b_offsets[i] < 0 || c_offsets[i] < 0)
            return fail(KAMI_ERR_MISALIGNED, "no-alloc grouped GEMM: problem %d: bad offsets", i);
    }

    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice *dev = nullptr;
    int st = noalloc_setup(in_type, &dev);
    if (st)
        return st;
    const int ctas = std::max(1, std::min(count, dev->ctas_max));
    const int esz = in_type == KAMI_F64 ? 8 : 2;
    const int osz = out_type == KAMI_F64 ? 8 : out_type == KAMI_F32 ? 4 : 2;
    const double balance = in_type == KAMI_F64 ? 6.0 : 150.0;
    for (int i = 0; i < count; ++i)
    {
        const double fl = 2.0 * M[i] * N[i] * K[i];
        const double by = (double)(M[i] + N[i]) * K[i] * esz + (double)M[i] * N[i] * osz;
        g_na_cost[i] = std::max(fl / balance, by) + 2048.0;
        g_na_order[i] = i;
    }
    std::sort(g_na_order, g_na_order + count, [](int a, int b) {
        return g_na_cost[a] > g_na_cost[b] || (g_na_cost[a] == g_na_cost[b] && a < b);
    });
    // longest-first onto the least-loaded CTA (a min-heap over static arrays)
    for (int c = 0; c < ctas; ++c)
    {
        g_na_load[c] = 0.0;
        g_na_heap[c] = c;
        g_na_begin[c] = 0;
    }
    for (int r = 0; r < count; ++r)
    {
        const int i = g_na_order[r];
        if (cfg_heuristic(in_type, M[i], N[i], K[i]) == 7)
        {
            g_na_cta[i] = -1; // single-warp problem: placed after the CTA lists
            continue;
        }
        const int c = g_na_heap[0];
        g_na_cta[i] = c;
        g_na_begin[c]++;
        g_na_load[c] += g_na_cost[i];
        heap_sift_down(ctas, 0);
    }
    int run = 0;
    for (int c = 0; c < ctas; ++c)
    {
        const int n = g_na_begin[c];
        g_na_begin[c] = run;
        run += n;
    }
    g_na_begin[ctas] = run;
    {
        // place problems in LPT order inside each CTA's range (cursor per CTA in g_na_heap)
        for (int c = 0; c < ctas; ++c)
            g_na_heap[c] = g_na_begin[c];
        int small_slot = run;
        for (int r = 0; r < count; ++r)
        {
            const int i = g_na_order[r];
            const int slot = g_na_cta[i] < 0 ? small_slot++ : g_na_heap[g_na_cta[i]]++;
            g_na_desc[slot] = GroupedDesc{M[i], N[i], K[i], cfg_heuristic(in_type, M[i], N[i], K[i]),
                                          a_offsets[i], b_offsets[i], c_offsets[i], K[i], K[i], N[i], 0};
        }
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned char *base = reinterpret_cast<unsigned char *>(dev->scratch);
    cudaError_t e = cudaMemcpyAsync(base, g_na_desc, sizeof(GroupedDesc) * (size_t)count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + kNoAllocDescBytes, g_na_begin, sizeof(int) * (size_t)(ctas + 1),
                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(no-alloc grouped schedule)");
    GroupedParams p{};
    p.desc = reinterpret_cast<const GroupedDesc *>(base);
    p.cta_begin = reinterpret_cast<const int *>(base + kNoAllocDescBytes);
    p.small_begin = run;
    p.small_end = count;
    p.A = A;
    p.B = B;
    p.C = C;
    p.out_type = out_type;
    p.alpha = alpha;
    p.beta = beta;
    p.num_iter = num_iter;
    void *args[] = {&p};
    e = cudaLaunchKernel(grouped_fn(in_type), dim3(ctas), dim3(kThreads), args, (size_t)grouped_smem(in_type), s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(grouped_kernel, no-alloc)");
    return KAMI_OK;
}
