// grouped_f64.cu -- the uneven (grouped) batched GEMM in FP64: thousands of
// problems of different M, N, K (each <= 128) in one persistent launch, on
// the DMMA pipe (m16n8k8), with the operands staged in shared memory.
//
// The warp-grid kernel of grouped.cu holds each warp's slice of A and B and
// of C in registers; in FP64 that is 255 registers with spills, one CTA of
// eight warps per SM, and the SM waits on latency between its loads and its
// DMMAs.  Here one CTA per SM walks its share of the plan's longest-first
// schedule with two warp roles:
//   warps 14-15 loaders: each K chunk of 32 (A rows, then B rows) is copied
//              with 16-byte cp.async into a ring of kSlots stages, laid out
//              as four 8-column k-step boxes per operand with the 64-byte
//              swizzle (the 16-byte chunk t of row r at t ^ ((r / 2) % 4)),
//              so the two rows of a quarter-warp's fragment fetch share one
//              128-byte line without bank conflicts; every loader thread's
//              arrival on full[s] is attached to its copies
//              (cp.async.mbarrier.arrive), so a chunk publishes itself when
//              it lands;
//   warps 0-13 compute: a problem's C is cut into 16 x 16 sub-tiles; warp w
//              owns sub-tiles w, w + 14, ... (at most 64 of them, five per
//              warp) for the whole problem, keeps their accumulators in
//              registers across the problem's K chunks (two m16n8k8 DMMAs
//              per sub-tile and k-step, fragments read from the
//              stage with one 16-byte load each -- the k index is permuted
//              identically for A and B: lane t holds k = 2t, 2t + 1 of a
//              k-step), frees the stage (empty[s]) and, after the last chunk,
//              stores its sub-tiles straight from the accumulators.
// The CTA's descriptors (up to kDescCache) are copied to shared memory at
// the start.  Columns past K are zero-filled by the copies; stale rows past
// M or N only reach rows and columns of C that are never stored.  Every
// mbarrier wait is bounded; a timeout sets g_gf64_error and ends that role's
// loop.
#include <cstdint>

#include "grouped.cuh"
#include "kami_common.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device status of the bounded waits (read and cleared by kami_device_status)
__device__ int g_gf64_error = 0;

namespace {

constexpr int kSlots = 3;                   // stages of one K chunk each
constexpr int kKChunk = 32;                 // K elements per chunk: four k-steps of 8
constexpr int kBox = 128 * 64;              // one k-step box of an operand: 128 rows x 64 bytes
constexpr int kOper = 4 * kBox;             // one operand's chunk
constexpr int kSlotBytes = 2 * kOper;       // A then B
// 16 warps in all (four per scheduler), so that each may hold 128 registers
constexpr int kComputeWarps = 14;
constexpr int kMaxSub = 5; // 16 x 16 sub-tiles per compute warp (64 in a 128 x 128 C)
constexpr int kLoadWarps = 2;
constexpr int kLoaders = kLoadWarps * 32;
constexpr int kThreads = (kComputeWarps + kLoadWarps) * 32;

struct SDesc
{
    int M, N, K, lda, ldb, ldc;
    int64_t a_off, b_off, c_off;
};
constexpr int kDescCache = 256;
constexpr int kBars = 2 * kSlots;
constexpr int kSmem = kSlots * kSlotBytes + kDescCache * (int)sizeof(SDesc) + kBars * 8 + 128;

__device__ __forceinline__ SDesc get_desc(const SDesc *cache, const GroupedDesc *g, int begin, int i)
{
    if (i - begin < kDescCache)
        return cache[i - begin];
    const GroupedDesc d = g[i];
    return SDesc{d.M, d.N, d.K, d.lda, d.ldb, d.ldc, d.a_off, d.b_off, d.c_off};
}

struct GfParams
{
    GroupedParams p;
    uint64_t timeout_ns;
};

__device__ __forceinline__ void gf_flag(int code) { atomicExch(&g_gf64_error, code); }

__device__ __forceinline__ void cp16(uint32_t dst, const void *src, bool valid)
{
    // src-size 0 writes 16 zero bytes
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
// arrive (once, counted in the barrier's expected arrivals) on `bar` when
// every cp.async this thread has issued so far has completed
__device__ __forceinline__ void cp_arrive_on(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// shared address of elements 2t, 2t + 1 of k-step ks in row r of an operand
__device__ __forceinline__ uint32_t frag_addr(uint32_t base, int r, int ks, int t)
{
    return base + ks * kBox + r * 64 + ((t ^ ((r >> 1) & 3)) << 4);
}

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

// One 16 x 16 sub-tile (rows r0.., columns c0.., second n8 tile live when
// two) over ksteps k-steps of the staged chunk.
__device__ __forceinline__ void subtile_chunk(uint32_t sa, uint32_t sb, int r0, int c0, bool two, int ksteps,
                                              int gq, int tq, double (&acc)[2][4])
{
    for (int ks = 0; ks < ksteps; ++ks)
    {
        const double2 lo = lds_d2(frag_addr(sa, r0 + gq, ks, tq));
        const double2 hi = lds_d2(frag_addr(sa, r0 + gq + 8, ks, tq));
        const double a[4] = {lo.x, hi.x, lo.y, hi.y};
        const double2 v0 = lds_d2(frag_addr(sb, c0 + gq, ks, tq));
        dmma(acc[0], a, v0.x, v0.y);
        if (two)
        {
            const double2 v1 = lds_d2(frag_addr(sb, c0 + 8 + gq, ks, tq));
            dmma(acc[1], a, v1.x, v1.y);
        }
    }
}

// C[r][c], C[r][c + 1] = alpha * (v0, v1) + beta * C (within M x N)
__device__ __forceinline__ void store_f64_pair(double *Cb, int M, int N, int64_t ldc, bool vec, double alpha,
                                               double beta, int r, int c, double v0, double v1)
{
    if (r >= M || c >= N)
        return;
    double *q = Cb + (int64_t)r * ldc + c;
    const bool two = c + 1 < N;
    double x0 = alpha * v0, x1 = alpha * v1;
    if (beta != 0.0)
    {
        x0 += beta * q[0];
        if (two)
            x1 += beta * q[1];
    }
    if (two && vec)
        *reinterpret_cast<double2 *>(q) = make_double2(x0, x1);
    else
    {
        q[0] = x0;
        if (two)
            q[1] = x1;
    }
}

__global__ void __launch_bounds__(kThreads, 1) grouped_f64_kernel(const __grid_constant__ GfParams gp)
{
    const GroupedParams &p = gp.p;
    extern __shared__ __align__(128) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((128u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 127u)) & 127u);
    SDesc *dcache = reinterpret_cast<SDesc *>(smem + kSlots * kSlotBytes);
    uint64_t *full = reinterpret_cast<uint64_t *>(dcache + kDescCache);
    uint64_t *empty = full + kSlots;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int begin = p.cta_begin[blockIdx.x], end = p.cta_begin[blockIdx.x + 1];
    const uint64_t limit = gp.timeout_ns;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kSlots; ++s)
        {
            tc::mbar_init(&full[s], kLoaders);
            tc::mbar_init(&empty[s], kComputeWarps);
        }
        tc::fence_mbar_init();
    }
    for (int i = threadIdx.x; i < end - begin && i < kDescCache; i += kThreads)
    {
        const GroupedDesc d = p.desc[begin + i];
        dcache[i] = SDesc{d.M, d.N, d.K, d.lda, d.ldb, d.ldc, d.a_off, d.b_off, d.c_off};
    }
    __syncthreads();
    const uint32_t slots = tc::smem_u32(smem);

    if (warp >= kComputeWarps)
    {
        // ---- loaders ----
        const int tl = threadIdx.x - kComputeWarps * 32;
        const int q = tl & 15, rsub = tl >> 4; // 16-byte chunk of a 256-byte chunk row; first row
        const int qb = q >> 2, qt = q & 3;     // its k-step box and chunk within the box
        const uint8_t *A = reinterpret_cast<const uint8_t *>(p.A);
        const uint8_t *B = reinterpret_cast<const uint8_t *>(p.B);
        int j = 0;
        bool ok = true;
        for (int i = begin; i < end && ok; ++i)
        {
            const SDesc d = get_desc(dcache, p.desc, begin, i);
            const uint8_t *Ab = A + d.a_off * 8, *Bb = B + d.b_off * 8;
            for (int k0 = 0; k0 < d.K; k0 += kKChunk, ++j)
            {
                const int s = j % kSlots;
                if (j >= kSlots && !tc::mbar_wait_bounded(&empty[s], ((j / kSlots) - 1) & 1, limit))
                {
                    gf_flag(1);
                    ok = false;
                    break;
                }
                const uint32_t sa = slots + s * kSlotBytes, sb = sa + kOper;
                // 16-byte chunks per row the DMMAs read: whole k-steps of 8
                const int kc = ((min(kKChunk, d.K - k0) + 7) >> 3) * 4;
                const bool live = q < kc;
                const bool kval = k0 + 2 * q < d.K;
                for (int row = rsub; row < d.M + d.N; row += kLoaders / 16)
                {
                    if (!live)
                        break;
                    const bool isA = row < d.M;
                    const int r = isA ? row : row - d.M;
                    const uint8_t *src = isA ? Ab + ((int64_t)r * d.lda + k0 + 2 * q) * 8
                                             : Bb + ((int64_t)r * d.ldb + k0 + 2 * q) * 8;
                    const uint32_t dst = (isA ? sa : sb) + qb * kBox + r * 64 + ((qt ^ ((r >> 1) & 3)) << 4);
                    cp16(dst, kval ? (const void *)src : (const void *)Ab, kval);
                }
                cp_arrive_on(&full[s]);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        return;
    }

    // ---- compute: warp w owns 16 x 16 sub-tiles w, w + 14, ... of each problem ----
    const int gq = lane >> 2, tq = lane & 3;
    const double alpha = p.alpha, beta = p.beta;
    double *C = reinterpret_cast<double *>(p.C);
    int j = 0;
    for (int i = begin; i < end; ++i)
    {
        const SDesc d = get_desc(dcache, p.desc, begin, i);
        const int nsn = (d.N + 15) >> 4, T = ((d.M + 15) >> 4) * nsn;
        double acc[kMaxSub][2][4];
#pragma unroll
        for (int u = 0; u < kMaxSub; ++u)
#pragma unroll
            for (int n = 0; n < 2; ++n)
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    acc[u][n][e] = 0.0;
        bool ok = true;
        for (int k0 = 0; k0 < d.K; k0 += kKChunk, ++j)
        {
            const int s = j % kSlots;
            if (!__all_sync(0xffffffffu, tc::mbar_wait_bounded(&full[s], (j / kSlots) & 1, limit)))
            {
                gf_flag(2);
                ok = false;
                break;
            }
            const uint32_t sa = slots + s * kSlotBytes, sb = sa + kOper;
            const int ksteps = (min(kKChunk, d.K - k0) + 7) >> 3;
            for (int it = 0; it < p.num_iter; ++it)
            {
#pragma unroll
                for (int u = 0; u < kMaxSub; ++u)
                {
                    const int t = warp + u * kComputeWarps;
                    if (t < T)
                    {
                        const int c0 = (t % nsn) * 16;
                        subtile_chunk(sa, sb, (t / nsn) * 16, c0, c0 + 8 < d.N, ksteps, gq, tq, acc[u]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0)
                tc::mbar_arrive(&empty[s]);
        }
        if (!ok)
            break;
        double *Cb = C + d.c_off;
        const bool vec = ((d.ldc & 1) == 0) && ((d.c_off & 1) == 0);
#pragma unroll
        for (int u = 0; u < kMaxSub; ++u)
        {
            const int t = warp + u * kComputeWarps;
            if (t >= T)
                continue;
            const int r0 = (t / nsn) * 16, c0 = (t % nsn) * 16;
#pragma unroll
            for (int n = 0; n < 2; ++n)
            {
                const int col = c0 + 8 * n + 2 * tq;
                store_f64_pair(Cb, d.M, d.N, d.ldc, vec, alpha, beta, r0 + gq, col, acc[u][n][0], acc[u][n][1]);
                store_f64_pair(Cb, d.M, d.N, d.ldc, vec, alpha, beta, r0 + gq + 8, col, acc[u][n][2], acc[u][n][3]);
            }
        }
    }
}

} // namespace

const void *grouped_f64s_fn() { return (const void *)&grouped_f64_kernel; }

int grouped_f64s_threads() { return kThreads; }

int grouped_f64s_smem() { return kSmem; }

int grouped_f64s_launch(const GroupedParams &p, int ctas, cudaStream_t s)
{
    GfParams gp{};
    gp.p = p;
    gp.timeout_ns = (uint64_t)(2e9 + (double)p.num_iter * 1e6); // generous: a chunk takes microseconds
    void *args[] = {&gp};
    cudaError_t e = cudaLaunchKernel(grouped_f64s_fn(), dim3(ctas), dim3(kThreads), args, kSmem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(grouped_f64_kernel)");
    return KAMI_OK;
}

int grouped_f64s_read_error(int *flag)
{
    int v = 0, z = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_gf64_error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_gf64_error, &z, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "reading the grouped FP64 status");
    *flag = v;
    return KAMI_OK;
}

} // namespace kami
