// grouped_tc05.cu -- the uneven (grouped) batched GEMM on the 5th-generation
// tensor cores: thousands of FP16/BF16 problems of different M, N, K (each
// <= 128) in one persistent launch, accumulators in tensor memory.
//
// The warp-grid kernel of grouped.cu spends thousands of instructions per
// problem on fragment loads, MMA issue and partition bookkeeping in eight
// warps that each hold a slice of the tile; at these sizes the SM is
// issue-bound long before HBM or the tensor pipe.  Here the MMA of a whole
// problem is a handful of tcgen05.mma issued by one thread, so the
// instruction budget goes to moving bytes.  Two CTAs per SM each walk their
// share of a longest-first schedule (the same host plan as the warp-grid
// kernel) with three warp roles:
//   warps 8-11 loaders: each K chunk of 64 (A rows, then B rows) is copied
//              with 16-byte cp.async straight into the 128-byte-swizzled
//              K-major layout the MMA reads (row r at r * 128, 16-byte chunk
//              c at c ^ (r % 8)), into a ring of kSlots stages; every loader
//              thread's arrival on full[s] is attached to its copies
//              (cp.async.mbarrier.arrive), so a chunk publishes itself when
//              it lands and the loaders only ever wait for a free stage
//              (publishing after a fixed look-ahead tied each chunk's MMAs
//              to the completion of the previous chunk's and measured 13 %
//              slower on the uneven workload);
//   warp 12    lane 0 waits for a chunk, fences the loaders' (generic-proxy)
//              writes for the tensor core's async-proxy reads, and issues
//              the chunk's MMAs -- M = 64 or 128 rows of TMEM
//              lanes (rows of A past M are never stored), N rounded up to
//              16 -- into one of the CTA's two TMEM accumulators (256
//              columns; the SM's other CTA holds the other 256),
//              frees the stage with tcgen05.commit and, after the problem's
//              last chunk, hands the accumulator to the epilogue; warp 12
//              also owns the TMEM allocation;
//   warps 0-3, 4-7  two epilogue groups taking alternate problems (warp w
//              reads TMEM lanes 32 (w % 4) .. + 31): TMEM -> registers -> C
//              (through a per-warp transpose tile, so stores are
//              row-contiguous), alpha / beta and the output type applied,
//              then the accumulator is freed.  Small problems are bound by
//              this hand-off chain (MMA completion, accumulator read-out),
//              so two accumulators and two groups per CTA, and two CTAs per
//              SM, keep several in flight.
// The CTA's descriptors (up to kDescCache of them) are copied to shared
// memory once at the start: read from global memory per problem, their
// latency sat on the loaders' path once per problem and bound small problems.
// Columns of a partial last k-step (K a multiple of 8, not of 16) are
// zero-filled by the copies; stale rows past M or N only reach rows and
// columns of the accumulator that are never stored.
// Every mbarrier wait is bounded; a timeout sets g_gtc_error, ends that
// role's loop, and the CTA waits (bounded) for its own copies and MMAs
// before it frees tensor memory and exits.
#include <cstdint>

#include "grouped.cuh"
#include "kami_common.cuh"
#include "tc05_epi.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device status of the bounded waits (read and cleared by kami_device_status)
__device__ int g_gtc_error = 0;

namespace {

// Two CTAs per SM, each with its own loaders, MMA thread, epilogue groups and
// rings: the per-problem hand-off chain (chunk lands -> one thread issues and
// commits -> accumulator drained) is latency-bound, so two independent chains
// per SM overlap where one CTA with deeper rings could not (20000 uneven
// FP16 problems: 0.096 ms, against 0.117-0.121 ms with one CTA of six stages
// and four accumulators per SM, and 0.172 ms with one CTA of this size).
constexpr int kCtasPerSm = 2;
constexpr int kSlots = 2;                 // shared-memory stages of one K chunk each
constexpr int kSlotBytes = 32768;         // A: 128 rows x 128 B, then B: 128 rows x 128 B
constexpr int kEpiGroups = 2;            // epilogue groups of 4 warps: warps 0-3 and 4-7
constexpr int kEpiWarps = 4 * kEpiGroups;
constexpr int kLoadWarps = 4;             // warps 8-11
constexpr int kMmaWarp = kEpiWarps + kLoadWarps;
constexpr int kThreads = (kMmaWarp + 1) * 32;
constexpr int kLoaders = kLoadWarps * 32;
constexpr int kAccs = 2;                  // TMEM accumulators (256 of the SM's 512 columns)
constexpr int kAccCols = 128;             // TMEM columns of one accumulator (N <= 128)
constexpr int kTmemCols = kAccs * kAccCols;
constexpr int kBars = 2 * kSlots + 2 * kAccs + 1;

// compact copy of a GroupedDesc for the shared-memory cache.  pk (the
// descriptor's cfg field in tcgen05 plans): the problem's row offset in its
// work item's A tile (bits 0-7), its column offset in the item's B tile and
// accumulator (bits 8-15, a multiple of 16) and the item's problem count
// (bits 16-23); the problems of an item are consecutive descriptors.
struct SDesc
{
    int M, N, K, lda, ldb, ldc, pk, it; // it: the item's extent (see item_at)
    int64_t a_off, b_off, c_off;
};
__device__ __forceinline__ int pk_m(int pk) { return pk & 0xff; }
__device__ __forceinline__ int pk_n(int pk) { return (pk >> 8) & 0xff; }
__device__ __forceinline__ int pk_count(int pk) { return max(1, (pk >> 16) & 0xff); }
constexpr int kMaxPack = 4; // problems per work item
constexpr int kDescCache = 96; // descriptors per CTA held in shared memory
constexpr int kSmem =
    kSlots * kSlotBytes + kEpiWarps * kEpiTileBytes + kDescCache * (int)sizeof(SDesc) + kBars * 8 + 16 + 1024;
static_assert(kCtasPerSm * (kSmem + 1024) <= 233472, "grouped tcgen05 kernel: two CTAs must fit one SM's shared memory");
static_assert(kCtasPerSm * kTmemCols <= 512, "grouped tcgen05 kernel: two CTAs must fit one SM's tensor memory");
static_assert(kEpiGroups <= kAccs, "grouped tcgen05 kernel: more epilogue groups than accumulators");

// descriptor i of the CTA's list: from the cache when it is there
__device__ __forceinline__ SDesc get_desc(const SDesc *cache, const GroupedDesc *g, int begin, int i)
{
    if (i - begin < kDescCache)
        return cache[i - begin];
    const GroupedDesc d = g[i];
    return SDesc{d.M, d.N, d.K, d.lda, d.ldb, d.ldc, d.cfg, d.ext, d.a_off, d.b_off, d.c_off};
}

// extent of the work item starting at descriptor i, precomputed by the plan
// in every member's descriptor (GroupedDesc::ext = n | Mt << 3 | (Nt / 16)
// << 11 | Kt << 15): its problem count, rows of A (Mt), rows of B with each
// problem's rounded up to 16 (Nt) and its largest K
struct Item
{
    int n, Mt, Nt, Kt;
};
__device__ __forceinline__ Item item_at(const SDesc *cache, const GroupedDesc *g, int begin, int i)
{
    const int v = i - begin < kDescCache ? cache[i - begin].it : g[i].ext;
    return Item{max(1, v & 7), (v >> 3) & 0xff, ((v >> 11) & 0xf) * 16, (v >> 15) & 0xff};
}

struct GtParams
{
    GroupedParams p;
    uint64_t timeout_ns;
};

__device__ __forceinline__ void gt_flag(int code) { atomicExch(&g_gtc_error, code); }

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
// order shared-memory writes this thread has observed before its later
// async-proxy (tensor core) reads
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ int mma_m(int M) { return M <= 64 ? 64 : 128; }
__device__ __forceinline__ int mma_n(int N) { return (N + 15) & ~15; }

// PACKED: the plan has work items of several problems (each role walks the
// items); otherwise every item is one problem and the roles index problems
// directly.
template <bool BF16, bool PACKED>
__global__ void __launch_bounds__(kThreads, kCtasPerSm) grouped_tc05_kernel(const __grid_constant__ GtParams gp)
{
    const GroupedParams &p = gp.p;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment of the swizzle atoms
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    float *epi = reinterpret_cast<float *>(smem + kSlots * kSlotBytes);
    SDesc *dcache = reinterpret_cast<SDesc *>(smem + kSlots * kSlotBytes + kEpiWarps * kEpiTileBytes);
    uint64_t *full = reinterpret_cast<uint64_t *>(dcache + kDescCache);
    uint64_t *empty = full + kSlots;
    uint64_t *accf = empty + kSlots; // accumulator b holds a finished product
    uint64_t *acce = accf + kAccs;   // accumulator b has been read out
    uint64_t *fin = acce + kAccs;    // every MMA of this CTA has completed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(fin + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int begin = p.cta_begin[blockIdx.x], end = p.cta_begin[blockIdx.x + 1];
    const uint64_t limit = gp.timeout_ns;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kSlots; ++s)
        {
            tc::mbar_init(&full[s], kLoaders);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < kAccs; ++b)
        {
            tc::mbar_init(&accf[b], 1);
            tc::mbar_init(&acce[b], 4); // the four warps of one epilogue group
        }
        tc::mbar_init(fin, 1);
        tc::fence_mbar_init();
    }
    if (warp == kMmaWarp)
    {
        tc::tmem_alloc(tmem_slot, kTmemCols);
        tc::tmem_relinquish();
    }
    for (int i = threadIdx.x; i < end - begin && i < kDescCache; i += kThreads)
    {
        const GroupedDesc d = p.desc[begin + i];
        dcache[i] = SDesc{d.M, d.N, d.K, d.lda, d.ldb, d.ldc, d.cfg, d.ext, d.a_off, d.b_off, d.c_off};
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp >= kEpiWarps && warp < kMmaWarp)
    {
        // ---- loaders ----
        const int tl = threadIdx.x - kEpiWarps * 32;
        const int c = tl & 7, rsub = tl >> 3; // 16-byte chunk of a row; first row
        const uint8_t *A = reinterpret_cast<const uint8_t *>(p.A);
        const uint8_t *B = reinterpret_cast<const uint8_t *>(p.B);
        const uint32_t slots = tc::smem_u32(smem);
        int j = 0;
        bool ok = true;
        if constexpr (!PACKED)
            for (int i = begin; i < end && ok; ++i)
            {
                const SDesc d = get_desc(dcache, p.desc, begin, i);
                const uint8_t *Ab = A + d.a_off * 2, *Bb = B + d.b_off * 2;
                for (int k0 = 0; k0 < d.K; k0 += 64, ++j)
                {
                    const int s = j % kSlots;
                    if (j >= kSlots && !tc::mbar_wait_bounded(&empty[s], ((j / kSlots) - 1) & 1, limit))
                    {
                        gt_flag(1);
                        ok = false;
                        break;
                    }
                    const uint32_t sa = slots + s * kSlotBytes, sb = sa + kSlotBytes / 2;
                    // 16-byte chunks per row that the MMAs read: whole k-steps of 16
                    const int kc = ((min(64, d.K - k0) + 15) >> 4) * 2;
                    const bool live = c < kc;
                    const bool kval = k0 + 8 * c < d.K;
                    for (int row = rsub; row < d.M + d.N; row += kLoaders / 8)
                    {
                        if (!live)
                            break;
                        const bool isA = row < d.M;
                        const int r = isA ? row : row - d.M;
                        const uint8_t *src = isA ? Ab + ((int64_t)r * d.lda + k0 + 8 * c) * 2
                                                 : Bb + ((int64_t)r * d.ldb + k0 + 8 * c) * 2;
                        const uint32_t dst = (isA ? sa : sb) + r * 128 + ((c ^ (r & 7)) << 4);
                        cp16(dst, kval ? (const void *)src : (const void *)Ab, kval);
                    }
                    // this thread's arrival on full[s] happens when its copies land
                    cp_arrive_on(&full[s]);
                }
            }
        else
        for (int i = begin; i < end && ok;)
        {
            // the work item's problems: A rows [m0, m1) and B rows [n0, n0 + N)
            // of the item's tiles belong to problem t
            const Item itm = item_at(dcache, p.desc, begin, i);
            int mlo[kMaxPack], nlo[kMaxPack], nhi[kMaxPack], kk[kMaxPack], lda[kMaxPack], ldb[kMaxPack];
            int64_t aoff[kMaxPack], boff[kMaxPack];
#pragma unroll
            for (int t = 0; t < kMaxPack; ++t)
                if (t < itm.n)
                {
                    const SDesc d = get_desc(dcache, p.desc, begin, i + t);
                    mlo[t] = pk_m(d.pk);
                    nlo[t] = pk_n(d.pk);
                    nhi[t] = nlo[t] + d.N;
                    kk[t] = d.K;
                    lda[t] = d.lda;
                    ldb[t] = d.ldb;
                    aoff[t] = d.a_off;
                    boff[t] = d.b_off;
                }
            i += itm.n;
            for (int k0 = 0; k0 < itm.Kt; k0 += 64, ++j)
            {
                const int s = j % kSlots;
                if (j >= kSlots && !tc::mbar_wait_bounded(&empty[s], ((j / kSlots) - 1) & 1, limit))
                {
                    gt_flag(1);
                    ok = false;
                    break;
                }
                const uint32_t sa = slots + s * kSlotBytes, sb = sa + kSlotBytes / 2;
                // 16-byte chunks per row that the MMAs read: whole k-steps of 16
                const int kc = ((min(64, itm.Kt - k0) + 15) >> 4) * 2;
                const bool live = c < kc;
                // member by member, so each copy's base, leading dimension and
                // K bound are loop constants; this thread copies chunk c of the
                // rows r = rsub (mod 16) of every member's A and B rows
                if (live)
                {
#pragma unroll
                    for (int t = 0; t < kMaxPack; ++t)
                    {
                        if (t >= itm.n)
                            break;
                        const bool kval = k0 + 8 * c < kk[t];
                        const int a0 = mlo[t], a1 = t + 1 < itm.n ? mlo[t + 1 < kMaxPack ? t + 1 : t] : itm.Mt;
                        const uint8_t *Ab = A + (aoff[t] + k0 + 8 * c) * 2;
                        for (int r = a0 + ((rsub - a0) & (kLoaders / 8 - 1)); r < a1; r += kLoaders / 8)
                            cp16(sa + r * 128 + ((c ^ (r & 7)) << 4),
                                 kval ? (const void *)(Ab + (int64_t)(r - a0) * lda[t] * 2) : (const void *)A, kval);
                        const int b0 = nlo[t], b1 = nhi[t]; // rows past N in the 16-row group are never read
                        const uint8_t *Bb = B + (boff[t] + k0 + 8 * c) * 2;
                        for (int r = b0 + ((rsub - b0) & (kLoaders / 8 - 1)); r < b1; r += kLoaders / 8)
                            cp16(sb + r * 128 + ((c ^ (r & 7)) << 4),
                                 kval ? (const void *)(Bb + (int64_t)(r - b0) * ldb[t] * 2) : (const void *)A, kval);
                    }
                }
                // this thread's arrival on full[s] happens when its copies land
                cp_arrive_on(&full[s]);
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    else if (warp == kMmaWarp)
    {
        // ---- MMA issue (one thread) ----
        if (lane == 0)
        {
            const uint32_t slots = tc::smem_u32(smem);
            int j = 0, pi = 0;
            bool ok = true;
            for (int i = begin; i < end && ok; ++pi)
            {
                const Item itm = item_at(dcache, p.desc, begin, i);
                i += itm.n;
                const SDesc d{itm.Mt, itm.Nt, itm.Kt, 0, 0, 0, 0, 0, 0, 0, 0}; // the item as one problem
                const uint32_t idesc = tc::idesc_f16(BF16, mma_m(d.M), mma_n(d.N));
                const int b = pi % kAccs;
                const uint32_t acc = tmem + b * kAccCols;
                if (pi >= kAccs && !tc::mbar_wait_bounded(&acce[b], ((pi / kAccs) - 1) & 1, limit))
                {
                    gt_flag(2);
                    break;
                }
                tc::tc_fence_after();
                for (int k0 = 0; k0 < d.K; k0 += 64, ++j)
                {
                    const int s = j % kSlots;
                    if (!tc::mbar_wait_bounded(&full[s], (j / kSlots) & 1, limit))
                    {
                        gt_flag(3);
                        ok = false;
                        break;
                    }
                    // the loaders' copies are generic-proxy writes: order them
                    // before the tensor core's (async-proxy) reads
                    fence_async_smem();
                    tc::tc_fence_after();
                    const uint32_t sa = slots + s * kSlotBytes, sb = sa + kSlotBytes / 2;
                    const int ksteps = (min(64, d.K - k0) + 15) >> 4;
                    for (int it = 0; it < p.num_iter; ++it)
                        for (int ks = 0; ks < ksteps; ++ks)
                            tc::mma_f16_ss(acc, tc::desc_kmajor_sw128(sa + ks * 32),
                                           tc::desc_kmajor_sw128(sb + ks * 32), idesc,
                                           (k0 > 0 || it > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_commit(&empty[s]); // the stage is free once these MMAs are done
                }
                if (!ok)
                    break;
                tc::mma_commit(&accf[b]);
            }
            tc::mma_commit(fin);
            if (!tc::mbar_wait_bounded(fin, 0, limit))
                gt_flag(4);
        }
        __syncwarp();
    }
    else
    {
        // ---- epilogue: group warp / 4 takes problems pi = group, + 2, ...;
        //      warp w reads TMEM lanes 32 (w % 4) .. + 31 ----
        const int grp = warp >> 2, q = warp & 3;
        float *T = epi + warp * (kEpiTileBytes / 4);
        const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
        GemmArgs g{};
        g.out_type = p.out_type;
        g.alpha = p.alpha;
        g.beta = p.beta;
        const int osz = p.out_type == KAMI_F32 ? 4 : 2;
        int i = begin; // first descriptor of item pi
        for (int pi = PACKED ? 0 : grp; i < end; pi += PACKED ? 1 : kEpiGroups)
        {
            int i0;
            Item itm;
            if constexpr (PACKED)
            {
                itm = item_at(dcache, p.desc, begin, i);
                i0 = i;
                i += itm.n;
                if (pi % kEpiGroups != grp)
                    continue;
            }
            else
            {
                i0 = begin + pi;
                if (i0 >= end)
                    break;
                itm = item_at(dcache, p.desc, begin, i0);
            }
            const int b = pi % kAccs;
            // tcgen05.ld is .sync.aligned: the outcome must be warp-uniform
            const bool done = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&accf[b], (pi / kAccs) & 1, limit));
            tc::tc_fence_after();
            if (!done)
            {
                gt_flag(5);
                break;
            }
            // this warp's band of accumulator rows: 32 rows (M = 128 MMAs) or
            // 16 (M = 64, rows 16q .. in lanes 32q ..)
            const bool m128 = itm.Mt > 64;
            const int row_base = m128 ? q * 32 : q * 16, nrows = m128 ? 32 : 16;
            for (int t = 0; t < itm.n; ++t)
            {
                const SDesc d = get_desc(dcache, p.desc, begin, i0 + t);
                const int m0 = pk_m(d.pk), n0 = pk_n(d.pk);
                if (m0 >= row_base + nrows || m0 + d.M <= row_base)
                    continue; // none of this problem's rows in the band
                g.M = d.M;
                g.N = d.N;
                g.ldc = d.ldc;
                g.c_vec = ((d.ldc & 1) == 0) && ((d.c_off & 1) == 0);
                g.c_vec4 = ((d.ldc & 3) == 0) && ((d.c_off & 3) == 0);
                void *Cb = reinterpret_cast<char *>(p.C) + d.c_off * osz;
                const int bn = mma_n(d.N);
                for (int c0 = 0; c0 < bn; c0 += 16)
                {
                    uint32_t v[16];
                    tc::tmem_ld16(tmem + b * kAccCols + lane_addr + n0 + c0, v);
                    tc::tmem_ld_wait();
                    tc::tmem_regs_ready(v);
                    float f[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        f[e] = __uint_as_float(v[e]);
                    // band row lr is the problem's row row_base - m0 + lr
                    store_chunk<PACKED>(g, Cb, f, row_base - m0, nrows, c0, T);
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0)
                tc::mbar_arrive(&acce[b]);
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp)
    {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

} // namespace

const void *grouped_tc05_fn(bool bf16, bool packed)
{
    if (packed)
        return bf16 ? (const void *)&grouped_tc05_kernel<true, true> : (const void *)&grouped_tc05_kernel<false, true>;
    return bf16 ? (const void *)&grouped_tc05_kernel<true, false> : (const void *)&grouped_tc05_kernel<false, false>;
}

int grouped_tc05_threads() { return kThreads; }

// CTAs of the kernel that share one SM (its shared memory, tensor memory and
// registers are sized for two); the occupancy query reports one for it
int grouped_tc05_ctas_per_sm() { return kCtasPerSm; }

int grouped_tc05_smem() { return kSmem; }

int grouped_tc05_launch(const GroupedParams &p, bool bf16, bool packed, int ctas, cudaStream_t s)
{
    GtParams gp{};
    gp.p = p;
    gp.timeout_ns = (uint64_t)(2e9 + (double)p.num_iter * 1e6); // generous: a chunk takes microseconds
    void *args[] = {&gp};
    cudaError_t e = cudaLaunchKernel(grouped_tc05_fn(bf16, packed), dim3(ctas), dim3(kThreads), args, kSmem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(grouped_tc05_kernel)");
    return KAMI_OK;
}

int grouped_tc05_read_error(int *flag)
{
    int v = 0, z = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_gtc_error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_gtc_error, &z, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "reading the grouped tcgen05 status");
    *flag = v;
    return KAMI_OK;
}

} // namespace kami
