// spgemm.cu -- block SpGEMM C = A * B on BSR matrices with 16 x 16 tiles.
//
// Reference path (src/sparse/spgemm/2d/block_spgemm_2d_half_mma.cu):
//   spgemm_symbolic_kernel (:58-86)  per block-row a dense flag array over
//                                    the block columns, then a count;
//   thrust::exclusive_scan (:806)    RowPtrC;
//   cudaMemcpy D2H of nnzC (:808)    so the host can allocate ColIdxC/ValC;
//   spgemm_symbolic_col_kernel (:88-116)  ColIdxC, ascending per row;
//   block_spgemm_2d_half_mma (:171-555)   numeric: per warp, local CSR
//                                    slices, staged exchange, and a linear
//                                    search for each product's C column.
//
// This implementation keeps the same three phases, the same outputs (RowPtrC,
// ColIdxC ascending per row, ValC tiles in ColIdxC order) and the same tile
// layouts (A and B tiles row-major 16 x 16, B used as K x N), re-designed for
// B200 and for large matrices (the reference handles one <= 192^2 block per
// CTA):
//   * symbolic: one warp per block-row builds the row's column set as a
//     bitmap in shared memory (shared atomics), counts it with popc, and the
//     column fill walks the bitmap words in order (ascending by
//     construction);  the scan is a single-CTA in-place scan; no scratch.
//   * numeric: one warp per C tile (i, j).  Its lanes take the nonzero
//     blocks A(i, k) of row i, binary-search j in block-row k of B (column
//     indices sorted ascending, as the reference generator emits them), and
//     the warp accumulates every matching A(i,k) * B(k,j) with two
//     m16n8k16 MMAs (FP32 accumulation) in ascending k -- the order of the
//     reference's sparse accumulator.  No C tile is touched twice, so the
//     kernel writes C once (the HBM floor of the product).
#include <atomic>
#include <cstdint>
#include <mutex>

#include "kami_common.cuh"
#include "spgemm_tiles.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// Grid barriers of the fused symbolic pass: [slot][0] arrivals, [slot][1]
// generation.  Each launch takes the next slot (zeroed on its stream just
// before it), so launches in flight on different streams do not share one.
constexpr int kFuseSlots = 64;
__device__ unsigned int g_spg_bar[kFuseSlots][2];
// device status of the fused pass's bounded barrier waits (read and cleared
// by kami_device_status)
__device__ int g_spg_error = 0;
// Look-back flags of the single-pass symbolic kernel: one 64-bit word per
// chunk of block-rows, [epoch (31 bits) | inclusive (1 bit) | value (32
// bits)].  Each launch takes the next slot and a new epoch, so a word left by
// an earlier launch never reads as ready and nothing is reset between
// launches.
constexpr int kLbSlots = 16;
constexpr int kLbMaxChunks = 16384;
__device__ unsigned long long g_spg_flags[kLbSlots][kLbMaxChunks];

namespace {

using namespace sptile;

constexpr int kBsr = 16;

// ---------------------------------------------------------------------------
// symbolic
// ---------------------------------------------------------------------------
__device__ __forceinline__ void build_row_bitmap(uint32_t *bm, int words, int row, const int *__restrict__ rpa,
                                                 const int *__restrict__ cia, const int *__restrict__ rpb,
                                                 const int *__restrict__ cib, int lane)
{
    for (int w = lane; w < words; w += 32)
        bm[w] = 0u;
    __syncwarp();
    const int a0 = rpa[row], a1 = rpa[row + 1];
    for (int e = a0 + lane; e < a1; e += 32)
    {
        const int k = cia[e];
        const int b1 = rpb[k + 1];
        for (int b = rpb[k]; b < b1; ++b)
        {
            const int c = cib[b];
            atomicOr(&bm[c >> 5], 1u << (c & 31));
        }
    }
    __syncwarp();
}

__global__ void spgemm_count_kernel(int mb, int nb, const int *__restrict__ rpa, const int *__restrict__ cia,
                                    const int *__restrict__ rpb, const int *__restrict__ cib, int *__restrict__ rpc)
{
    extern __shared__ uint32_t bm_all[];
    const int words = (nb + 31) >> 5;
    const int wpc = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    uint32_t *bm = bm_all + (threadIdx.x >> 5) * words;
    for (int row = blockIdx.x * wpc + (threadIdx.x >> 5); row < mb; row += gridDim.x * wpc)
    {
        build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
        int cnt = 0;
        for (int w = lane; w < words; w += 32)
            cnt += __popc(bm[w]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0)
            rpc[row] = cnt;
        __syncwarp();
    }
}

// In-place exclusive scan of rpc[0..n-1] by one CTA of 1024 threads; the
// total lands in rpc[n].
__global__ void __launch_bounds__(1024) spgemm_scan_kernel(int n, int *__restrict__ rpc)
{
    __shared__ int warp_sums[32];
    __shared__ int carry_s;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    if (t == 0)
        carry_s = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024)
    {
        const int i = base + t;
        const int v = i < n ? rpc[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0)
        {
            int s = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o)
                    s += y;
            }
            warp_sums[lane] = s; // inclusive over warps
        }
        __syncthreads();
        const int carry = carry_s;
        const int incl = x + (wid > 0 ? warp_sums[wid - 1] : 0);
        if (i < n)
            rpc[i] = carry + incl - v;
        __syncthreads();
        if (t == 1023)
            carry_s = carry + incl;
        __syncthreads();
    }
    if (t == 0)
        rpc[n] = carry_s;
}

__global__ void spgemm_colfill_kernel(int mb, int nb, const int *__restrict__ rpa, const int *__restrict__ cia,
                                      const int *__restrict__ rpb, const int *__restrict__ cib,
                                      const int *__restrict__ rpc, int *__restrict__ cic, int64_t cap)
{
    extern __shared__ uint32_t bm_all[];
    const int words = (nb + 31) >> 5;
    const int wpc = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    uint32_t *bm = bm_all + (threadIdx.x >> 5) * words;
    for (int row = blockIdx.x * wpc + (threadIdx.x >> 5); row < mb; row += gridDim.x * wpc)
    {
        build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
        int out = rpc[row];
        for (int w0 = 0; w0 < words; w0 += 32)
        {
            const int w = w0 + lane;
            uint32_t bits = w < words ? bm[w] : 0u;
            const int c = __popc(bits);
            int pre = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, pre, o);
                if (lane >= o)
                    pre += y;
            }
            int pos = out + pre - c;
            while (bits)
            {
                const int b = __ffs(bits) - 1;
                if (pos < cap) // entries beyond the caller's capacity are not written
                    cic[pos] = w * 32 + b;
                ++pos;
                bits &= bits - 1;
            }
            out += __shfl_sync(0xffffffffu, pre, 31);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// The symbolic pass in ONE launch: count, scan and column fill as phases of a
// cooperative persistent kernel, separated by grid barriers (the reference
// runs three launches with a device-to-host copy of nnzC between them,
// block_spgemm_2d_half_mma.cu:805-812).  A cooperative launch keeps every CTA
// resident, so the barrier cannot wait for a CTA that never runs; its waits
// are bounded all the same, and a timeout sets g_spg_error and ends the CTA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t spg_globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Every CTA of the grid arrives; returns false (block-uniform) on a timeout.
__device__ __forceinline__ bool spg_grid_barrier(unsigned int *bar, uint64_t limit_ns)
{
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0)
    {
        volatile unsigned int *gen = bar + 1;
        const unsigned int g0 = *gen;
        __threadfence(); // the generation read and this CTA's writes precede its arrival
        if (atomicAdd(bar, 1u) == gridDim.x - 1)
        {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
        else
        {
            const uint64_t t0 = spg_globaltimer();
            while (*gen == g0)
            {
                if (spg_globaltimer() - t0 > limit_ns)
                {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    return __syncthreads_and(ok) != 0;
}

// In-place exclusive scan of rpc[0..n-1] by the calling CTA; total in rpc[n].
__device__ __forceinline__ void spg_block_scan(int n, int *__restrict__ rpc)
{
    __shared__ int warp_sums[32];
    __shared__ int carry_s;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5, nw = blockDim.x >> 5;
    if (t == 0)
        carry_s = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x)
    {
        const int i = base + t;
        const int v = i < n ? rpc[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_sums[wid] = x;
        __syncthreads();
        if (wid == 0)
        {
            int sum = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, sum, o);
                if (lane >= o)
                    sum += y;
            }
            if (lane < nw)
                warp_sums[lane] = sum; // inclusive over warps
        }
        __syncthreads();
        const int carry = carry_s;
        const int incl = x + (wid > 0 ? warp_sums[wid - 1] : 0);
        if (i < n)
            rpc[i] = carry + incl - v;
        __syncthreads();
        if (t == (int)blockDim.x - 1)
            carry_s = carry + incl;
        __syncthreads();
    }
    if (t == 0)
        rpc[n] = carry_s;
}

// keep_rows > 0: every warp holds at most keep_rows block-rows and keeps
// each row's bitmap in shared memory from phase 1 to phase 3 (the column fill
// then re-reads neither A's row nor B's rows); 0: one bitmap per warp,
// rebuilt in phase 3.
__global__ void spgemm_symbolic_fused_kernel(int mb, int nb, const int *__restrict__ rpa,
                                             const int *__restrict__ cia, const int *__restrict__ rpb,
                                             const int *__restrict__ cib, int *__restrict__ rpc,
                                             int *__restrict__ cic, int64_t cap, unsigned int *bar,
                                             uint64_t limit_ns, int keep_rows)
{
    extern __shared__ uint32_t bm_all[];
    const int words = (nb + 31) >> 5;
    const int wpc = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    const int keep = keep_rows > 0;
    uint32_t *bm_warp = bm_all + (size_t)(threadIdx.x >> 5) * (keep ? keep_rows : 1) * words;
    // phase 1: nnz of every C block-row
    int r = 0;
    for (int row = blockIdx.x * wpc + (threadIdx.x >> 5); row < mb; row += gridDim.x * wpc, ++r)
    {
        uint32_t *bm = bm_warp + (keep ? r * words : 0);
        build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
        int cnt = 0;
        for (int w = lane; w < words; w += 32)
            cnt += __popc(bm[w]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0)
            rpc[row] = cnt;
        __syncwarp();
    }
    if (!spg_grid_barrier(bar, limit_ns))
    {
        if (threadIdx.x == 0)
            atomicExch(&g_spg_error, 1);
        return;
    }
    // phase 2: exclusive scan into RowPtrC (one CTA; the others wait)
    if (blockIdx.x == 0)
        spg_block_scan(mb, rpc);
    if (!spg_grid_barrier(bar, limit_ns))
    {
        if (threadIdx.x == 0)
            atomicExch(&g_spg_error, 2);
        return;
    }
    if (cap == 0)
        return;
    // phase 3: ColIdxC, ascending per block-row, up to the capacity
    r = 0;
    for (int row = blockIdx.x * wpc + (threadIdx.x >> 5); row < mb; row += gridDim.x * wpc, ++r)
    {
        uint32_t *bm = bm_warp + (keep ? r * words : 0);
        if (!keep)
            build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
        int out = rpc[row];
        for (int w0 = 0; w0 < words; w0 += 32)
        {
            const int w = w0 + lane;
            uint32_t bits = w < words ? bm[w] : 0u;
            const int c = __popc(bits);
            int pre = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, pre, o);
                if (lane >= o)
                    pre += y;
            }
            int pos = out + pre - c;
            while (bits)
            {
                const int b = __ffs(bits) - 1;
                if (pos < cap)
                    cic[pos] = w * 32 + b;
                ++pos;
                bits &= bits - 1;
            }
            out += __shfl_sync(0xffffffffu, pre, 31);
        }
        __syncwarp();
    }
}


// ---------------------------------------------------------------------------
// The symbolic pass in one launch and one pass: chunk c of block-rows (R
// consecutive rows, c = blockIdx.x, + gridDim.x, ...) is counted by its CTA,
// which publishes the chunk's total, finds the exclusive prefix of the
// chunks before it by a decoupled look-back over their flags (a chunk's flag
// carries its own total, or the inclusive prefix once its CTA found it), writes
// RowPtrC for its rows and fills their ColIdxC.  No grid barrier: a chunk's
// fill starts as soon as its prefix is known.  The launch is cooperative, so
// every chunk's CTA is resident and a look-back never waits for a CTA that
// does not run; the waits are bounded all the same (a timeout sets
// g_spg_error).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long lb_word(unsigned epoch, bool incl, int value)
{
    return ((unsigned long long)epoch << 33) | ((unsigned long long)incl << 32) | (uint32_t)value;
}

// Exclusive prefix of chunk c (c > 0), by warp 0 of its CTA: lane l reads the
// flag of chunk p - l for a window of 32 predecessors; the window's sum up to
// and including the nearest inclusive flag ends the walk.  Returns false on
// a timeout.
__device__ __forceinline__ bool lb_prefix(const unsigned long long *flags, int c, unsigned epoch, uint64_t limit_ns,
                                          int lane, int *prefix)
{
    int acc = 0;
    int p = c - 1;
    const uint64_t t0 = spg_globaltimer();
    while (p >= 0)
    {
        const int q = p - lane;
        unsigned long long w = 0;
        bool ready = true;
        if (q >= 0)
        {
            w = *reinterpret_cast<const volatile unsigned long long *>(&flags[q]);
            ready = (unsigned)(w >> 33) == epoch;
        }
        const bool incl = q >= 0 && ready && ((w >> 32) & 1ull);
        const unsigned incl_mask = __ballot_sync(0xffffffffu, incl);
        // lanes up to the nearest inclusive flag (or all 32 / down to chunk 0)
        const int last = incl_mask ? __ffs(incl_mask) - 1 : 31;
        const bool need = lane <= last && q >= 0;
        if (!__all_sync(0xffffffffu, !need || ready))
        {
            if (spg_globaltimer() - t0 > limit_ns)
                return false;
            __nanosleep(32);
            continue; // a predecessor has not published yet: read the window again
        }
        int v = need ? (int)(uint32_t)w : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        acc += v;
        if (incl_mask)
            break;
        p -= 32;
    }
    *prefix = acc;
    return true;
}

// rows_per_warp (k): each warp takes rows r0 + w + wpc t of its chunk (R =
// wpc k rows); with k = 1 the row's bitmap stays in shared memory from the
// count to the fill, otherwise it is rebuilt for the fill.
__global__ void spgemm_symbolic_lookback_kernel(int mb, int nb, const int *__restrict__ rpa,
                                                const int *__restrict__ cia, const int *__restrict__ rpb,
                                                const int *__restrict__ cib, int *__restrict__ rpc,
                                                int *__restrict__ cic, int64_t cap, unsigned long long *flags,
                                                unsigned epoch, int rows_per_warp, uint64_t limit_ns)
{
    extern __shared__ uint32_t bm_all[];
    __shared__ int s_cnt[1024]; // row counts of the chunk, then their exclusive offsets
    __shared__ int s_prefix, s_ok;
    const int words = (nb + 31) >> 5;
    const int wpc = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = rows_per_warp, R = wpc * k;
    uint32_t *bm = bm_all + (size_t)warp * words;
    const int nchunks = (mb + R - 1) / R;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x)
    {
        const int r0 = c * R;
        // ---- count: row r0 + w + wpc t of the chunk ----
        for (int t = 0; t < k; ++t)
        {
            const int lr = warp + wpc * t, row = r0 + lr;
            int cnt = 0;
            if (row < mb)
            {
                build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
                for (int w = lane; w < words; w += 32)
                    cnt += __popc(bm[w]);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            }
            if (lane == 0)
                s_cnt[lr] = cnt;
            __syncwarp();
        }
        __syncthreads();
        // ---- warp 0: the chunk's exclusive row offsets and total, publish,
        //      look back, publish the inclusive prefix ----
        if (warp == 0)
        {
            int carry = 0;
            for (int b = 0; b < R; b += 32)
            {
                const int v = b + lane < R ? s_cnt[b + lane] : 0;
                int x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o)
                        x += y;
                }
                if (b + lane < R)
                    s_cnt[b + lane] = carry + x - v;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            const int total = carry;
            if (lane == 0)
                atomicExch(&flags[c], lb_word(epoch, c == 0, total));
            int prefix = 0;
            bool ok = true;
            if (c > 0)
                ok = lb_prefix(flags, c, epoch, limit_ns, lane, &prefix);
            if (lane == 0)
            {
                if (ok && c > 0)
                    atomicExch(&flags[c], lb_word(epoch, true, prefix + total));
                if (!ok)
                    atomicExch(&g_spg_error, 3);
                s_prefix = prefix;
                s_ok = ok;
                if (r0 + R >= mb) // the last chunk: the total of all rows
                    rpc[mb] = prefix + total;
            }
        }
        __syncthreads();
        if (!s_ok)
            return;
        const int prefix = s_prefix;
        for (int lr = threadIdx.x; lr < R; lr += blockDim.x)
            if (r0 + lr < mb)
                rpc[r0 + lr] = prefix + s_cnt[lr];
        // ---- fill: ColIdxC ascending per row, up to the capacity ----
        if (cap > 0)
            for (int t = 0; t < k; ++t)
            {
                const int lr = warp + wpc * t, row = r0 + lr;
                if (row >= mb)
                    break;
                if (k > 1)
                    build_row_bitmap(bm, words, row, rpa, cia, rpb, cib, lane);
                int out = prefix + s_cnt[lr];
                for (int w0 = 0; w0 < words; w0 += 32)
                {
                    const int w = w0 + lane;
                    uint32_t bits = w < words ? bm[w] : 0u;
                    const int cb = __popc(bits);
                    int pre = cb;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1)
                    {
                        const int y = __shfl_up_sync(0xffffffffu, pre, o);
                        if (lane >= o)
                            pre += y;
                    }
                    int pos = out + pre - cb;
                    while (bits)
                    {
                        const int b = __ffs(bits) - 1;
                        if (pos < cap)
                            cic[pos] = w * 32 + b;
                        ++pos;
                        bits &= bits - 1;
                    }
                    out += __shfl_sync(0xffffffffu, pre, 31);
                }
                __syncwarp();
            }
        __syncthreads(); // s_cnt and the bitmaps are reused by the next chunk
    }
}

// ---------------------------------------------------------------------------
// numeric
// ---------------------------------------------------------------------------
struct SpNumArgs
{
    int mb, nb;
    const int *rpa, *cia, *rpb, *cib, *rpc, *cic;
    const uint16_t *va, *vb;
    void *vc;
    int64_t nnzc;
    int out_type;
    float alpha, beta;
    int num_iter;
};

// Store one C tile with alpha / beta (lane layout of store_tile_frag).
__device__ __forceinline__ void store_c_tile(const SpNumArgs &p, int64_t c, int gq, int tq, const float (&acc0)[4],
                                             const float (&acc1)[4])
{
    store_tile_frag(p.vc, c, p.out_type, p.alpha, p.beta, gq, tq, acc0, acc1);
}

template <bool BF16>
__global__ void __launch_bounds__(256) spgemm_numeric_kernel(const SpNumArgs p)
{
    const int lane = threadIdx.x & 31;
    const int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= p.nnzc || c >= p.rpc[p.mb]) // nnz_c may be an upper bound
        return;
    // block-row of this C tile: last i with rpc[i] <= c
    int lo = 0, hi = p.mb - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (p.rpc[mid] <= c)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int i = lo;
    const int j = p.cic[c];
    const int gq = lane >> 2, tq = lane & 3;

    float acc0[4] = {0.f, 0.f, 0.f, 0.f}; // C columns 0..7
    float acc1[4] = {0.f, 0.f, 0.f, 0.f}; // C columns 8..15
    const int a_begin = p.rpa[i], a_end = p.rpa[i + 1];
    for (int it = 0; it < p.num_iter; ++it)
    {
        for (int base = a_begin; base < a_end; base += 32)
        {
            // each lane searches one A block of the row for a matching B block
            const int e = base + lane;
            int match = -1;
            if (e < a_end)
            {
                const int k = p.cia[e];
                int l = p.rpb[k], h = p.rpb[k + 1] - 1;
                while (l <= h)
                {
                    const int m = (l + h) >> 1;
                    const int v = p.cib[m];
                    if (v == j)
                    {
                        match = m;
                        break;
                    }
                    if (v < j)
                        l = m + 1;
                    else
                        h = m - 1;
                }
            }
            uint32_t hits = __ballot_sync(0xffffffffu, match >= 0);
            while (hits)
            {
                const int src = __ffs(hits) - 1;
                hits &= hits - 1;
                const int eb = __shfl_sync(0xffffffffu, match, src);
                const int ea = base + src;
                const uint16_t *ta = p.va + (int64_t)ea * 256;
                const uint16_t *tb = p.vb + (int64_t)eb * 256;
                // A fragment with the k index permuted inside the k-step: lane
                // (g, t) holds A[g][4t..4t+3] and A[g+8][4t..4t+3]
                const uint2 ra = __ldg(reinterpret_cast<const uint2 *>(ta + gq * 16 + 4 * tq));
                const uint2 rb = __ldg(reinterpret_cast<const uint2 *>(ta + (gq + 8) * 16 + 4 * tq));
                // B fragment (K x N, row-major tile), same k permutation
                uint32_t b00, b01, b10, b11;
                {
                    const uint16_t *col0 = tb + gq;     // n = g      (columns 0..7)
                    const uint16_t *col1 = tb + gq + 8; // n = g + 8  (columns 8..15)
                    const int k0 = 4 * tq;
                    b00 = (uint32_t)__ldg(col0 + (k0 + 0) * 16) | ((uint32_t)__ldg(col0 + (k0 + 1) * 16) << 16);
                    b01 = (uint32_t)__ldg(col0 + (k0 + 2) * 16) | ((uint32_t)__ldg(col0 + (k0 + 3) * 16) << 16);
                    b10 = (uint32_t)__ldg(col1 + (k0 + 0) * 16) | ((uint32_t)__ldg(col1 + (k0 + 1) * 16) << 16);
                    b11 = (uint32_t)__ldg(col1 + (k0 + 2) * 16) | ((uint32_t)__ldg(col1 + (k0 + 3) * 16) << 16);
                }
                mma16816<BF16>(acc0, ra.x, rb.x, ra.y, rb.y, b00, b01);
                mma16816<BF16>(acc1, ra.x, rb.x, ra.y, rb.y, b10, b11);
            }
        }
    }

    store_c_tile(p, c, gq, tq, acc0, acc1);
}

// ---------------------------------------------------------------------------
// numeric, one CTA per block-row of C (16-byte aligned tiles)
//
// The C tiles of block-row i all multiply the same A tiles A(i, k) and search
// the same B block-rows k for their column j.  So the CTA stages, once, the
// A tiles of row i (ldmatrix layout) and the column indices of every B row k
// it touches in shared memory; each of its 8 warps then takes C tiles
// (i, j) in turn: lanes binary-search j in the staged lists (shared-memory
// latency instead of dependent global loads), and every match costs one
// coalesced 512-byte load of the B tile into the warp's slot, one ldmatrix
// (transposed) for its fragments, and two MMAs.  Products are accumulated in
// ascending k, as the reference's sparse accumulator does.  Rows whose A
// tiles or B lists exceed the staging capacity read them from global memory.
// ---------------------------------------------------------------------------
constexpr int kRowWarps = 8;
constexpr int kMaxATiles = 32;   // 16 KB of A tiles (about 28 KB per CTA: 8 CTAs per SM)
constexpr int kMaxBList = 2048;  // 8 KB of B column indices

// The row's C tiles pulled one at a time (the per-tile search form); the
// CTA's shared buffers are passed in: sA kMaxATiles * 512 bytes, sB
// kRowWarps * 512, sList kMaxBList ints, sOff kMaxATiles + 1, sK kMaxATiles.
template <bool BF16, int WARPS, int MAXA = kMaxATiles>
__device__ __forceinline__ void numeric_row_pull(const SpNumArgs &p, const int i, uint8_t *sA, uint8_t *sB,
                                                 int *sList, int *sOff, int *sK)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = p.rpc[i];
    const int c1 = (int)min((int64_t)p.rpc[i + 1], p.nnzc); // tiles past the caller's bound are untouched
    if (c1 <= c0)
        return;
    const int a0 = p.rpa[i], na = p.rpa[i + 1] - a0;
    const bool a_staged = na <= MAXA;

    // ---- staging (whole CTA): A tiles, B row lengths, their prefix, lists ----
    bool l_staged = false;
    if (a_staged)
    {
        for (int e = warp; e < na; e += WARPS)
            stage_tile(sA + e * 512, p.va + (int64_t)(a0 + e) * 256, lane);
        if (warp == 0)
        {
            // lengths of the B rows, exclusive prefix over the (<= 48) entries
            int total = 0;
            for (int base = 0; base < na; base += 32)
            {
                const int e = base + lane;
                int len = 0;
                if (e < na)
                {
                    const int k = p.cia[a0 + e];
                    sK[e] = k;
                    len = p.rpb[k + 1] - p.rpb[k];
                }
                int pre = len;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(0xffffffffu, pre, o);
                    if (lane >= o)
                        pre += y;
                }
                if (e < na)
                    sOff[e] = total + pre - len;
                total += __shfl_sync(0xffffffffu, pre, 31);
            }
            if (lane == 0)
                sOff[na] = total;
        }
        __syncthreads();
        l_staged = sOff[na] <= kMaxBList;
        if (l_staged)
            for (int e = warp; e < na; e += WARPS)
            {
                const int b0 = p.rpb[sK[e]], len = sOff[e + 1] - sOff[e];
                for (int q = lane; q < len; q += 32)
                    sList[sOff[e] + q] = p.cib[b0 + q];
            }
        __syncthreads();
    }

    const int gq = lane >> 2, tq = lane & 3;
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA);
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(sB + warp * 512);
    uint8_t *slot_p = sB + warp * 512;
    for (int c = c0 + warp; c < c1; c += WARPS)
    {
        const int j = p.cic[c];
        float acc0[4] = {0.f, 0.f, 0.f, 0.f}; // C columns 0..7
        float acc1[4] = {0.f, 0.f, 0.f, 0.f}; // C columns 8..15
        for (int it = 0; it < p.num_iter; ++it)
            for (int base = 0; base < na; base += 32)
            {
                // lane e: position of column j in B row k_e (global B entry), or -1
                const int e = base + lane;
                int match = -1;
                if (e < na)
                {
                    const int k = a_staged ? sK[e] : p.cia[a0 + e];
                    const int bstart = p.rpb[k];
                    if (l_staged)
                    {
                        int l = sOff[e], h = sOff[e + 1] - 1;
                        const int o = l;
                        while (l <= h)
                        {
                            const int m = (l + h) >> 1, v = sList[m];
                            if (v == j)
                            {
                                match = bstart + (m - o);
                                break;
                            }
                            if (v < j)
                                l = m + 1;
                            else
                                h = m - 1;
                        }
                    }
                    else
                    {
                        int l = bstart, h = p.rpb[k + 1] - 1;
                        while (l <= h)
                        {
                            const int m = (l + h) >> 1, v = p.cib[m];
                            if (v == j)
                            {
                                match = m;
                                break;
                            }
                            if (v < j)
                                l = m + 1;
                            else
                                h = m - 1;
                        }
                    }
                }
                uint32_t hits = __ballot_sync(0xffffffffu, match >= 0);
                while (hits)
                {
                    const int src = __ffs(hits) - 1;
                    hits &= hits - 1;
                    const int eb = __shfl_sync(0xffffffffu, match, src);
                    const int ea = base + src;
                    uint32_t a[4];
                    if (a_staged)
                        ldsm4(tile_ldsm_addr(sA_u + ea * 512, lane), a);
                    else
                    {
                        const uint32_t *ta = reinterpret_cast<const uint32_t *>(p.va + (int64_t)(a0 + ea) * 256);
                        a[0] = __ldg(ta + (gq * 16 + 2 * tq) / 2);
                        a[1] = __ldg(ta + ((gq + 8) * 16 + 2 * tq) / 2);
                        a[2] = __ldg(ta + (gq * 16 + 2 * tq + 8) / 2);
                        a[3] = __ldg(ta + ((gq + 8) * 16 + 2 * tq + 8) / 2);
                    }
                    __syncwarp(); // the slot's previous tile has been read
                    stage_tile(slot_p, p.vb + (int64_t)eb * 256, lane);
                    __syncwarp();
                    uint32_t b[4];
                    ldsm4_t(tile_ldsm_addr(slot, lane), b); // (k lo, n 0-7), (k hi, n 0-7), (k lo, n 8-15), (k hi, n 8-15)
                    mma16816<BF16>(acc0, a[0], a[1], a[2], a[3], b[0], b[1]);
                    mma16816<BF16>(acc1, a[0], a[1], a[2], a[3], b[2], b[3]);
                }
            }
        store_c_tile(p, c, gq, tq, acc0, acc1);
    }
}

template <bool BF16>
__global__ void __launch_bounds__(kRowWarps * 32) spgemm_numeric_row_kernel(const SpNumArgs p)
{
    __shared__ __align__(16) uint8_t sA[kMaxATiles * 512];
    __shared__ __align__(16) uint8_t sB[kRowWarps * 512]; // one B tile slot per warp
    __shared__ int sList[kMaxBList];
    __shared__ int sOff[kMaxATiles + 1];
    __shared__ int sK[kMaxATiles];
    numeric_row_pull<BF16, kRowWarps>(p, blockIdx.x, sA, sB, sList, sOff, sK);
}

// ---------------------------------------------------------------------------
// numeric, one CTA per block-row of C, products pushed to their tiles
//
// The per-tile search above costs one binary search per (C tile, A entry)
// pair -- about ten per tile at 1 % density -- in dependent shared-memory
// loads, and each tile's B tile load is exposed.  Here the row's products
// are enumerated once: all threads walk the flattened (A entry, B entry)
// space, find each product's C position by one binary search in the row's
// ColIdxC (staged in shared memory), and a counting sort by position
// groups them per C tile (each tile's short list then re-sorted by
// enumeration index, so products still accumulate in ascending k).  The
// warps then take the tiles in turn; each streams its products' B tiles
// with 16-byte cp.async into a two-slot ring (the next product's tile in
// flight while the current one is multiplied), A tiles read from the staged
// row.  Rows beyond the staging capacities fall back to the per-tile form.
// ---------------------------------------------------------------------------
constexpr int kPushWarps = 4;     // 4-warp CTAs, ~31 KB each: seven per SM, every row of a 1024-row matrix in one wave
constexpr int kPushMaxC = 512;    // C tiles of a row
constexpr int kPushMaxProd = 512; // products of a row
constexpr int kPushMaxA = 24;     // A tiles of a row staged (12 KB)
constexpr int kPushDepth = 4;     // B tiles in flight per warp

template <bool BF16>
__global__ void __launch_bounds__(kPushWarps * 32) spgemm_numeric_push_kernel(const SpNumArgs p)
{
    constexpr int kRowWarps = kPushWarps;
    __shared__ __align__(16) uint8_t sA[kPushMaxA * 512];
    __shared__ __align__(16) uint8_t sB[kRowWarps * kPushDepth * 512]; // B slots per warp
    // one pool of indices (the per-tile fallback uses its first kMaxBList
    // entries as its list buffer): the row's ColIdxC, then per tile the
    // product count / range end; per product (A entry << 16) | C position
    // (-1 when absent), its B entry, and the products grouped by C tile
    __shared__ int sPool[5 * kPushMaxC];
    static_assert(5 * kPushMaxC >= kMaxBList && kPushMaxProd == kPushMaxC, "fallback list buffer");
    int *sCol = sPool, *sCnt = sPool + kPushMaxC, *sPep = sPool + 2 * kPushMaxC, *sPb = sPool + 3 * kPushMaxC,
        *sOrd = sPool + 4 * kPushMaxC;
    __shared__ int sOff[kPushMaxA + 1];
    __shared__ int sK[kPushMaxA];
    __shared__ int sRb[kPushMaxA];
    const int i = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int kT = kRowWarps * 32;
    const int c0 = p.rpc[i];
    const int c1 = (int)min((int64_t)p.rpc[i + 1], p.nnzc); // tiles past the caller's bound are untouched
    if (c1 <= c0)
        return;
    const int nt = c1 - c0;
    const int a0 = p.rpa[i], na = p.rpa[i + 1] - a0;
    if (nt > kPushMaxC || na > kPushMaxA)
    {
        numeric_row_pull<BF16, kPushWarps, kPushMaxA>(p, i, sA, sB, sPool, sOff, sK);
        return;
    }
    // ---- stage: ColIdxC, B row ranges and their prefix, A tiles ----
    for (int t = tid; t < nt; t += kT)
    {
        sCol[t] = p.cic[c0 + t];
        sCnt[t] = 0;
    }
    if (warp == 0)
    {
        int len = 0;
        if (lane < na)
        {
            const int k = p.cia[a0 + lane];
            const int rb = p.rpb[k];
            len = p.rpb[k + 1] - rb;
            sK[lane] = k;
            sRb[lane] = rb;
        }
        int pre = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o)
                pre += y;
        }
        if (lane < na)
            sOff[lane] = pre - len;
        if (lane == 31)
            sOff[na] = pre;
    }
    for (int e = warp; e < na; e += kRowWarps)
        stage_tile(sA + e * 512, p.va + (int64_t)(a0 + e) * 256, lane);
    __syncthreads();
    const int np = sOff[na];
    if (np > kPushMaxProd)
    {
        __syncthreads();
        numeric_row_pull<BF16, kPushWarps, kPushMaxA>(p, i, sA, sB, sPool, sOff, sK);
        return;
    }
    // ---- enumerate the products and count them per C tile ----
    for (int f = tid; f < np; f += kT)
    {
        int lo = 0, hi = na - 1; // entry e with sOff[e] <= f < sOff[e + 1]
        while (lo < hi)
        {
            const int m = (lo + hi + 1) >> 1;
            if (sOff[m] <= f)
                lo = m;
            else
                hi = m - 1;
        }
        const int e = lo;
        const int eb = sRb[e] + (f - sOff[e]);
        const int j = p.cib[eb];
        int l = 0, h = nt;
        while (l < h)
        {
            const int m = (l + h) >> 1;
            if (sCol[m] < j)
                l = m + 1;
            else
                h = m;
        }
        const bool hit = l < nt && sCol[l] == j;
        sPep[f] = hit ? ((e << 16) | l) : -1;
        sPb[f] = eb;
        if (hit)
            atomicAdd(&sCnt[l], 1);
    }
    __syncthreads();
    // ---- exclusive scan of the counts (warp 0, 32 consecutive entries per lane) ----
    if (warp == 0)
    {
        const int per = (nt + 31) >> 5;
        const int b0 = lane * per, b1 = min(nt, b0 + per);
        int run = 0;
        for (int t = b0; t < b1; ++t)
            run += sCnt[t];
        int pre = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o)
                pre += y;
        }
        int acc = pre - run;
        for (int t = b0; t < b1; ++t)
        {
            const int c = sCnt[t];
            sCnt[t] = acc;
            acc += c;
        }
    }
    __syncthreads();
    // ---- scatter: afterwards sCnt[t] is the end of tile t's range ----
    for (int f = tid; f < np; f += kT)
    {
        const int v = sPep[f];
        if (v >= 0)
            sOrd[atomicAdd(&sCnt[v & 0xffff], 1)] = f;
    }
    __syncthreads();
    // ---- each tile's products in enumeration order (ascending k) ----
    for (int t = tid; t < nt; t += kT)
    {
        const int b = t ? sCnt[t - 1] : 0, e = sCnt[t];
        for (int x = b + 1; x < e; ++x)
        {
            const int v = sOrd[x];
            int y = x - 1;
            while (y >= b && sOrd[y] > v)
            {
                sOrd[y + 1] = sOrd[y];
                --y;
            }
            sOrd[y + 1] = v;
        }
    }
    __syncthreads();

    // ---- multiply: warp w takes the contiguous tile range [t0, t1), whose
    //      products are contiguous in sOrd (ascending tile, then k); their
    //      indices are read 32 at a time, one per lane, and broadcast, so a
    //      product costs no dependent shared-memory lookups; kPushDepth B
    //      tiles in flight ----
    const int gq = lane >> 2, tq = lane & 3;
    const uint32_t sA_u = (uint32_t)__cvta_generic_to_shared(sA);
    const uint32_t slots = (uint32_t)__cvta_generic_to_shared(sB + warp * kPushDepth * 512);
    const int swz = tile_swz(lane >> 1, lane & 1);
    const int t0 = (nt * warp) / kRowWarps, t1 = (nt * (warp + 1)) / kRowWarps;
    if (t0 < t1)
    {
        const int q0 = t0 ? sCnt[t0 - 1] : 0, q1 = sCnt[t1 - 1]; // this warp's products
        // product q's (A entry << 16 | tile) and B entry, for q = base + lane
        auto load_info = [&](int base, int &pep, int &pb) {
            const int q = base + lane;
            pep = 0;
            pb = 0;
            if (q < q1)
            {
                const int f = sOrd[q];
                pep = sPep[f];
                pb = sPb[f];
            }
        };
        int ib = q0, i_pep, i_pb; // issue side: info chunk at ib
        load_info(ib, i_pep, i_pb);
        int qi = q0, issued = 0;
        auto issue = [&]() {
            if (qi < q1)
            {
                if (qi - ib >= 32)
                {
                    ib += 32;
                    load_info(ib, i_pep, i_pb);
                }
                const int eb = __shfl_sync(0xffffffffu, i_pb, qi - ib);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(slots + (issued % kPushDepth) * 512 +
                                                                                swz),
                             "l"(p.vb + (int64_t)eb * 256 + lane * 8)
                             : "memory");
                ++qi;
                ++issued;
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
#pragma unroll
        for (int d = 0; d < kPushDepth - 1; ++d)
            issue();
        int cb = q0, c_pep, c_pb; // consumer side: info chunk at cb
        load_info(cb, c_pep, c_pb);
        float acc0[4] = {0.f, 0.f, 0.f, 0.f};
        float acc1[4] = {0.f, 0.f, 0.f, 0.f};
        int tile = t0;
        for (int qc = q0; qc < q1; ++qc)
        {
            issue(); // kPushDepth - 1 products ahead, into the slot read last
            if (qc - cb >= 32)
            {
                cb += 32;
                load_info(cb, c_pep, c_pb);
            }
            const int pep = __shfl_sync(0xffffffffu, c_pep, qc - cb);
            const int pt = pep & 0xffff, e = pep >> 16;
            while (tile < pt) // the previous tile is complete (tiles without products store zeros)
            {
                store_c_tile(p, (int64_t)c0 + tile, gq, tq, acc0, acc1);
#pragma unroll
                for (int x = 0; x < 4; ++x)
                    acc0[x] = acc1[x] = 0.f;
                ++tile;
            }
            asm volatile("cp.async.wait_group %0;" ::"n"(kPushDepth - 1) : "memory");
            __syncwarp();
            uint32_t a[4], b[4];
            ldsm4(tile_ldsm_addr(sA_u + e * 512, lane), a);
            ldsm4_t(tile_ldsm_addr(slots + ((qc - q0) % kPushDepth) * 512, lane), b);
            for (int r = 0; r < p.num_iter; ++r)
            {
                mma16816<BF16>(acc0, a[0], a[1], a[2], a[3], b[0], b[1]);
                mma16816<BF16>(acc1, a[0], a[1], a[2], a[3], b[2], b[3]);
            }
            __syncwarp(); // every lane's fragments are read before the slot is refilled
        }
        for (; tile < t1; ++tile)
        {
            store_c_tile(p, (int64_t)c0 + tile, gq, tq, acc0, acc1);
#pragma unroll
            for (int x = 0; x < 4; ++x)
                acc0[x] = acc1[x] = 0.f;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

int bitmap_launch(int nb, int *warps_per_cta, size_t *smem)
{
    const int words = (nb + 31) >> 5;
    int w = 8;
    while (w > 1 && (size_t)w * words * 4 > 96 * 1024)
        w >>= 1;
    if ((size_t)w * words * 4 > 200 * 1024)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm: %d block columns exceed the shared-memory bitmap", nb);
    *warps_per_cta = w;
    *smem = (size_t)w * words * 4;
    return KAMI_OK;
}

int prep_bitmap_fn(const void *fn, size_t smem)
{
    if (smem > 48 * 1024)
    {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(spgemm bitmap kernel)");
    }
    return KAMI_OK;
}

// Row pointers must be present; column-index arrays may be NULL when the
// matrix has no nonzero block.
int check_bsr_args(int bsr, int mb, int kb, int nb, const void *a, const void *, const void *c, const void *)
{
    if (bsr != kBsr)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm: only 16 x 16 BSR tiles are supported (got %d)", bsr);
    if (mb < 0 || kb < 0 || nb < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm: negative block dimensions");
    if (mb > 0 && (!a || !c))
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm: null row pointer");
    return KAMI_OK;
}

// The fused one-launch symbolic pass; KAMI_ERR_UNSUPPORTED (nothing
// launched) when the device has no cooperative launch.
int symbolic_fused(int mb, int nb, const int *rpa, const int *cia, const int *rpb, const int *cib, int *rpc, int *cic,
                   int64_t cap, cudaStream_t s)
{
    int dev = 0, sms = 0, coop = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return KAMI_ERR_UNSUPPORTED;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop)
        return KAMI_ERR_UNSUPPORTED;
    static std::once_flag once[64];
    static unsigned int *bar_base[64];
    static cudaError_t bar_err[64];
    std::call_once(once[dev], [&] {
        void *ptr = nullptr;
        bar_err[dev] = cudaGetSymbolAddress(&ptr, g_spg_bar);
        bar_base[dev] = reinterpret_cast<unsigned int *>(ptr);
    });
    if (bar_err[dev] != cudaSuccess)
        return cuda_fail(bar_err[dev], "cudaGetSymbolAddress(spgemm barrier)");
    int wpc;
    size_t smem;
    int st = bitmap_launch(nb, &wpc, &smem);
    if (st)
        return st;
    const void *fn = (const void *)spgemm_symbolic_fused_kernel;
    if ((st = prep_bitmap_fn(fn, smem)))
        return st;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, wpc * 32, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(spgemm fused)");
    if (occ < 1)
        return KAMI_ERR_UNSUPPORTED;
    const int rows_ctas = (mb + wpc - 1) / wpc;
    int grid = rows_ctas < sms * occ ? rows_ctas : sms * occ;
    // keep every row's bitmap from the count to the fill when the warps' rows
    // fit in 96 KB of shared memory at a grid that stays co-resident
    int keep_rows = 0;
    const int words = (nb + 31) >> 5;
    const int rpw = (mb + grid * wpc - 1) / (grid * wpc);
    const size_t keep_smem = (size_t)wpc * rpw * words * 4;
    if (cap > 0 && rpw > 0 && keep_smem <= 96 * 1024)
    {
        int occ_k = 0;
        if (keep_smem > smem && (st = prep_bitmap_fn(fn, keep_smem)))
            return st;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_k, fn, wpc * 32, keep_smem) == cudaSuccess &&
            grid <= sms * occ_k)
        {
            keep_rows = rpw;
            smem = keep_smem > smem ? keep_smem : smem;
        }
    }
    static std::atomic<unsigned int> next_slot{0};
    unsigned int *bar = bar_base[dev] + 2 * (next_slot.fetch_add(1) % kFuseSlots);
    if ((e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), s)) != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync(spgemm barrier)");
    // generous: a barrier waits for the slowest CTA's share of the rows
    uint64_t limit = (uint64_t)2e9 + (uint64_t)mb * 20000ull;
    void *args[] = {&mb, &nb, &rpa, &cia, &rpb, &cib, &rpc, &cic, &cap, &bar, &limit, &keep_rows};
    if ((e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(wpc * 32), args, smem, s)) != cudaSuccess)
        return cuda_fail(e, "cudaLaunchCooperativeKernel(spgemm_symbolic_fused_kernel)");
    return KAMI_OK;
}


// The single-pass symbolic launch; KAMI_ERR_UNSUPPORTED (nothing launched)
// when the device has no cooperative launch or the rows need more chunks
// than the flag array holds.
int symbolic_lookback(int mb, int nb, const int *rpa, const int *cia, const int *rpb, const int *cib, int *rpc,
                      int *cic, int64_t cap, cudaStream_t s)
{
    int dev = 0, sms = 0, coop = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return KAMI_ERR_UNSUPPORTED;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop || mb < 1)
        return KAMI_ERR_UNSUPPORTED;
    static std::once_flag once[64];
    static unsigned long long *flag_base[64];
    static cudaError_t flag_err[64];
    std::call_once(once[dev], [&] {
        void *ptr = nullptr;
        flag_err[dev] = cudaGetSymbolAddress(&ptr, g_spg_flags);
        flag_base[dev] = reinterpret_cast<unsigned long long *>(ptr);
    });
    if (flag_err[dev] != cudaSuccess)
        return cuda_fail(flag_err[dev], "cudaGetSymbolAddress(spgemm look-back flags)");
    int wpc;
    size_t smem;
    int st = bitmap_launch(nb, &wpc, &smem);
    if (st)
        return st;
    // rows per warp per chunk: the chunks must fit the flag array and R = wpc k
    // rows the kernel's offset array
    const int64_t k64 = ((int64_t)mb + (int64_t)wpc * kLbMaxChunks - 1) / ((int64_t)wpc * kLbMaxChunks);
    if (k64 < 1 || wpc * k64 > 1024)
        return KAMI_ERR_UNSUPPORTED;
    const int k = (int)k64, R = wpc * k;
    const int nchunks = (mb + R - 1) / R;
    const void *fn = (const void *)spgemm_symbolic_lookback_kernel;
    if ((st = prep_bitmap_fn(fn, smem)))
        return st;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, wpc * 32, smem)) != cudaSuccess)
        return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor(spgemm look-back)");
    if (occ < 1)
        return KAMI_ERR_UNSUPPORTED;
    const int grid = nchunks < sms * occ ? nchunks : sms * occ;
    static std::atomic<unsigned int> next_launch{0};
    const unsigned int n = next_launch.fetch_add(1);
    unsigned long long *flags = flag_base[dev] + (size_t)(n % kLbSlots) * kLbMaxChunks;
    unsigned epoch = (n % 0x7fffffffu) + 1; // never 0, the value of untouched flags
    uint64_t limit = (uint64_t)2e9 + (uint64_t)mb * 20000ull;
    void *args[] = {&mb, &nb, &rpa, &cia, &rpb, &cib, &rpc, &cic, &cap, &flags, &epoch, (void *)&k, &limit};
    if ((e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(wpc * 32), args, smem, s)) != cudaSuccess)
        return cuda_fail(e, "cudaLaunchCooperativeKernel(spgemm_symbolic_lookback_kernel)");
    return KAMI_OK;
}

} // namespace

int spgemm_tc05_launch(bool bf16, int mb, int64_t nnzc, const int *rpa, const int *cia, const int *rpb, const int *cib,
                       const int *rpc, const int *cic, const void *va, const void *vb, void *vc, int out_type,
                       double alpha, double beta, int num_iter, cudaStream_t s);

// AUTO's choice of the numeric kernel: the mma.sync row kernel (false) or
// the tcgen05 kernel (true).
bool spgemm_auto_tc05() { return false; }

int spgemm_read_error(int *flag)
{
    int v = 0, z = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_spg_error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_spg_error, &z, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "reading the spgemm status");
    *flag = v;
    return KAMI_OK;
}

} // namespace kami

using namespace kami;

extern "C" {

int kami_spgemm_bsr_symbolic(int bsr, int mb, int kb, int nb, const int *row_ptr_a, const int *col_idx_a,
                             const int *row_ptr_b, const int *col_idx_b, int *row_ptr_c, int *nnz_c_host,
                             void *stream)
{
    int st = check_bsr_args(bsr, mb, kb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b);
    if (st)
        return st;
    if (!row_ptr_c)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm: row_ptr_c is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (mb > 0 && nb > 0)
    {
        int wpc;
        size_t smem;
        if ((st = bitmap_launch(nb, &wpc, &smem)))
            return st;
        if ((st = prep_bitmap_fn((const void *)spgemm_count_kernel, smem)))
            return st;
        const int grid = (mb + wpc - 1) / wpc;
        spgemm_count_kernel<<<grid, wpc * 32, smem, s>>>(mb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b,
                                                        row_ptr_c);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return cuda_fail(e, "spgemm_count_kernel");
        spgemm_scan_kernel<<<1, 1024, 0, s>>>(mb, row_ptr_c);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return cuda_fail(e, "spgemm_scan_kernel");
    }
    else
    {
        if ((e = cudaMemsetAsync(row_ptr_c, 0, sizeof(int) * (size_t)(mb + 1), s)) != cudaSuccess)
            return cuda_fail(e, "cudaMemsetAsync(row_ptr_c)");
    }
    if (nnz_c_host)
    {
        if ((e = cudaMemcpyAsync(nnz_c_host, row_ptr_c + mb, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(nnzC)");
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamSynchronize");
    }
    return KAMI_OK;
}

int kami_spgemm_bsr_fill_colidx(int bsr, int mb, int kb, int nb, const int *row_ptr_a, const int *col_idx_a,
                                const int *row_ptr_b, const int *col_idx_b, const int *row_ptr_c, int *col_idx_c,
                                void *stream)
{
    int st = check_bsr_args(bsr, mb, kb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b);
    if (st)
        return st;
    if (mb == 0 || nb == 0)
        return KAMI_OK;
    if (!row_ptr_c || !col_idx_c)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm: row_ptr_c / col_idx_c is NULL");
    int wpc;
    size_t smem;
    if ((st = bitmap_launch(nb, &wpc, &smem)))
        return st;
    if ((st = prep_bitmap_fn((const void *)spgemm_colfill_kernel, smem)))
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    spgemm_colfill_kernel<<<(mb + wpc - 1) / wpc, wpc * 32, smem, s>>>(mb, nb, row_ptr_a, col_idx_a, row_ptr_b,
                                                                      col_idx_b, row_ptr_c, col_idx_c, INT64_MAX);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(e, "spgemm_colfill_kernel");
    return KAMI_OK;
}

int kami_spgemm_bsr_symbolic_device(int bsr, int mb, int kb, int nb, const int *row_ptr_a, const int *col_idx_a,
                                    const int *row_ptr_b, const int *col_idx_b, int *row_ptr_c, int *col_idx_c,
                                    int64_t capacity, void *stream)
{
    if (capacity < 0 || (capacity > 0 && !col_idx_c))
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm symbolic: capacity must be >= 0 with a column array");
    if (mb > 0 && nb > 0)
    {
        const int st0 = check_bsr_args(bsr, mb, kb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b);
        if (st0)
            return st0;
        if (!row_ptr_c)
            return fail(KAMI_ERR_INVALID_VALUE, "spgemm: row_ptr_c is NULL");
        // one pass with a decoupled look-back; past the flag array's capacity
        // the three-phase form with grid barriers
        const int stl = symbolic_lookback(mb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b, row_ptr_c, col_idx_c,
                                          capacity, reinterpret_cast<cudaStream_t>(stream));
        if (stl != KAMI_ERR_UNSUPPORTED)
            return stl;
        const int st1 = symbolic_fused(mb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b, row_ptr_c, col_idx_c,
                                       capacity, reinterpret_cast<cudaStream_t>(stream));
        if (st1 != KAMI_ERR_UNSUPPORTED)
            return st1;
    }
    // count + scan, with no copy of nnzC to the host
    int st = kami_spgemm_bsr_symbolic(bsr, mb, kb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b, row_ptr_c,
                                      nullptr, stream);
    if (st || mb == 0 || nb == 0 || capacity == 0)
        return st;
    int wpc;
    size_t smem;
    if ((st = bitmap_launch(nb, &wpc, &smem)))
        return st;
    if ((st = prep_bitmap_fn((const void *)spgemm_colfill_kernel, smem)))
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    spgemm_colfill_kernel<<<(mb + wpc - 1) / wpc, wpc * 32, smem, s>>>(mb, nb, row_ptr_a, col_idx_a, row_ptr_b,
                                                                      col_idx_b, row_ptr_c, col_idx_c, capacity);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(e, "spgemm_colfill_kernel");
    return KAMI_OK;
}

int kami_spgemm_bsr_numeric(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int nb,
                            const int *row_ptr_a, const int *col_idx_a, const void *val_a, const int *row_ptr_b,
                            const int *col_idx_b, const void *val_b, const int *row_ptr_c, const int *col_idx_c,
                            void *val_c, int64_t nnz_c, double alpha, double beta, int num_iter, void *stream)
{
    return kami_spgemm_bsr_numeric_variant(KAMI_VARIANT_AUTO, in_type, out_type, bsr, mb, kb, nb, row_ptr_a,
                                           col_idx_a, val_a, row_ptr_b, col_idx_b, val_b, row_ptr_c, col_idx_c,
                                           val_c, nnz_c, alpha, beta, num_iter, stream);
}

int kami_spgemm_bsr_numeric_variant(kami_variant_t variant, kami_dtype_t in_type, kami_dtype_t out_type, int bsr,
                                    int mb, int kb, int nb, const int *row_ptr_a, const int *col_idx_a,
                                    const void *val_a, const int *row_ptr_b, const int *col_idx_b, const void *val_b,
                                    const int *row_ptr_c, const int *col_idx_c, void *val_c, int64_t nnz_c,
                                    double alpha, double beta, int num_iter, void *stream)
{
    if (variant != KAMI_VARIANT_AUTO && variant != KAMI_VARIANT_MMA_SYNC && variant != KAMI_VARIANT_TCGEN05)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm numeric: variant must be AUTO, MMA_SYNC or TCGEN05");
    int st = check_bsr_args(bsr, mb, kb, nb, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b);
    if (st)
        return st;
    if (in_type != KAMI_F16 && in_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm numeric: FP16/BF16 tiles only");
    if (out_type != KAMI_F32 && out_type != KAMI_F16 && out_type != KAMI_BF16)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm numeric: FP32/FP16/BF16 output only");
    if (num_iter < 1 || nnz_c < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm numeric: num_iter >= 1 and nnz_c >= 0 required");
    if (nnz_c == 0 || mb == 0)
        return KAMI_OK;
    // val_a / val_b may be NULL for an operand without entries (nothing is read)
    if (!row_ptr_c || !col_idx_c || !val_c)
        return fail(KAMI_ERR_INVALID_VALUE, "spgemm numeric: null pointer");
    if ((reinterpret_cast<uintptr_t>(val_a) & 7) || (reinterpret_cast<uintptr_t>(val_b) & 1) ||
        (reinterpret_cast<uintptr_t>(val_c) & 7))
        return fail(KAMI_ERR_MISALIGNED, "spgemm numeric: tile arrays must be 8-byte aligned");
    SpNumArgs p{};
    p.mb = mb;
    p.nb = nb;
    p.rpa = row_ptr_a;
    p.cia = col_idx_a;
    p.rpb = row_ptr_b;
    p.cib = col_idx_b;
    p.rpc = row_ptr_c;
    p.cic = col_idx_c;
    p.va = reinterpret_cast<const uint16_t *>(val_a);
    p.vb = reinterpret_cast<const uint16_t *>(val_b);
    p.vc = val_c;
    p.nnzc = nnz_c;
    p.out_type = out_type;
    p.alpha = (float)alpha;
    p.beta = (float)beta;
    p.num_iter = num_iter;
    const int64_t grid = (nnz_c + 7) / 8;
    if (grid > 0x7fffffff)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm numeric: too many C tiles");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const bool aligned16 = !(reinterpret_cast<uintptr_t>(val_a) & 15) && !(reinterpret_cast<uintptr_t>(val_b) & 15);
    const bool tc_ok = aligned16 && !(reinterpret_cast<uintptr_t>(val_c) & 15);
    if (variant == KAMI_VARIANT_TCGEN05 && !tc_ok)
        return fail(KAMI_ERR_MISALIGNED, "spgemm numeric (tcgen05): tile arrays must be 16-byte aligned");
    if (variant == KAMI_VARIANT_TCGEN05 || (variant == KAMI_VARIANT_AUTO && tc_ok && spgemm_auto_tc05()))
        return spgemm_tc05_launch(in_type == KAMI_BF16, mb, nnz_c, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b, row_ptr_c,
                                  col_idx_c, val_a, val_b, val_c, out_type, alpha, beta, num_iter, s);
    const bool rowwise = aligned16;
    if (rowwise) // one CTA per block-row, staged operands, products pushed to their tiles
    {
        if (in_type == KAMI_BF16)
            spgemm_numeric_push_kernel<true><<<(unsigned)mb, kPushWarps * 32, 0, s>>>(p);
        else
            spgemm_numeric_push_kernel<false><<<(unsigned)mb, kPushWarps * 32, 0, s>>>(p);
    }
    else if (in_type == KAMI_BF16)
        spgemm_numeric_kernel<true><<<(unsigned)grid, 256, 0, s>>>(p);
    else
        spgemm_numeric_kernel<false><<<(unsigned)grid, 256, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_fail(e, "spgemm_numeric_kernel");
    return KAMI_OK;
}

} // extern "C"
