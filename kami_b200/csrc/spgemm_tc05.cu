// spgemm_tc05.cu -- numeric block SpGEMM (BSR, 16 x 16 tiles) on the
// 5th-generation tensor cores, accumulators in tensor memory.
//
// Reference: the numeric kernels block_spgemm_{1d,2d,3d}_half_mma
// (src/sparse/spgemm/2d/block_spgemm_2d_half_mma.cu:171-555), which multiply
// one <= 192^2 block per CTA with mma.sync; and the host SPA
// (:557-646), whose per-row dense accumulator this kernel keeps on chip.
//
// One CTA per SM walks block-rows i = blockIdx.x, + gridDim.x, ...  The C
// tiles of row i (ColIdxC order, contiguous in ValC) are processed in units
// of up to 64 tiles; a unit's accumulators live in one of two 256-column
// halves of tensor memory, tile s of the unit in TMEM lanes 32 (s % 4) ..
// + 15 (the 16 rows of the tile), columns 16 (s / 4) .. + 15.  Each product
// A(i, k) B(k, j) is ONE tcgen05.mma of M = 64, N = 16, K = 16: the A
// operand's descriptor starts 16 (s % 4) rows before the A tile, so the
// tile's rows land in the quadrant of tile s, and the instruction's
// disable-output-lane mask leaves every other lane -- the other tiles that
// share these columns -- untouched.  Products are issued in ascending k for
// every C tile (the order of the reference's sparse accumulator), and a
// tile accumulates them in place; tiles with no product read the zeroed
// accumulator.
//
// Roles (192 threads):
//   warp 0   planner / loader: per unit, enumerates the row's products
//            (the A entries' B rows, flattened; each product's C position
//            found by binary search in the row's ColIdxC staged in shared
//            memory) and copies each product's A and B tiles with 16-byte
//            cp.async into a ring slot, in the 32-byte-swizzled layout the
//            MMA reads; each lane's arrival on the slot's barrier is
//            attached to its copies; an end-of-unit record closes a unit;
//   warp 1   lane 0 issues the MMAs (the product repeated num_iter times)
//            and frees each slot with tcgen05.commit; owns the TMEM;
//   warps 2-5  epilogue, warp w reading TMEM lanes 32 (w % 4) ..: each
//            tile's row r in lane r, 16 FP32 values, stored with alpha /
//            beta and the output type; then the accumulator is zeroed with
//            tcgen05.st for the next unit on this half.
// Every wait is bounded; a timeout sets g_sptc_error and ends the role.
#include <cstdint>

#include "kami_common.cuh"
#include "spgemm_tiles.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device status of the bounded waits (read and cleared by kami_device_status)
__device__ int g_sptc_error = 0;

namespace {

using namespace sptile;

constexpr int kWarps = 6;
constexpr int kThreads = kWarps * 32;
constexpr int kRing = 48;          // product slots: A tile then B tile, 1 KB each
constexpr int kUnit = 64;          // C tiles per unit (one TMEM half)
constexpr int kHalfCols = 256;     // TMEM columns per half
constexpr int kTmemCols = 2 * kHalfCols;
constexpr int kMaxCRow = 2048;     // ColIdxC entries of a row staged for the position search
constexpr int kMaxA = 256;         // A entries of a row handled per enumeration chunk
constexpr int kPad = 3 * 512;      // A operand rows read before / after a slot's tile
constexpr int kRingOff = kPad;
constexpr int kColOff = kPad + kRing * 1024 + kPad;
constexpr int kKOff = kColOff + kMaxCRow * 4;
constexpr int kRbOff = kKOff + kMaxA * 4;
constexpr int kOffOff = kRbOff + kMaxA * 4;
constexpr int kRecOff = kOffOff + (kMaxA + 1) * 4 + 12;
constexpr int kBarOff = (kRecOff + kRing * 4 + 15) & ~15;
constexpr int kNumBars = 2 * kRing + 4 + 1;
constexpr int kSmem = kBarOff + kNumBars * 8 + 16 + 1024;

struct SpTcArgs
{
    int mb;
    int64_t nnzc; // C tiles past nnzc (a capacity below row_ptr_c[mb]) are neither read nor written
    const int *rpa, *cia, *rpb, *cib, *rpc, *cic;
    const uint16_t *va, *vb;
    void *vc;
    int out_type;
    float alpha, beta;
    int num_iter;
    uint64_t limit_ns;
};

__device__ __forceinline__ void sp_flag(int code) { atomicExch(&g_sptc_error, code); }

// C tiles of block-row i that lie below the caller's bound nnzc
__device__ __forceinline__ int row_tiles(const SpTcArgs &p, int i, int c0)
{
    const int64_t c1 = min((int64_t)p.rpc[i + 1], p.nnzc);
    return c1 > c0 ? (int)(c1 - c0) : 0;
}

__device__ __forceinline__ void cp16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_arrive_on(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// first index in sorted a[0..n) with a[idx] >= v
__device__ __forceinline__ int lower_bound(const int *a, int n, int v)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        const int m = (lo + hi) >> 1;
        if (a[m] < v)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

// last index e in [0, n) with off[e] <= f (off ascending, off[0] = 0)
__device__ __forceinline__ int entry_of(const int *off, int n, int f)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int m = (lo + hi + 1) >> 1;
        if (off[m] <= f)
            lo = m;
        else
            hi = m - 1;
    }
    return lo;
}

template <bool BF16>
__global__ void __launch_bounds__(kThreads, 1) spgemm_tc05_kernel(const __grid_constant__ SpTcArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = smem_raw + ((1024u - (uint32_t)(reinterpret_cast<uintptr_t>(smem_raw) & 1023u)) & 1023u);
    int *sCol = reinterpret_cast<int *>(smem + kColOff);
    int *sK = reinterpret_cast<int *>(smem + kKOff);
    int *sRb = reinterpret_cast<int *>(smem + kRbOff);
    int *sOff = reinterpret_cast<int *>(smem + kOffOff);
    volatile int *rec = reinterpret_cast<volatile int *>(smem + kRecOff);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kBarOff);
    uint64_t *empty = full + kRing;
    uint64_t *tfull = empty + kRing;  // [2] a unit's MMAs are complete
    uint64_t *tempty = tfull + 2;     // [2] a TMEM half is drained and zeroed
    uint64_t *fin = tempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(fin + 1);
    const uint32_t ring = tc::smem_u32(smem + kRingOff);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t limit = p.limit_ns;

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kRing; ++s)
        {
            tc::mbar_init(&full[s], 33); // 32 lanes (with their copies) + the record writer
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b)
        {
            tc::mbar_init(&tfull[b], 1);
            tc::mbar_init(&tempty[b], 4);
        }
        tc::mbar_init(fin, 1);
        tc::fence_mbar_init();
    }
    if (warp == 1)
    {
        tc::tmem_alloc(tmem_slot, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0)
    {
        // ---- planner / loader ----
        int n = 0; // records pushed
        bool ok = true;
        // claim ring slot n (all lanes): wait until its previous record is consumed
        auto claim = [&](int &ds) -> bool {
            ds = n % kRing;
            if (n >= kRing)
            {
                const bool w = tc::mbar_wait_bounded(&empty[ds], ((n / kRing) - 1) & 1, limit);
                if (!__all_sync(0xffffffffu, w))
                {
                    sp_flag(1);
                    return false;
                }
            }
            return true;
        };
        for (int i = blockIdx.x; i < p.mb && ok; i += gridDim.x)
        {
            const int c0 = p.rpc[i], nt = row_tiles(p, i, c0);
            if (nt <= 0)
                continue;
            const int a0 = p.rpa[i], na = p.rpa[i + 1] - a0;
            const bool col_staged = nt <= kMaxCRow;
            __syncwarp();
            if (col_staged)
                for (int t = lane; t < nt; t += 32)
                    sCol[t] = p.cic[c0 + t];
            __syncwarp();
            for (int lo = 0; lo < nt && ok; lo += kUnit)
            {
                const int hi = min(nt, lo + kUnit);
                for (int ach = 0; ach < na && ok; ach += kMaxA)
                {
                    const int nch = min(kMaxA, na - ach);
                    // B-row ranges of this chunk's A entries and their prefix
                    int total = 0;
                    for (int base = 0; base < nch; base += 32)
                    {
                        const int e = base + lane;
                        int len = 0;
                        if (e < nch)
                        {
                            const int k = p.cia[a0 + ach + e];
                            const int rb = p.rpb[k];
                            len = p.rpb[k + 1] - rb;
                            sK[e] = k;
                            sRb[e] = rb;
                        }
                        int pre = len;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1)
                        {
                            const int y = __shfl_up_sync(0xffffffffu, pre, o);
                            if (lane >= o)
                                pre += y;
                        }
                        if (e < nch)
                            sOff[e] = total + pre - len;
                        total += __shfl_sync(0xffffffffu, pre, 31);
                    }
                    if (lane == 0)
                        sOff[nch] = total;
                    __syncwarp();
                    for (int fb = 0; fb < total && ok; fb += 32)
                    {
                        const int f = fb + lane;
                        int pos = -1, e = 0, eb = 0;
                        if (f < total)
                        {
                            e = entry_of(sOff, nch, f);
                            eb = sRb[e] + (f - sOff[e]);
                            const int j = p.cib[eb];
                            const int q = col_staged ? lower_bound(sCol, nt, j) : lower_bound(p.cic + c0, nt, j);
                            const int cj = q < nt ? (col_staged ? sCol[q] : p.cic[c0 + q]) : -1;
                            if (cj == j && q >= lo && q < hi)
                                pos = q - lo;
                        }
                        uint32_t hits = __ballot_sync(0xffffffffu, pos >= 0);
                        while (hits)
                        {
                            const int src = __ffs(hits) - 1;
                            hits &= hits - 1;
                            const int s_pos = __shfl_sync(0xffffffffu, pos, src);
                            const int s_ea = a0 + ach + __shfl_sync(0xffffffffu, e, src);
                            const int s_eb = __shfl_sync(0xffffffffu, eb, src);
                            int ds;
                            if (!claim(ds))
                            {
                                ok = false;
                                break;
                            }
                            const uint32_t sa = ring + ds * 1024, sb = sa + 512;
                            const int off = tile_swz(lane >> 1, lane & 1);
                            cp16(sa + off, p.va + (int64_t)s_ea * 256 + lane * 8);
                            cp16(sb + off, p.vb + (int64_t)s_eb * 256 + lane * 8);
                            cp_arrive_on(&full[ds]);
                            if (lane == 0)
                            {
                                rec[ds] = s_pos;
                                tc::mbar_arrive(&full[ds]);
                            }
                            ++n;
                        }
                    }
                    __syncwarp();
                }
                // end of unit
                int ds;
                if (!ok || !claim(ds))
                {
                    ok = false;
                    break;
                }
                if (lane == 0)
                    rec[ds] = -1;
                __syncwarp();
                tc::mbar_arrive(&full[ds]);
                if (lane == 0)
                    tc::mbar_arrive(&full[ds]);
                ++n;
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    else if (warp == 1)
    {
        // ---- MMA issue (one thread) ----
        if (lane == 0)
        {
            const uint32_t idesc = tc::idesc_f16(BF16, 64, 16, 0, 1);
            int n = 0, u = 0;
            bool ok = true;
            for (int i = blockIdx.x; i < p.mb && ok; i += gridDim.x)
            {
                const int nt = row_tiles(p, i, p.rpc[i]);
                for (int lo = 0; lo < nt && ok; lo += kUnit, ++u)
                {
                    const int b = u & 1;
                    if (!tc::mbar_wait_bounded(&tempty[b], (u >> 1) & 1, limit))
                    {
                        sp_flag(2);
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    while (true)
                    {
                        const int ds = n % kRing;
                        if (!tc::mbar_wait_bounded(&full[ds], (n / kRing) & 1, limit))
                        {
                            sp_flag(3);
                            ok = false;
                            break;
                        }
                        // the copies are generic-proxy writes: order them before
                        // the tensor core's reads
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        tc::tc_fence_after();
                        const int s = rec[ds];
                        ++n;
                        if (s < 0)
                        {
                            tc::mbar_arrive(&empty[ds]);
                            tc::mma_commit(&tfull[b]);
                            break;
                        }
                        const int q = s & 3, cb = s >> 2;
                        const uint32_t sa = ring + ds * 1024, sb = sa + 512;
                        const uint64_t ad = tc::desc_kmajor_sw32(sa - q * 512);
                        const uint64_t bd = tc::desc_mnmajor_sw32(sb);
                        uint32_t off[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
                        off[q] = 0xffff0000u; // write lanes 32q .. 32q + 15 only
                        const uint32_t d = tmem + b * kHalfCols + cb * 16;
                        for (int it = 0; it < p.num_iter; ++it)
                            tc::mma_f16_ss_lanes(d, ad, bd, idesc, off);
                        tc::mma_commit(&empty[ds]);
                    }
                }
            }
            tc::mma_commit(fin);
            if (!tc::mbar_wait_bounded(fin, 0, limit))
                sp_flag(4);
        }
        __syncwarp();
    }
    else
    {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 ----
        const int q = warp & 3;
        const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
        uint32_t zero[16];
#pragma unroll
        for (int t = 0; t < 16; ++t)
            zero[t] = 0u;
        for (int c = 0; c < kTmemCols; c += 16)
            tc::tmem_st16(tmem + lane_addr + c, zero);
        tc::tmem_st_wait();
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0)
        {
            tc::mbar_arrive(&tempty[0]);
            tc::mbar_arrive(&tempty[1]);
        }
        const bool f32 = p.out_type == KAMI_F32, bf = p.out_type == KAMI_BF16;
        int u = 0;
        bool ok = true;
        for (int i = blockIdx.x; i < p.mb && ok; i += gridDim.x)
        {
            const int c0 = p.rpc[i], nt = row_tiles(p, i, c0);
            for (int lo = 0; lo < nt; lo += kUnit, ++u)
            {
                const int b = u & 1;
                const int ntile = min(kUnit, nt - lo);
                const bool done = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&tfull[b], (u >> 1) & 1, limit));
                tc::tc_fence_after();
                if (!done)
                {
                    sp_flag(5);
                    ok = false;
                    break;
                }
                for (int cb = 0; cb * 4 < ntile; ++cb)
                {
                    const uint32_t addr = tmem + lane_addr + b * kHalfCols + cb * 16;
                    uint32_t v[16];
                    tc::tmem_ld16(addr, v);
                    tc::tmem_ld_wait();
                    tc::tmem_regs_ready(v);
                    tc::tmem_st16(addr, zero);
                    const int s = cb * 4 + q;
                    if (s < ntile && lane < 16)
                    {
                        const int64_t c = c0 + lo + s;
                        float x[16];
#pragma unroll
                        for (int t = 0; t < 16; ++t)
                            x[t] = p.alpha * __uint_as_float(v[t]);
                        if (f32)
                        {
                            float4 *out = reinterpret_cast<float4 *>(reinterpret_cast<float *>(p.vc) + c * 256 +
                                                                     lane * 16);
                            if (p.beta != 0.f)
#pragma unroll
                                for (int t = 0; t < 4; ++t)
                                {
                                    const float4 o = out[t];
                                    x[4 * t] += p.beta * o.x;
                                    x[4 * t + 1] += p.beta * o.y;
                                    x[4 * t + 2] += p.beta * o.z;
                                    x[4 * t + 3] += p.beta * o.w;
                                }
#pragma unroll
                            for (int t = 0; t < 4; ++t)
                                out[t] = make_float4(x[4 * t], x[4 * t + 1], x[4 * t + 2], x[4 * t + 3]);
                        }
                        else
                        {
                            uint4 *out = reinterpret_cast<uint4 *>(reinterpret_cast<uint16_t *>(p.vc) + c * 256 +
                                                                   lane * 16);
                            uint32_t w[8];
                            uint4 o[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
                            if (p.beta != 0.f)
                            {
                                o[0] = out[0];
                                o[1] = out[1];
                            }
                            const uint32_t *ow = reinterpret_cast<const uint32_t *>(o);
#pragma unroll
                            for (int t = 0; t < 8; ++t)
                            {
                                float y0 = x[2 * t], y1 = x[2 * t + 1];
                                if (p.beta != 0.f)
                                {
                                    y0 += p.beta * to_float((uint16_t)(ow[t] & 0xffff), bf);
                                    y1 += p.beta * to_float((uint16_t)(ow[t] >> 16), bf);
                                }
                                const uint16_t h0 = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(y0))
                                                       : __half_as_ushort(__float2half_rn(y0));
                                const uint16_t h1 = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(y1))
                                                       : __half_as_ushort(__float2half_rn(y1));
                                w[t] = (uint32_t)h0 | ((uint32_t)h1 << 16);
                            }
                            out[0] = make_uint4(w[0], w[1], w[2], w[3]);
                            out[1] = make_uint4(w[4], w[5], w[6], w[7]);
                        }
                    }
                }
                tc::tmem_st_wait();
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0)
                    tc::mbar_arrive(&tempty[b]);
            }
        }
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1)
    {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, kTmemCols);
    }
}

} // namespace

// Launch the tcgen05 numeric pass (tile arrays 16-byte aligned).
int spgemm_tc05_launch(bool bf16, int mb, int64_t nnzc, const int *rpa, const int *cia, const int *rpb, const int *cib,
                       const int *rpc, const int *cic, const void *va, const void *vb, void *vc, int out_type,
                       double alpha, double beta, int num_iter, cudaStream_t s)
{
    static int sms[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return fail(KAMI_ERR_UNSUPPORTED, "spgemm tcgen05: device ordinal %d above 63", dev);
    const void *fn = bf16 ? (const void *)spgemm_tc05_kernel<true> : (const void *)spgemm_tc05_kernel<false>;
    if (!sms[dev])
    {
        int n = 0;
        if ((e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
            return cuda_fail(e, "cudaDeviceGetAttribute");
        if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem)) != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(spgemm_tc05_kernel)");
        if ((e = cudaFuncSetAttribute(bf16 ? (const void *)spgemm_tc05_kernel<false>
                                           : (const void *)spgemm_tc05_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem)) != cudaSuccess)
            return cuda_fail(e, "cudaFuncSetAttribute(spgemm_tc05_kernel)");
        sms[dev] = n;
    }
    SpTcArgs a{};
    a.mb = mb;
    a.nnzc = nnzc;
    a.rpa = rpa;
    a.cia = cia;
    a.rpb = rpb;
    a.cib = cib;
    a.rpc = rpc;
    a.cic = cic;
    a.va = reinterpret_cast<const uint16_t *>(va);
    a.vb = reinterpret_cast<const uint16_t *>(vb);
    a.vc = vc;
    a.out_type = out_type;
    a.alpha = (float)alpha;
    a.beta = (float)beta;
    a.num_iter = num_iter;
    a.limit_ns = (uint64_t)(2e9 + (double)num_iter * 2e6); // generous: a unit takes microseconds
    const int grid = mb < sms[dev] ? mb : sms[dev];
    void *args[] = {&a};
    if ((e = cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, (size_t)kSmem, s)) != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(spgemm_tc05_kernel)");
    return KAMI_OK;
}

int spgemm_tc05_read_error(int *flag)
{
    int v = 0, z = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_sptc_error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_sptc_error, &z, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "reading the spgemm tcgen05 status");
    *flag = v;
    return KAMI_OK;
}

} // namespace kami
