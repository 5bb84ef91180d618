// spmm_tc05.cu -- block SpMM C = A B (A BSR with 16 x 16 tiles, B dense
// K x N row-major or N x K row-major (the reference's layout), C dense
// M x N) on the 5th-generation tensor cores, for the streamed regime of large
// sparse matrices (K beyond a staged panel).
//
// A block-row of C is only 16 rows high, below the smallest tcgen05 MMA
// (M = 64).  So each block-row is computed transposed:
//   C_i^T (N x 16) = sum over the row's tiles (i, k) of  B_k^T (N x 16) A_ik^T,
// where B_k is rows 16k .. 16k + 15 of B.  B_k^T is the MMA's A operand with
// M = 128 columns of B per MMA, read MN-major straight from B's row-major
// rows (TMA boxes of 64 columns x 16 rows, 128-byte swizzle) -- or, for B
// as N x K, K-major: the slice's 16 K values of a column are 32 contiguous
// bytes, loaded by TMA boxes of 16 x 128 rows with 32-byte swizzling (one
// 32-byte request per column -- boxes of 8 values, two 16-byte requests per
// column, measured 38.9 us, no faster than the mma.sync form); the tile A_ik
// is the MMA's B operand with N = 16 (its rows) and K = 16 (its columns),
// K-major without swizzle: the loaders write its 16-byte row halves into the
// 8-row x 16-byte core matrices the descriptor describes.  The accumulator of
// a block-row (TMEM lanes = columns of C, TMEM columns = its 16 rows) is read
// back one lane per column, so every store instruction of the epilogue
// writes 32 consecutive columns of one C row -- coalesced with no transpose.
//
// Four CTAs per SM walk the block-rows i = blockIdx.x, + gridDim.x, ...:
//   warps 0, 6  load the tiles alternately (tile j by warp 0 when j is even):
//               each tile's B slice (TMA, lane 0) and the tile itself
//               (cp.async, all lanes, each arriving on the slot's barrier
//               when its copy lands) into a ring of at least two slots.  A
//               loader at tile j waited, at its previous tile j - 2, for the
//               commit of tile j - 2 - S, so the MMAs (consumed in order)
//               have already freed its own previous fill of the slot: no
//               parity wait runs more than one phase ahead;
//   warp 1      lane 0 issues the MMAs (ceil(N / 128) per tile and repeat)
//               into a ring of four TMEM accumulators, and owns the TMEM
//               allocation;
// both read the row pointers of the next 32 block-rows and the column
// indices of the next 32 tiles one per lane and pass them on by shuffle, so
// no dependent index load sits between two tiles (read one at a time, their
// latency made this kernel slower than the mma.sync form);
//   warps 2-5   the epilogue: TMEM -> registers -> C with alpha / beta and
//               the output type.
// A block column outside [0, kb) reads rows past the end of B, which the
// tensor copy fills with zeros (the mma.sync kernels skip such tiles).  Every
// mbarrier wait is bounded; a timeout sets g_spmm_tc_error.
#include <cstdint>
#include <mutex>

#include "kami_common.cuh"
#include "tc05_ptx.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// device status of the bounded waits (read and cleared by kami_device_status)
__device__ int g_spmm_tc_error = 0;

namespace {

// Four CTAs per SM: the per-tile work is two tiny MMAs, so a CTA's loading
// lanes and single MMA-issuing lane set the pace (one loader: ~850 and ~430
// cycles a tile); four CTAs run four such pipelines side by side (one CTA
// per SM: 55 us for the n = 16384, 1 % case; two: 37 us; four: 27.6 us), and
// two loader warps per CTA bring it to 25.7 us.  60 registers x 224 threads
// x 4 and 4 x 128 TMEM columns fit the SM.
constexpr int kCtasPerSm = 4;                 // resident CTAs per SM (the grid is this many per SM)
constexpr int kEpiGroups = 1;                 // epilogue groups of four warps
constexpr int kAccs = 4;                      // TMEM accumulators (block-rows in flight) per CTA
constexpr int kMaxSlots = 16;
constexpr int kLoadWarp2 = 2 + 4 * kEpiGroups; // the second loader warp, after the epilogue
constexpr int kThreads = (kLoadWarp2 + 1) * 32;

struct SpTcParams
{
    int mb, kb, N;
    int npad;          // N rounded up to 128
    int slot_bytes;    // B slice (npad x 16 x 2 bytes) + 512-byte tile, 1024-byte multiple
    int slots;
    int acc_cols;      // TMEM columns of one accumulator: 16 per 128 columns of C
    uint32_t tmem_cols;
    const int *rowptr;
    const int *colidx;
    const uint16_t *vals;
    void *C;
    int64_t ldc;
    int out_type;
    float alpha, beta;
    int num_iter;
    uint32_t idesc;
    uint64_t timeout_ns;
};

__device__ __forceinline__ void sp_flag(int code) { atomicExch(&g_spmm_tc_error, code); }

__device__ __forceinline__ void cp16(uint32_t dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_arrive_on(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// K-major operand without swizzle: 8-row x 16-byte core matrices, `lbo`
// bytes apart along K and `sbo` bytes apart along the rows
__device__ __forceinline__ uint64_t desc_kmajor_noswz(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46; // version
    return d;               // layout type 0: no swizzle
}

__device__ __forceinline__ float to_f(uint16_t b, bool bf)
{
    return bf ? __bfloat162float(__ushort_as_bfloat16(b)) : __half2float(__ushort_as_half(b));
}

// KMAJ: B is N x K and its slices are K-major (32-byte rows, 4 KB per 128
// columns); else B is K x N and its slices MN-major (boxes of 64 columns).
template <bool BF16, bool KMAJ>
__global__ void __launch_bounds__(kThreads, kCtasPerSm) spmm_tc05_kernel(const __grid_constant__ CUtensorMap tmB,
                                                                const SpTcParams p)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = p.slots;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)S * p.slot_bytes);
    uint64_t *empty = full + S;
    uint64_t *accf = empty + S;
    uint64_t *acce = accf + kAccs;
    uint64_t *fin = acce + kAccs;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(fin + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t limit = p.timeout_ns;
    const int tile_off = p.npad * 32; // the tile after the B slice in a slot

    if (threadIdx.x == 0)
    {
        for (int s = 0; s < S; ++s)
        {
            tc::mbar_init(&full[s], 33); // 32 tile copies + the TMA's expect-tx arrival
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < kAccs; ++b)
        {
            tc::mbar_init(&accf[b], 1);
            tc::mbar_init(&acce[b], 4);
        }
        tc::mbar_init(fin, 1);
        tc::fence_mbar_init();
    }
    if (warp == 1)
    {
        tc::tmem_alloc(tmem_slot, p.tmem_cols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 || warp == kLoadWarp2)
    {
        // ---- loads: the B slice by TMA (lane 0), the tile by cp.async; this
        //      warp takes the tiles j with j % 2 == lid ----
        const int lid = warp == 0 ? 0 : 1;
        if (lane == 0)
            tc::prefetch_tmap(&tmB);
        const uint32_t base = tc::smem_u32(smem);
        const int r = lane >> 1, h = lane & 1; // this lane's 16 bytes of the tile: row r, half h
        const uint32_t tdst = (uint32_t)((r >> 3) * 256 + h * 128 + (r & 7) * 16);
        const int nbox = p.npad / 64;
        int j = 0;
        bool ok = true;
        for (int i0 = blockIdx.x; i0 < p.mb && ok; i0 += 32 * gridDim.x)
        {
            // row pointers of the next 32 block-rows of this CTA, one per lane
            const int il = i0 + lane * gridDim.x;
            const int le0 = il < p.mb ? p.rowptr[il] : 0, le1 = il < p.mb ? p.rowptr[il + 1] : 0;
            for (int u = 0; u < 32 && ok; ++u)
            {
            if (i0 + u * gridDim.x >= p.mb)
                break;
            const int e0 = __shfl_sync(0xffffffffu, le0, u), e1 = __shfl_sync(0xffffffffu, le1, u);
            for (int eb = e0; eb < e1 && ok; eb += 32)
            {
            const int kl = eb + lane < e1 ? p.colidx[eb + lane] : 0; // 32 column indices, one per lane
            const int ee = e1 - eb < 32 ? e1 - eb : 32;
            for (int t = 0; t < ee; ++t, ++j)
            {
                if ((j & 1) != lid)
                    continue; // the other loader's tile
                const int e = eb + t;
                const int s = j % S;
                bool w = true;
                if (j >= S && lane == 0)
                    w = tc::mbar_wait_bounded(&empty[s], ((j / S) - 1) & 1, limit);
                if (!__shfl_sync(0xffffffffu, w, 0))
                {
                    if (lane == 0)
                        sp_flag(1);
                    ok = false;
                    break;
                }
                const uint32_t slot = base + (uint32_t)s * p.slot_bytes;
                const int k = __shfl_sync(0xffffffffu, kl, t);
                if (lane == 0)
                {
                    const int krow = (k >= 0 && k < p.kb) ? k * 16 : p.kb * 16; // past the end: zeros
                    tc::mbar_expect_tx(&full[s], (uint32_t)(nbox * 2048));
                    if (KMAJ) // K values krow .. krow + 15 of 128 columns per box
                        for (int c = 0; c < nbox / 2; ++c)
                            tc::tma_load_3d(smem + (size_t)s * p.slot_bytes + c * 4096, &tmB, &full[s], krow, c * 128,
                                            0);
                    else
                        for (int b = 0; b < nbox; ++b)
                            tc::tma_load_3d(smem + (size_t)s * p.slot_bytes + b * 2048, &tmB, &full[s], b * 64, krow,
                                            0);
                }
                cp16(slot + tile_off + tdst, p.vals + (int64_t)e * 256 + r * 16 + h * 8);
                cp_arrive_on(&full[s]);
            }
            }
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    else if (warp == 1)
    {
        // ---- MMA issue (lane 0; the warp prefetches the row pointers) ----
        {
            const uint32_t base = tc::smem_u32(smem);
            const int nch = p.npad / 128;
            int j = 0, q = 0;
            bool ok = true;
            int lT = 0;
            for (int i = blockIdx.x; i < p.mb && ok; i += gridDim.x, ++q)
            {
                if ((q & 31) == 0)
                {
                    const int il = i + lane * gridDim.x;
                    lT = il < p.mb ? p.rowptr[il + 1] - p.rowptr[il] : 0;
                }
                const int T = __shfl_sync(0xffffffffu, lT, q & 31);
                if (lane != 0)
                {
                    j += T;
                    continue;
                }
                const int b = q % kAccs;
                if (q >= kAccs && !tc::mbar_wait_bounded(&acce[b], ((q / kAccs) - 1) & 1, limit))
                {
                    sp_flag(2);
                    break;
                }
                tc::tc_fence_after();
                const uint32_t acc = tmem + (uint32_t)(b * p.acc_cols);
                for (int t = 0; t < T; ++t, ++j)
                {
                    const int s = j % S;
                    if (!tc::mbar_wait_bounded(&full[s], (j / S) & 1, limit))
                    {
                        sp_flag(3);
                        ok = false;
                        break;
                    }
                    fence_async_smem(); // the tile's cp.async writes, for the async proxy
                    tc::tc_fence_after();
                    const uint32_t slot = base + (uint32_t)s * p.slot_bytes;
                    const uint64_t bd = desc_kmajor_noswz(slot + p.npad * 32, 128, 256);
                    for (int it = 0; it < p.num_iter; ++it)
                        for (int c = 0; c < nch; ++c)
                        {
                            // columns 128c .. of the slice, 4 KB in both layouts
                            const uint64_t ad = KMAJ ? tc::desc_kmajor_sw32(slot + c * 4096)
                                                     : tc::desc_mnmajor_sw128(slot + c * 4096, 2048);
                            tc::mma_f16_ss(acc + (uint32_t)(c * 16), ad, bd, p.idesc, (t > 0 || it > 0) ? 1u : 0u);
                        }
                    tc::mma_commit(&empty[s]);
                }
                if (!ok)
                    break;
                tc::mma_commit(&accf[b]);
            }
            if (lane == 0)
            {
                tc::mma_commit(fin);
                if (!tc::mbar_wait_bounded(fin, 0, limit))
                    sp_flag(4);
            }
        }
        __syncwarp();
    }
    else
    {
        // ---- epilogue: group (warp - 2) / 4; warp w reads TMEM lanes 32 (w % 4) .. + 31 ----
        const int grp = (warp - 2) >> 2, quad = warp & 3;
        const uint32_t lane_addr = (uint32_t)(quad * 32) << 16;
        const int nch = p.npad / 128;
        const bool plain = p.alpha == 1.f && p.beta == 0.f;
        int q = grp;
        for (int i = blockIdx.x + grp * gridDim.x; i < p.mb; i += kEpiGroups * gridDim.x, q += kEpiGroups)
        {
            const int b = q % kAccs;
            const bool done = __all_sync(0xffffffffu, tc::mbar_wait_bounded(&accf[b], (q / kAccs) & 1, limit));
            tc::tc_fence_after();
            if (!done)
            {
                sp_flag(5);
                break;
            }
            const bool any = p.rowptr[i + 1] > p.rowptr[i];
            for (int c = 0; c < nch; ++c)
            {
                uint32_t v[16];
                if (any)
                {
                    tc::tmem_ld16(tmem + lane_addr + (uint32_t)(b * p.acc_cols + c * 16), v);
                    tc::tmem_ld_wait();
                    tc::tmem_regs_ready(v);
                }
                const int n = c * 128 + quad * 32 + lane;
                if (n < p.N)
                {
#pragma unroll
                    for (int r = 0; r < 16; ++r)
                    {
                        float x = any ? __uint_as_float(v[r]) : 0.f;
                        const int64_t off = (int64_t)(i * 16 + r) * p.ldc + n;
                        if (p.out_type == KAMI_F32)
                        {
                            float *dst = reinterpret_cast<float *>(p.C) + off;
                            if (!plain)
                                x = p.alpha * x + (p.beta != 0.f ? p.beta * *dst : 0.f);
                            *dst = x;
                        }
                        else
                        {
                            const bool bf = p.out_type == KAMI_BF16;
                            uint16_t *dst = reinterpret_cast<uint16_t *>(p.C) + off;
                            if (!plain)
                                x = p.alpha * x + (p.beta != 0.f ? p.beta * to_f(*dst, bf) : 0.f);
                            *dst = bf ? __bfloat16_as_ushort(__float2bfloat16_rn(x)) : __half_as_ushort(__float2half_rn(x));
                        }
                    }
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
    if (warp == 1)
    {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, p.tmem_cols);
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
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

} // namespace

// The tcgen05 SpMM for one problem with B K x N row-major, or N x K
// row-major when b_nk (16-byte aligned, ldb a multiple of 8), tiles 16-byte
// aligned, N <= 512; else KAMI_ERR_UNSUPPORTED without launching anything.
int spmm_tc05_launch(bool bf16, int out_type, int mb, int kb, int N, const int *rowptr, const int *colidx,
                     const void *vals, const void *B, int64_t ldb, bool b_nk, void *C, int64_t ldc, double alpha,
                     double beta, int num_iter, cudaStream_t s)
{
    if (N < 1 || N > 512 || mb < 1 || kb < 1 || (reinterpret_cast<uintptr_t>(B) & 15) || (ldb & 7) ||
        (reinterpret_cast<uintptr_t>(vals) & 15) || (int64_t)kb * 16 > 0x7fffffff)
        return KAMI_ERR_UNSUPPORTED;
    EncodeTiledFn fn = encode_fn();
    if (!fn)
        return KAMI_ERR_UNSUPPORTED;
    CUtensorMap map;
    const int64_t K = (int64_t)kb * 16;
    // K x N: boxes of 64 columns x 16 rows, 128-byte swizzle; N x K: boxes of
    // 16 K values (32 bytes) x 128 rows, 32-byte swizzle
    const int64_t rows = b_nk ? N : K;
    cuuint64_t dims[3] = {(cuuint64_t)(b_nk ? K : N), (cuuint64_t)rows, 1};
    cuuint64_t strides[2] = {(cuuint64_t)(ldb * 2), (cuuint64_t)(ldb * 2 * rows)};
    cuuint32_t box[3] = {b_nk ? 16u : 64u, b_nk ? 128u : 16u, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    if (fn(&map, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(B),
           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           b_nk ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return KAMI_ERR_UNSUPPORTED;
    SpTcParams p{};
    p.mb = mb;
    p.kb = kb;
    p.N = N;
    p.npad = (N + 127) / 128 * 128;
    p.slot_bytes = (p.npad * 32 + 512 + 1023) / 1024 * 1024;
    const int budget = 228 * 1024 / kCtasPerSm - 1024 - 1024 - 512;
    p.slots = budget / p.slot_bytes < kMaxSlots ? budget / p.slot_bytes : kMaxSlots;
    if (p.slots < 2) // the two loaders need two slots (see the kernel)
        return KAMI_ERR_UNSUPPORTED;
    p.acc_cols = (p.npad / 128) * 16;
    uint32_t cols = 32;
    while ((int)cols < kAccs * p.acc_cols)
        cols <<= 1;
    p.tmem_cols = cols;
    p.rowptr = rowptr;
    p.colidx = colidx;
    p.vals = reinterpret_cast<const uint16_t *>(vals);
    p.C = C;
    p.ldc = ldc;
    p.out_type = out_type;
    p.alpha = (float)alpha;
    p.beta = (float)beta;
    p.num_iter = num_iter;
    // A (B's slice) MN-major for K x N, K-major for N x K; B (the tile) K-major
    p.idesc = tc::idesc_f16(bf16, 128, 16, b_nk ? 0 : 1, 0);
    p.timeout_ns = (uint64_t)(2e9 + (double)num_iter * 1e6);
    const size_t smem = (size_t)p.slots * p.slot_bytes + (2 * p.slots + 2 * kAccs + 1) * 8 + 16 + 1024;
    const void *kfn = b_nk ? (bf16 ? (const void *)&spmm_tc05_kernel<true, true>
                                   : (const void *)&spmm_tc05_kernel<false, true>)
                           : (bf16 ? (const void *)&spmm_tc05_kernel<true, false>
                                   : (const void *)&spmm_tc05_kernel<false, false>);
    static std::once_flag once[4];
    cudaError_t e = cudaSuccess;
    std::call_once(once[(bf16 ? 1 : 0) + (b_nk ? 2 : 0)],
                   [&] { e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024); });
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaFuncSetAttribute(spmm_tc05_kernel)");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = mb < sms * kCtasPerSm ? mb : sms * kCtasPerSm;
    void *args[] = {&map, &p};
    e = cudaLaunchKernel(kfn, dim3(grid), dim3(kThreads), args, smem, s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaLaunchKernel(spmm_tc05_kernel)");
    return KAMI_OK;
}

int spmm_tc05_read_error(int *flag)
{
    int v = 0, z = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_spmm_tc_error, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbol(g_spmm_tc_error, &z, sizeof(int));
    if (e != cudaSuccess)
        return cuda_fail(e, "reading the tcgen05 SpMM status");
    *flag = v;
    return KAMI_OK;
}

} // namespace kami
