// host_pipeline.cu -- the batched block GEMM on HOST buffers, with the
// copies overlapped with the computation.
//
// The reference's programs copy A and B to the device, launch, and copy C
// back, one after the other (e.g. batched_gemm_2d_double_mma.cu: cudaMemcpy,
// kernel, cudaMemcpy).  Here the batch is cut into chunks of about one
// problem per four SMs.  The input copies run back to back on one stream, the
// result copies on another (each direction on its own copy engine), and each
// chunk's product is launched on one of several compute streams as soon as
// its inputs have landed, so it takes the SMs the earlier chunks leave free.
// The repeated-products kernel runs one CTA per SM here: SMs then free up in
// the order they started, each runs its problems back to back, and the last
// results arrive spread over time as the first inputs did, so that little
// but the first chunk's input copy and the last chunk's result copy is left
// outside the overlap.  (FP16 128^3 x 592, 1000 repeats: copy in 0.71 ms,
// products 1.30 ms, copy out 0.68 ms; two chunks of two waves 1.99 ms, 4
// chunks of 148 on two CTAs per SM 1.64-1.67 ms, 16 chunks of 37 at one CTA
// per SM 1.555 ms.)  Each chunk has its own device buffers (a ring of
// buffers once the whole batch would need more than 1 GiB).  The caller's
// stream waits for the last copy, so work queued after the call sees C
// complete.
#include <algorithm>
#include <map>
#include <mutex>

#include "kami_common.cuh"

namespace kami {

int gemm_batched_hinted(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition,
                        kami_variant_t variant, int M, int N, int K, int P, int alloc_warps, int64_t batch,
                        const void *A, int64_t lda, int64_t strideA, kami_a_layout_t a_layout, const void *B,
                        int64_t ldb, int64_t strideB, kami_b_layout_t b_layout, void *C, int64_t ldc,
                        int64_t strideC, double alpha, double beta, int num_iter, void *workspace, size_t ws_bytes,
                        void *stream, int one_per_sm);

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

namespace {

int esize(int t) { return t == KAMI_F64 ? 8 : t == KAMI_F32 ? 4 : 2; }
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr int kMaxChunks = 16;               // chunks (and device buffers) per call
constexpr int kStreams = 8;                  // compute streams the chunks' products spread over
constexpr size_t kBufCap = (size_t)1 << 30;  // one buffer per chunk up to this many bytes in all

struct Chunking
{
    int64_t chunk;  // problems per chunk
    int64_t chunks; // number of chunks
    int bufs;       // device buffers; chunk c uses buffer c % bufs
    size_t a, b, c; // bytes of one chunk's A, B, C buffers (256-byte multiples)
};

Chunking chunking(int in_type, int out_type, int M, int N, int K, int64_t batch, int sms)
{
    Chunking ch{};
    // about one problem per four SMs per chunk (FP16 128^3 x 592 with 1000
    // repeats: 16 chunks of 37), the products at most one CTA per SM
    const int64_t target = std::max(1, sms / 4);
    ch.chunks = std::min<int64_t>(kMaxChunks, std::max<int64_t>(1, (batch + target - 1) / target));
    ch.chunk = (batch + ch.chunks - 1) / ch.chunks;
    ch.chunks = (batch + ch.chunk - 1) / ch.chunk;
    ch.a = align256((size_t)ch.chunk * M * K * esize(in_type));
    ch.b = align256((size_t)ch.chunk * N * K * esize(in_type));
    ch.c = align256((size_t)ch.chunk * M * N * esize(out_type));
    const size_t per = ch.a + ch.b + ch.c;
    int64_t bufs = ch.chunks;
    if (bufs > 2 && (size_t)bufs * per > kBufCap)
        bufs = std::max<int64_t>(2, (int64_t)(kBufCap / per));
    ch.bufs = (int)bufs;
    return ch;
}

// per device: the copy and compute streams, the events that chain the
// chunks, and a library-owned workspace for callers that pass none
struct DeviceCtx
{
    cudaStream_t h2d = nullptr, d2h = nullptr, comp[kStreams] = {};
    cudaEvent_t entry = nullptr, call_done = nullptr;
    cudaEvent_t h2d_done[kMaxChunks], comp_done[kMaxChunks], d2h_done[kMaxChunks];
    void *ws = nullptr;
    size_t ws_bytes = 0;
    bool ready = false;
};
std::mutex g_mu; // one pipelined call at a time per process (the streams and events are shared)
std::map<int, DeviceCtx> g_ctx;

int get_ctx(int dev, DeviceCtx **out)
{
    DeviceCtx &c = g_ctx[dev];
    if (!c.ready)
    {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&c.h2d, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&c.d2h, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamCreate(host pipeline)");
        for (int i = 0; i < kStreams; ++i)
            if ((e = cudaStreamCreateWithFlags(&c.comp[i], cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate(host pipeline)");
        if ((e = cudaEventCreateWithFlags(&c.entry, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c.call_done, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate(host pipeline)");
        for (int i = 0; i < kMaxChunks; ++i)
            if ((e = cudaEventCreateWithFlags(&c.h2d_done[i], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&c.comp_done[i], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&c.d2h_done[i], cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate(host pipeline)");
        c.ready = true;
    }
    *out = &c;
    return KAMI_OK;
}

} // namespace
} // namespace kami

using namespace kami;

extern "C" {

int kami_gemm_batched_host_workspace_size(kami_dtype_t in_type, kami_dtype_t out_type, int M, int N, int K,
                                          int64_t batch, size_t *bytes)
{
    if (!bytes || M < 1 || N < 1 || K < 1 || batch < 0)
        return fail(KAMI_ERR_INVALID_VALUE, "host gemm: bad shape or null output");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const Chunking ch = chunking(in_type, out_type, M, N, K, std::max<int64_t>(batch, 1), sms);
    *bytes = (size_t)ch.bufs * (ch.a + ch.b + ch.c);
    return KAMI_OK;
}

int kami_gemm_batched_host(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition,
                           kami_variant_t variant, int M, int N, int K, int64_t batch, const void *A, const void *B,
                           void *C, int num_iter, void *workspace, size_t ws_bytes, void *stream)
{
    if (M < 1 || N < 1 || K < 1 || batch < 0 || num_iter < 1)
        return fail(KAMI_ERR_INVALID_VALUE, "host gemm: bad shape, batch or num_iter");
    if (!A || !B || !C)
        return fail(KAMI_ERR_INVALID_VALUE, "host gemm: null host buffer");
    if (batch == 0)
        return KAMI_OK;
    int dev = 0, sms = 148;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const Chunking ch = chunking(in_type, out_type, M, N, K, batch, sms);
    const size_t need = (size_t)ch.bufs * (ch.a + ch.b + ch.c);
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceCtx *ctx = nullptr;
    int st = get_ctx(dev, &ctx);
    if (st)
        return st;
    uint8_t *ws = reinterpret_cast<uint8_t *>(workspace);
    if (ws)
    {
        if (ws_bytes < need)
            return fail(KAMI_ERR_WORKSPACE, "host gemm: workspace of %zu bytes, %zu needed", ws_bytes, need);
    }
    else
    {
        if (ctx->ws_bytes < need)
        {
            if (ctx->ws)
            {
                cudaDeviceSynchronize(); // the old workspace may still be in use
                cudaFree(ctx->ws);
                ctx->ws = nullptr;
                ctx->ws_bytes = 0;
            }
            if ((e = cudaMalloc(&ctx->ws, need)) != cudaSuccess)
                return cuda_fail(e, "cudaMalloc(host gemm workspace)");
            ctx->ws_bytes = need;
        }
        ws = reinterpret_cast<uint8_t *>(ctx->ws);
    }
    cudaStream_t s0 = reinterpret_cast<cudaStream_t>(stream);
    const int isz = esize(in_type), osz = esize(out_type);
    const uint8_t *Ah = reinterpret_cast<const uint8_t *>(A), *Bh = reinterpret_cast<const uint8_t *>(B);
    uint8_t *Ch = reinterpret_cast<uint8_t *>(C);
    // the copies start after the work already queued on the caller's stream
    // and after the previous call's last result copy (whose products precede
    // it) has left the shared workspace
    if ((e = cudaEventRecord(ctx->entry, s0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ctx->h2d, ctx->entry, 0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(ctx->h2d, ctx->call_done, 0)) != cudaSuccess)
        return cuda_fail(e, "host gemm: stream ordering");
    const size_t per = ch.a + ch.b + ch.c;
    for (int64_t c = 0; c < ch.chunks; ++c)
    {
        const int buf = (int)(c % ch.bufs);
        const int64_t p0 = c * ch.chunk, n = std::min(ch.chunk, batch - p0);
        uint8_t *dA = ws + (size_t)buf * per, *dB = dA + ch.a, *dC = dB + ch.b;
        cudaStream_t cs = ctx->comp[c % kStreams];
        // inputs in: a reused buffer is free once chunk c - bufs's product is done
        if (c >= ch.bufs && (e = cudaStreamWaitEvent(ctx->h2d, ctx->comp_done[buf], 0)) != cudaSuccess)
            return cuda_fail(e, "host gemm: stream ordering");
        if ((e = cudaMemcpyAsync(dA, Ah + (size_t)p0 * M * K * isz, (size_t)n * M * K * isz, cudaMemcpyHostToDevice,
                                 ctx->h2d)) != cudaSuccess ||
            (e = cudaMemcpyAsync(dB, Bh + (size_t)p0 * N * K * isz, (size_t)n * N * K * isz, cudaMemcpyHostToDevice,
                                 ctx->h2d)) != cudaSuccess ||
            (e = cudaEventRecord(ctx->h2d_done[buf], ctx->h2d)) != cudaSuccess)
            return cuda_fail(e, "host gemm: input copy");
        // the product: after its inputs, and after chunk c - bufs's C left a reused buffer
        if ((e = cudaStreamWaitEvent(cs, ctx->h2d_done[buf], 0)) != cudaSuccess ||
            (c >= ch.bufs && (e = cudaStreamWaitEvent(cs, ctx->d2h_done[buf], 0)) != cudaSuccess))
            return cuda_fail(e, "host gemm: stream ordering");
        st = gemm_batched_hinted(in_type, out_type, partition, variant, M, N, K, 0, 0, n, dA, K, (int64_t)M * K,
                                 KAMI_A_ROW_MK, dB, K, (int64_t)N * K, KAMI_B_REF_NK, dC, N, (int64_t)M * N, 1.0, 0.0,
                                 num_iter, nullptr, 0, cs, 1);
        if (st)
            return st;
        if ((e = cudaEventRecord(ctx->comp_done[buf], cs)) != cudaSuccess)
            return cuda_fail(e, "host gemm: stream ordering");
        // result out
        if ((e = cudaStreamWaitEvent(ctx->d2h, ctx->comp_done[buf], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(Ch + (size_t)p0 * M * N * osz, dC, (size_t)n * M * N * osz, cudaMemcpyDeviceToHost,
                                 ctx->d2h)) != cudaSuccess ||
            (e = cudaEventRecord(ctx->d2h_done[buf], ctx->d2h)) != cudaSuccess)
            return cuda_fail(e, "host gemm: result copy");
    }
    // the result copies run in order on one stream: the caller's stream
    // continues once the last one is done
    if ((e = cudaEventRecord(ctx->call_done, ctx->d2h)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(s0, ctx->call_done, 0)) != cudaSuccess)
        return cuda_fail(e, "host gemm: stream ordering");
    return KAMI_OK;
}

} // extern "C"
