// tc05_gemm.cuh -- host interface of the tcgen05 (5th-generation tensor core)
// block GEMM variant: operands staged in shared memory by TMA, accumulators
// in tensor memory (TMEM).  Implemented in tc05_gemm.cu.
#pragma once
#include "kami_common.cuh"

namespace kami {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);

// True when AUTO should try the tcgen05 variant first for this request.
bool tc05_prefer(int in_type, int partition, int M, int N, int K, int a_layout, int b_layout);

// True when AUTO should keep A in tensor memory (the TS form).
bool tc05_prefer_ts(int M, int a_layout);

// Resolve (without launching) the tcgen05 launch for a request; a_tmem
// selects the form with A resident in tensor memory.
int tc05_plan(int in_type, int out_type, int partition, int P, int M, int N, int K, int64_t batch, int a_layout,
              int b_layout, LaunchInfo *info, int a_tmem);

// Launch; returns KAMI_ERR_UNSUPPORTED (and launches nothing) when the
// request is outside what the variant handles.
int tc05_launch(const GemmArgs &g, int in_type, int partition, int P, void *workspace, size_t ws_bytes,
                cudaStream_t stream, int a_tmem);

// Read and clear the device-side error flag of the tcgen05 kernels (0 = none,
// 1 = operand loads timed out, 2 = MMA completion timed out).  Synchronous.
int tc05_read_error(int *flag);

// Launch a one-thread kernel whose bounded wait must time out (status 4).
int tc05_selftest_bounded_wait(uint64_t limit_ns, cudaStream_t s);

// Fused backward (dA = dC B^T, dB = A^T dC) of packed row-major problems;
// KAMI_ERR_UNSUPPORTED (nothing launched) outside FP16 / BF16 with M, N, K in
// {64, 128}.
int tc05_backward_launch(int in_type, int out_type, int M, int N, int K, int64_t batch, const void *A, const void *B,
                         const void *dC, void *dA, void *dB, cudaStream_t stream);

} // namespace kami
