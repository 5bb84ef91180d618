// grouped.cuh -- device descriptors of the uneven (grouped) batched GEMM,
// shared by its three kernels: the mma.sync warp-grid kernel (grouped.cu),
// the tcgen05 kernel (grouped_tc05.cu, FP16 / BF16) and the staged DMMA
// kernel (grouped_f64.cu, FP64).
#pragma once
#include "kami_common.cuh"

namespace kami {

// One problem: shape, warp partition (mma.sync kernel), element offsets of
// A (M x K), B (N x K) and C (M x N) and their leading dimensions.
struct GroupedDesc
{
    int M, N, K, cfg;
    int64_t a_off, b_off, c_off;
    int lda, ldb, ldc;
    int ext; // tcgen05 plans: extent of the work item this problem belongs to (grouped_tc05.cu, item_at)
};

struct GroupedParams
{
    const GroupedDesc *desc; // problems in schedule order
    const int *cta_begin;    // ctas + 1 offsets into desc
    const void *A;
    const void *B;
    void *C;
    int out_type;
    double alpha, beta;
    int num_iter;
    int small_begin, small_end; // desc range of problems run by single warps
};

// tcgen05 grouped kernel (grouped_tc05.cu): entry point, launch geometry and
// the device status of its bounded waits.
const void *grouped_tc05_fn(bool bf16, bool packed);
int grouped_tc05_threads();
int grouped_tc05_smem();
int grouped_tc05_ctas_per_sm();
int grouped_tc05_launch(const GroupedParams &p, bool bf16, bool packed, int ctas, cudaStream_t s);
int grouped_tc05_read_error(int *flag);

// staged FP64 grouped kernel (grouped_f64.cu)
const void *grouped_f64s_fn();
int grouped_f64s_threads();
int grouped_f64s_smem();
int grouped_f64s_launch(const GroupedParams &p, int ctas, cudaStream_t s);
int grouped_f64s_read_error(int *flag);

} // namespace kami
