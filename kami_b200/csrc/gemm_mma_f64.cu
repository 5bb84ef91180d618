// gemm_mma_f64.cu -- compiled instances of the mma.sync (DMMA m16n8k8) block
// GEMM for FP64 (see mma_engine.cuh).
//
// Shapes: per-rank register budgets.  Register-resident FP64 tops out at
// 64^3 per CTA: a 128^3 problem would need 2D P = 4 (512 threads) at ~240
// registers per thread, beyond the 64K-register file; the reference folds K
// for its 1D 128^3 variant instead (batched_gemm_1d_double_mma_128.cu).
#include "mma_engine.cuh"

#define KAMI_F64_TABLE(X)                                                                          \
    X(16, 16, 16, 1, 1) X(16, 16, 16, 1, 2) X(16, 16, 16, 1, 3)                                    \
    X(32, 32, 32, 1, 1) X(32, 32, 32, 2, 1) X(32, 32, 32, 1, 2) X(32, 32, 32, 2, 2)                \
    X(32, 32, 32, 1, 3) X(32, 32, 32, 2, 3)                                                        \
    X(64, 64, 64, 4, 1) X(64, 64, 64, 2, 2) X(64, 64, 64, 4, 2)                \
    X(64, 64, 64, 2, 3)

namespace kami {
static const MmaInstance kF64[] = {
#define X(BM, BN, BK, P, PART) KAMI_MMA_INSTANCE(TrF64, KAMI_F64, BM, BN, BK, P, PART),
    KAMI_F64_TABLE(X)
#undef X
};
const MmaInstance *mma_instances_f64(int *count)
{
    *count = (int)(sizeof(kF64) / sizeof(kF64[0]));
    return kF64;
}
} // namespace kami
