// gemm_mma_bf16.cu -- compiled instances of the mma.sync block GEMM for
// bfloat16 inputs with FP32 accumulation (see mma_engine.cuh).
#include "mma_engine.cuh"
#include "mma_table_h16.inc"

namespace kami {
using TrBF16 = TrH16<true>;
static const MmaInstance kBF16[] = {
#define X(BM, BN, BK, P, PART) KAMI_MMA_INSTANCE(TrBF16, KAMI_BF16, BM, BN, BK, P, PART),
    KAMI_H16_TABLE(X)
#undef X
};
const MmaInstance *mma_instances_bf16(int *count)
{
    *count = (int)(sizeof(kBF16) / sizeof(kBF16[0]));
    return kBF16;
}
} // namespace kami
