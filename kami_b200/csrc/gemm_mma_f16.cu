// gemm_mma_f16.cu -- compiled instances of the mma.sync block GEMM for
// binary16 inputs with FP32 accumulation (see mma_engine.cuh).
#include "mma_engine.cuh"
#include "mma_table_h16.inc"

namespace kami {
using TrF16 = TrH16<false>;
static const MmaInstance kF16[] = {
#define X(BM, BN, BK, P, PART) KAMI_MMA_INSTANCE(TrF16, KAMI_F16, BM, BN, BK, P, PART),
    KAMI_H16_TABLE(X)
#undef X
};
const MmaInstance *mma_instances_f16(int *count)
{
    *count = (int)(sizeof(kF16) / sizeof(kF16[0]));
    return kF16;
}
} // namespace kami
