// tc05_gemm.cu -- tcgen05 block GEMM (placeholder until the kernel lands).
#include "tc05_gemm.cuh"

namespace kami {

bool tc05_prefer(int, int, int, int, int, int, int) { return false; }

int tc05_plan(int, int, int, int, int, int, int, int64_t, int, int, LaunchInfo *)
{
    return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant not built");
}

int tc05_launch(const GemmArgs &, int, int, int, void *, size_t, cudaStream_t)
{
    return fail(KAMI_ERR_UNSUPPORTED, "tcgen05 variant not built");
}

} // namespace kami
