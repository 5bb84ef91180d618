// cutlass_sm100.cu -- comparator only (not part of libkami_b200.so): the
// batched GEMM of the CUTLASS library built for sm_100a from its 5th-
// generation tensor-core collectives (TMA loads, tcgen05.mma, TMEM
// accumulators; warp-specialised persistent kernel, cluster 1 x 1 x 1, so
// every CTA loads its own tiles), on the same buffers and layouts as
// kami_gemm_batched:
// A batch x M x K row-major, B the reference's batch x N x K row-major
// operand (K x N column-major for CUTLASS), C batch x M x N row-major.
// The benchmark times it beside this library's kernels.
#include <cstdint>
#include <cstdio>

#include "cute/tensor.hpp"
#include "cutlass/cutlass.h"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/gemm/collective/collective_builder.hpp"
#include "cutlass/gemm/device/gemm_universal_adapter.h"
#include "cutlass/gemm/dispatch_policy.hpp"
#include "cutlass/gemm/kernel/gemm_universal.hpp"
#include "cutlass/util/packed_stride.hpp"

using namespace cute;

namespace {

template <class ElementAB, class ElementC, class TileShape>
struct Sm100Batched
{
    using LayoutA = cutlass::layout::RowMajor;
    using LayoutB = cutlass::layout::ColumnMajor;
    using LayoutC = cutlass::layout::RowMajor;
    static constexpr int kAlignAB = 16 / sizeof(ElementAB);
    static constexpr int kAlignC = 16 / sizeof(ElementC);
    using ClusterShape = Shape<_1, _1, _1>;
    using CollectiveEpilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, TileShape, ClusterShape,
        cutlass::epilogue::collective::EpilogueTileAuto, float, float, ElementC, LayoutC, kAlignC, ElementC, LayoutC,
        kAlignC, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;
    using CollectiveMainloop = typename cutlass::gemm::collective::CollectiveBuilder<
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementAB, LayoutA, kAlignAB, ElementAB, LayoutB, kAlignAB,
        float, TileShape, ClusterShape,
        cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(
            sizeof(typename CollectiveEpilogue::SharedStorage))>,
        cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;
    using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, CollectiveMainloop,
                                                        CollectiveEpilogue>;
    using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;

    static int run(int M, int N, int K, int L, const void *A, const void *B, void *C, void *ws, size_t ws_bytes,
                   size_t *ws_needed, cudaStream_t s)
    {
        using StrideA = typename Gemm::GemmKernel::StrideA;
        using StrideB = typename Gemm::GemmKernel::StrideB;
        using StrideC = typename Gemm::GemmKernel::StrideC;
        using StrideD = typename Gemm::GemmKernel::StrideD;
        auto sa = cutlass::make_cute_packed_stride(StrideA{}, make_shape(M, K, L));
        auto sb = cutlass::make_cute_packed_stride(StrideB{}, make_shape(N, K, L));
        auto sc = cutlass::make_cute_packed_stride(StrideC{}, make_shape(M, N, L));
        auto sd = cutlass::make_cute_packed_stride(StrideD{}, make_shape(M, N, L));
        typename Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,
                                      {M, N, K, L},
                                      {reinterpret_cast<const ElementAB *>(A), sa,
                                       reinterpret_cast<const ElementAB *>(B), sb},
                                      {{1.0f, 0.0f}, reinterpret_cast<const ElementC *>(C), sc,
                                       reinterpret_cast<ElementC *>(C), sd}};
        Gemm gemm;
        if (gemm.can_implement(args) != cutlass::Status::kSuccess)
            return -2;
        const size_t need = Gemm::get_workspace_size(args);
        if (ws_needed)
            *ws_needed = need;
        if (need > ws_bytes)
            return -4;
        if (gemm.initialize(args, ws, s) != cutlass::Status::kSuccess)
            return -7;
        if (gemm.run(s) != cutlass::Status::kSuccess)
            return -5;
        return cudaGetLastError() == cudaSuccess ? 0 : -5;
    }
};

} // namespace

// in_type 0 = FP16, 1 = BF16; out_type 3 = FP32, else the input type;
// tile 128 (128 x 128 x 64 CTA tile) or 64 (64 x 64 x 64).  Returns 0, or
// -2 (unsupported), -4 (workspace too small; *ws_needed tells), -5 / -7.
extern "C" int kami_cmp_cutlass_gemm_batched(int in_type, int out_type, int tile, int M, int N, int K,
                                             int64_t batch, const void *A, const void *B, void *C, void *ws,
                                             size_t ws_bytes, size_t *ws_needed, void *stream)
{
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int L = (int)batch;
    using T128 = Shape<_128, _128, _64>;
    using T64 = Shape<_64, _64, _64>;
    if (in_type == 0 && out_type == 3)
        return tile == 64 ? Sm100Batched<cutlass::half_t, float, T64>::run(M, N, K, L, A, B, C, ws, ws_bytes,
                                                                           ws_needed, s)
                          : Sm100Batched<cutlass::half_t, float, T128>::run(M, N, K, L, A, B, C, ws, ws_bytes,
                                                                            ws_needed, s);
    if (in_type == 0 && out_type == 0)
        return tile == 64 ? Sm100Batched<cutlass::half_t, cutlass::half_t, T64>::run(M, N, K, L, A, B, C, ws,
                                                                                     ws_bytes, ws_needed, s)
                          : Sm100Batched<cutlass::half_t, cutlass::half_t, T128>::run(M, N, K, L, A, B, C, ws,
                                                                                      ws_bytes, ws_needed, s);
    if (in_type == 1 && out_type == 1)
        return tile == 64 ? Sm100Batched<cutlass::bfloat16_t, cutlass::bfloat16_t, T64>::run(M, N, K, L, A, B, C, ws,
                                                                                             ws_bytes, ws_needed, s)
                          : Sm100Batched<cutlass::bfloat16_t, cutlass::bfloat16_t, T128>::run(
                                M, N, K, L, A, B, C, ws, ws_bytes, ws_needed, s);
    return -2;
}
