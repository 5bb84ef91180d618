// kami_torch_ops.cpp -- the differentiable batched GEMM as a torch operator
// implemented in C++ (torch.ops.kami.bmm), over the C ABI of
// libkami_b200.so.
//
// A Python torch.autograd.Function spends tens of microseconds of host time
// per step (the Python apply, two ctypes calls with their argument checks,
// the autograd node); at 4096 x 64^3 the forward and the fused backward
// kernels take ~75 us together, so that host time decides the step.  Here
// the forward, the backward node and both launches are C++: torch's
// dispatcher calls kami_gemm_batched (forward, B as the K x N operand) and
// kami_gemm_backward_batched (dA = dC B^T and dB = A^T dC in one fused
// kernel for FP16 / BF16 64 / 128 shapes) on the operands' device and its
// current stream.  Semantics are torch.bmm's: A [batch, M, K], B [batch, K,
// N], C in the input dtype (FP32 accumulation for FP16 / BF16).
#include <ATen/ATen.h>
#include <ATen/core/dispatch/Dispatcher.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/autograd.h>
#include <torch/library.h>

#include "kami.h"

namespace {

using at::Tensor;

kami_dtype_t kami_type(const Tensor &t)
{
    switch (t.scalar_type())
    {
    case at::kHalf: return KAMI_F16;
    case at::kBFloat16: return KAMI_BF16;
    case at::kDouble: return KAMI_F64;
    default: TORCH_CHECK(false, "kami::bmm takes float16, bfloat16 or float64 tensors, got ", t.scalar_type());
    }
}

void check_operands(const Tensor &A, const Tensor &B)
{
    TORCH_CHECK(A.dim() == 3 && B.dim() == 3, "kami::bmm: A and B must be 3-D ([batch, M, K], [batch, K, N])");
    TORCH_CHECK(A.scalar_type() == B.scalar_type(), "kami::bmm: A and B must have the same dtype");
    TORCH_CHECK(A.is_cuda() && B.is_cuda(), "kami::bmm: A and B must be CUDA tensors");
    TORCH_CHECK(A.device() == B.device(), "kami::bmm: A and B are on different devices");
    TORCH_CHECK(A.size(0) == B.size(0) && A.size(2) == B.size(1), "kami::bmm: shapes do not match C = A @ B");
}

Tensor bmm_cuda(const Tensor &A_, const Tensor &B_)
{
    check_operands(A_, B_);
    const c10::cuda::CUDAGuard guard(A_.device());
    const Tensor A = A_.contiguous(), B = B_.contiguous();
    const int64_t batch = A.size(0), M = A.size(1), K = A.size(2), N = B.size(2);
    Tensor C = at::empty({batch, M, N}, A.options());
    if (batch == 0 || M == 0 || N == 0)
        return C;
    const kami_dtype_t dt = kami_type(A);
    void *stream = c10::cuda::getCurrentCUDAStream(A.device().index()).stream();
    const int st = kami_gemm_batched(dt, dt, KAMI_PARTITION_AUTO, KAMI_VARIANT_AUTO, (int)M, (int)N, (int)K, 0, 0,
                                     batch, A.data_ptr(), K, M * K, KAMI_A_ROW_MK, B.data_ptr(), N, K * N,
                                     KAMI_B_ROW_KN, C.data_ptr(), N, M * N, 1.0, 0.0, 1, nullptr, 0, stream);
    TORCH_CHECK(st == KAMI_OK, "kami_gemm_batched: ", kami_last_error_string());
    return C;
}

std::tuple<Tensor, Tensor> bmm_backward_cuda(const Tensor &A_, const Tensor &B_, const Tensor &dC_, bool need_dA,
                                             bool need_dB)
{
    check_operands(A_, B_);
    const c10::cuda::CUDAGuard guard(A_.device());
    const Tensor A = A_.contiguous(), B = B_.contiguous(), dC = dC_.contiguous().to(A.scalar_type());
    const int64_t batch = A.size(0), M = A.size(1), K = A.size(2), N = B.size(2);
    TORCH_CHECK(dC.size(0) == batch && dC.size(1) == M && dC.size(2) == N, "kami::bmm_backward: dC shape");
    Tensor dA = need_dA ? at::empty({batch, M, K}, A.options()) : Tensor();
    Tensor dB = need_dB ? at::empty({batch, K, N}, A.options()) : Tensor();
    if (batch == 0 || (!need_dA && !need_dB))
        return {dA, dB};
    const kami_dtype_t dt = kami_type(A);
    void *stream = c10::cuda::getCurrentCUDAStream(A.device().index()).stream();
    const int st = kami_gemm_backward_batched(dt, dt, (int)M, (int)N, (int)K, batch, A.data_ptr(), B.data_ptr(),
                                              dC.data_ptr(), need_dA ? dA.data_ptr() : nullptr,
                                              need_dB ? dB.data_ptr() : nullptr, stream);
    TORCH_CHECK(st == KAMI_OK, "kami_gemm_backward_batched: ", kami_last_error_string());
    return {dA, dB};
}

class KamiBmmFunction : public torch::autograd::Function<KamiBmmFunction>
{
  public:
    static Tensor forward(torch::autograd::AutogradContext *ctx, const Tensor &A, const Tensor &B)
    {
        ctx->save_for_backward({A, B});
        at::AutoDispatchBelowADInplaceOrView below;
        static auto op = c10::Dispatcher::singleton().findSchemaOrThrow("kami::bmm", "").typed<Tensor(const Tensor &,
                                                                                                    const Tensor &)>();
        return op.call(A, B);
    }

    static torch::autograd::tensor_list backward(torch::autograd::AutogradContext *ctx,
                                                 torch::autograd::tensor_list grads)
    {
        const auto saved = ctx->get_saved_variables();
        static auto op = c10::Dispatcher::singleton()
                             .findSchemaOrThrow("kami::bmm_backward", "")
                             .typed<std::tuple<Tensor, Tensor>(const Tensor &, const Tensor &, const Tensor &, bool,
                                                               bool)>();
        auto [dA, dB] = op.call(saved[0], saved[1], grads[0], ctx->needs_input_grad(0), ctx->needs_input_grad(1));
        return {dA, dB};
    }
};

Tensor bmm_autograd(const Tensor &A, const Tensor &B) { return KamiBmmFunction::apply(A, B); }

} // namespace

TORCH_LIBRARY(kami, m)
{
    m.def("bmm(Tensor a, Tensor b) -> Tensor");
    m.def("bmm_backward(Tensor a, Tensor b, Tensor grad, bool need_a, bool need_b) -> (Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(kami, CUDA, m)
{
    m.impl("bmm", bmm_cuda);
    m.impl("bmm_backward", bmm_backward_cuda);
}

TORCH_LIBRARY_IMPL(kami, Autograd, m) { m.impl("bmm", bmm_autograd); }
