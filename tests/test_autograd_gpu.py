"""The differentiable batched GEMM (forward and hand-written backward on the
library's kernels): torch.autograd.gradcheck in FP64 (finite differences)
on 8x8x8, and BF16/FP16 gradients against torch.bmm's on 64x64x64."""
import pytest
import torch

from kami_b200.autograd import bmm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("partition", ["auto", "1d", "2d", "3d"])
def test_gradcheck_fp64(cuda, partition):
    torch.manual_seed(0)
    A = torch.randn(3, 8, 8, dtype=torch.float64, device="cuda", requires_grad=True)
    B = torch.randn(3, 8, 8, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: bmm(a, b, partition), (A, B), eps=1e-6, atol=1e-8, rtol=1e-6)


def test_gradcheck_fp64_rectangular(cuda):
    torch.manual_seed(1)
    A = torch.randn(2, 24, 16, dtype=torch.float64, device="cuda", requires_grad=True)
    B = torch.randn(2, 16, 40, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(bmm, (A, B), eps=1e-6, atol=1e-8, rtol=1e-6)


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_grads_match_torch_bmm(cuda, dtype):
    torch.manual_seed(2)
    A0 = (torch.rand(256, 64, 64, device="cuda") * 2 - 1).to(dtype)
    B0 = (torch.rand(256, 64, 64, device="cuda") * 2 - 1).to(dtype)
    G = (torch.rand(256, 64, 64, device="cuda") * 2 - 1).to(dtype)
    A, B = A0.clone().requires_grad_(), B0.clone().requires_grad_()
    C = bmm(A, B)
    C.backward(G)
    # reference in FP32 from the same 16-bit values
    Af, Bf, Gf = A0.float().requires_grad_(), B0.float().requires_grad_(), G.float()
    Cf = torch.bmm(Af, Bf)
    Cf.backward(Gf)
    assert C.dtype == dtype and A.grad.dtype == dtype
    tol = 2 * (2.0 ** -8 if dtype == torch.bfloat16 else 2.0 ** -11)
    for got, ref in [(C, Cf), (A.grad, Af.grad), (B.grad, Bf.grad)]:
        err = (got.float() - ref).abs().max() / ref.abs().max()
        assert err <= tol, (err, tol)
