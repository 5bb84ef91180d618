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


def _ints(shape, seed):
    import numpy as np
    return np.random.default_rng(seed).integers(-2, 3, shape).astype(np.float64)


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (128, 64, 64), (64, 128, 64), (64, 64, 128), (128, 128, 64),
                                   (128, 64, 128), (64, 128, 128), (128, 128, 128)])
@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_fused_backward_exact(cuda, M, N, K, dtype):
    """kami_gemm_backward_batched on the fused kernel: both gradients exact
    on integer-valued inputs against the oracle (FP32 out)."""
    import numpy as np
    import oracle
    from kami_b200 import api
    batch = 200
    A, B, G = _ints((batch, M, K), M), _ints((batch, K, N), N + 1), _ints((batch, M, N), K + 2)
    t = lambda x: torch.tensor(x, dtype=dtype, device="cuda")
    dA, dB = api.gemm_backward(t(A), t(B), t(G), out_dtype=torch.float32)
    # dA = G B^T: B^T is the oracle's N x K ("ref_nk") operand when B is K x N
    assert np.array_equal(dA.double().cpu().numpy(), oracle.gemm(G, B))
    # dB = A^T G
    assert np.array_equal(dB.double().cpu().numpy(), oracle.gemm(np.ascontiguousarray(A.transpose(0, 2, 1)),
                                                                 np.ascontiguousarray(G.transpose(0, 2, 1))))


@pytest.mark.parametrize("need", [(True, False), (False, True)])
@pytest.mark.parametrize("out_dtype", [torch.bfloat16, torch.float16])
def test_fused_backward_one_gradient_and_out_types(cuda, need, out_dtype):
    import numpy as np
    import oracle
    from kami_b200 import api
    A, B, G = _ints((64, 128, 64), 3), _ints((64, 64, 128), 4), _ints((64, 128, 128), 5)
    t = lambda x: torch.tensor(x, dtype=torch.bfloat16, device="cuda")
    dA, dB = api.gemm_backward(t(A), t(B), t(G), need_dA=need[0], need_dB=need[1], out_dtype=out_dtype)
    assert (dA is None) != need[0] and (dB is None) != need[1]
    rnd = lambda x: torch.tensor(x, dtype=torch.float32).to(out_dtype).double().numpy()
    if need[0]:
        assert np.array_equal(dA.double().cpu().numpy(), rnd(oracle.gemm(G, B)))
    else:
        ref = oracle.gemm(np.ascontiguousarray(A.transpose(0, 2, 1)), np.ascontiguousarray(G.transpose(0, 2, 1)))
        assert np.array_equal(dB.double().cpu().numpy(), rnd(ref))


@pytest.mark.parametrize("M,N,K,dtype", [(48, 80, 32, torch.float16), (64, 64, 64, torch.float64),
                                         (100, 64, 64, torch.bfloat16), (16, 8, 24, torch.float64)])
def test_backward_two_product_path(cuda, M, N, K, dtype):
    """Requests outside the fused kernel (other sizes, FP64) run as two
    forward products and give the same gradients."""
    import numpy as np
    import oracle
    from kami_b200 import api
    batch = 50
    A, B, G = _ints((batch, M, K), 6), _ints((batch, K, N), 7), _ints((batch, M, N), 8)
    t = lambda x: torch.tensor(x, dtype=dtype, device="cuda")
    dA, dB = api.gemm_backward(t(A), t(B), t(G), out_dtype=torch.float64 if dtype == torch.float64 else torch.float32)
    assert np.array_equal(dA.double().cpu().numpy(), oracle.gemm(G, B))
    assert np.array_equal(dB.double().cpu().numpy(), oracle.gemm(np.ascontiguousarray(A.transpose(0, 2, 1)),
                                                                 np.ascontiguousarray(G.transpose(0, 2, 1))))


def test_grads_match_torch_bmm_rectangular_fused(cuda):
    torch.manual_seed(3)
    A0 = (torch.rand(64, 128, 64, device="cuda") * 2 - 1).bfloat16()
    B0 = (torch.rand(64, 64, 128, device="cuda") * 2 - 1).bfloat16()
    G = (torch.rand(64, 128, 128, device="cuda") * 2 - 1).bfloat16()
    A, B = A0.clone().requires_grad_(), B0.clone().requires_grad_()
    bmm(A, B).backward(G)
    Af, Bf = A0.float().requires_grad_(), B0.float().requires_grad_()
    torch.bmm(Af, Bf).backward(G.float())
    for got, ref in [(A.grad, Af.grad), (B.grad, Bf.grad)]:
        assert ((got.float() - ref).abs().max() / ref.abs().max()) <= 2 * 2.0 ** -8


def test_default_path_is_the_cpp_operator(cuda):
    """With the library's kernel choice the step runs through the C++
    operator torch.ops.kami.bmm (its backward node is the C++ function), and
    its gradients are the Python function's."""
    from kami_b200 import autograd
    assert autograd.ops_available()
    torch.manual_seed(4)
    A0 = (torch.rand(64, 64, 64, device="cuda") * 2 - 1).bfloat16()
    B0 = (torch.rand(64, 64, 64, device="cuda") * 2 - 1).bfloat16()
    G = (torch.rand(64, 64, 64, device="cuda") * 2 - 1).bfloat16()
    A, B = A0.clone().requires_grad_(), B0.clone().requires_grad_()
    C = bmm(A, B)
    assert "KamiBmmFunction" in C.grad_fn.name()
    C.backward(G)
    A2, B2 = A0.clone().requires_grad_(), B0.clone().requires_grad_()
    C2 = autograd.KamiBmm.apply(A2, B2, "auto", "auto")
    C2.backward(G)
    assert torch.equal(C, C2) and torch.equal(A.grad, A2.grad) and torch.equal(B.grad, B2.grad)


@pytest.mark.parametrize("batch", [2, 7, 4099])
@pytest.mark.parametrize("need", [(True, True), (True, False), (False, True)])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.bfloat16])
def test_fused_backward_pairs_exact(cuda, batch, need, out_dtype):
    """64^3 problems run two per CTA in the fused backward (stacked 128-row
    tiles, each gradient on a 128 x 128 accumulator's diagonal): odd batches
    (a last CTA with one problem), either gradient alone; exact on integers."""
    import numpy as np
    import oracle
    from kami_b200 import api
    A, B, G = _ints((batch, 64, 64), 40 + batch), _ints((batch, 64, 64), 41), _ints((batch, 64, 64), 42)
    t = lambda x: torch.tensor(x, dtype=torch.bfloat16, device="cuda")
    dA, dB = api.gemm_backward(t(A), t(B), t(G), need_dA=need[0], need_dB=need[1], out_dtype=out_dtype)
    rnd = lambda x: torch.tensor(x, dtype=torch.float32).to(out_dtype).double().numpy()
    if need[0]:
        assert np.array_equal(dA.double().cpu().numpy(), rnd(oracle.gemm(G, B)))
    if need[1]:
        ref = oracle.gemm(np.ascontiguousarray(A.transpose(0, 2, 1)), np.ascontiguousarray(G.transpose(0, 2, 1)))
        assert np.array_equal(dB.double().cpu().numpy(), rnd(ref))
