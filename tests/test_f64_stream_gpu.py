"""The persistent streamed FP64 kernel (chosen automatically for FP64
problems of 48 < M <= 64, 32 < N <= 64, 32 <= K <= 64 with few repeats, the
N x K B layout and at least two problems per SM) against the CPU oracle:
exact on integer inputs, odd shapes (columns past K and rows past M / N
arrive as zeros from the tensor copies), alpha/beta and repeats; and the
shapes and the K x N B layout that take the per-problem kernel."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api

pytestmark = pytest.mark.gpu


# the streamed kernel takes 48 < M <= 64, 32 < N <= 64, 32 <= K <= 64 (N x K B);
# the smaller shapes take the per-problem kernel
@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (64, 64, 58), (49, 33, 32), (57, 64, 42), (64, 40, 34), (50, 62, 64),
                                   (32, 32, 32), (40, 24, 18), (64, 8, 64), (1, 64, 2), (17, 33, 64), (16, 16, 10)])
@pytest.mark.parametrize("b_layout", ["ref_nk", "row_kn"])
def test_exact_integer_inputs(cuda, M, N, K, b_layout):
    if b_layout == "row_kn" and N % 2:
        pytest.skip("row_kn rows of odd length take the per-problem kernel")
    rng = np.random.default_rng(M * 100 + N + K)
    batch = 700
    A = rng.integers(-50, 51, (batch, M, K)).astype(np.float64)
    Bt = rng.integers(-50, 51, (batch, K, N)).astype(np.float64)
    B = np.ascontiguousarray(Bt.transpose(0, 2, 1)) if b_layout == "ref_nk" else Bt
    C = api.gemm_batched(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), b_layout=b_layout)
    assert np.array_equal(C.cpu().numpy(), np.matmul(A, Bt))


def test_alpha_beta_and_repeats(cuda):
    rng = np.random.default_rng(9)
    batch, n = 500, 64
    A = rng.integers(-8, 9, (batch, n, n)).astype(np.float64)
    B = rng.integers(-8, 9, (batch, n, n)).astype(np.float64)
    C0 = rng.integers(-8, 9, (batch, n, n)).astype(np.float64)
    dC = torch.tensor(C0, device="cuda")
    api.gemm_batched(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), dC, alpha=2.0, beta=-3.0,
                     num_iter=3)
    assert np.array_equal(dC.cpu().numpy(), 2.0 * 3 * oracle.gemm(A, B) - 3.0 * C0)


def test_random_reals_within_bound(cuda):
    rng = np.random.default_rng(10)
    batch, n = 1200, 64
    A = rng.uniform(-1, 1, (batch, n, n))
    B = rng.uniform(-1, 1, (batch, n, n))
    C = api.gemm_batched(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")).cpu().numpy()
    bound = (n + 2) * 2.0 ** -52 * np.matmul(np.abs(A), np.abs(B).transpose(0, 2, 1))
    assert np.all(np.abs(C - oracle.gemm(A, B)) <= bound)


def test_device_status_clean_after_runs(cuda):
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0
