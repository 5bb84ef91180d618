"""kami_gemm_batched_host: the batched GEMM on host buffers with the copies
pipelined against the product, through the C ABI, against the device-buffer
entry point on the same inputs (identical results: the same kernels run per
chunk) and the CPU oracle."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("batch", [1, 100, 592, 1000, 3001])
@pytest.mark.parametrize("dtype,n", [(torch.float16, 128), (torch.bfloat16, 64), (torch.float64, 32)])
def test_host_matches_device(cuda, batch, dtype, n):
    rng = np.random.default_rng(batch + n)
    A = torch.tensor(rng.integers(-2, 3, (batch, n, n)), dtype=dtype)
    B = torch.tensor(rng.integers(-2, 3, (batch, n, n)), dtype=dtype)
    odt = torch.float64 if dtype == torch.float64 else torch.float32
    Ap, Bp = A.pin_memory(), B.pin_memory()
    Cp = torch.full((batch, n, n), 7.0, dtype=odt).pin_memory()
    for _ in range(2):  # two calls in a row on the shared workspace
        api.gemm_batched_host(Ap, Bp, Cp, num_iter=2)
        torch.cuda.synchronize()
        ref = api.gemm_batched(A.cuda(), B.cuda(), num_iter=2).cpu()
        assert torch.equal(Cp, ref)
    sel = [0, batch // 2, batch - 1]
    assert np.array_equal(Cp[sel].double().numpy(), 2 * oracle.gemm(A[sel].double().numpy(), B[sel].double().numpy()))


def test_host_pageable_and_caller_workspace(cuda):
    """Pageable host buffers work (without overlap); a caller workspace of
    the reported size is used, a smaller one is rejected."""
    L = _lib.load()
    batch, n = 400, 64
    rng = np.random.default_rng(3)
    A = torch.tensor(rng.integers(-2, 3, (batch, n, n)), dtype=torch.float16)
    B = torch.tensor(rng.integers(-2, 3, (batch, n, n)), dtype=torch.float16)
    C = torch.zeros((batch, n, n), dtype=torch.float32)
    need = ctypes.c_size_t(0)
    assert L.kami_gemm_batched_host_workspace_size(_lib.F16, _lib.F32, n, n, n, batch, ctypes.byref(need)) == 0
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    assert L.kami_gemm_batched_host(_lib.F16, _lib.F32, 0, 0, n, n, n, batch, A.data_ptr(), B.data_ptr(),
                                    C.data_ptr(), 1, ws.data_ptr(), need.value, s.cuda_stream) == 0
    torch.cuda.synchronize()
    assert torch.equal(C, api.gemm_batched(A.cuda(), B.cuda()).cpu())
    assert L.kami_gemm_batched_host(_lib.F16, _lib.F32, 0, 0, n, n, n, batch, A.data_ptr(), B.data_ptr(),
                                    C.data_ptr(), 1, ws.data_ptr(), need.value - 256, s.cuda_stream) != 0
