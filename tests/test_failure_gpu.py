"""Failure detection without a GPU fault: a bounded device wait that runs out
(an mbarrier nothing arrives at) returns an error status the host reads, and
the context stays usable for the next launch."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(cuda):
    L = _lib.load()
    code = ctypes.c_int(0)
    assert L.kami_device_status(ctypes.byref(code)) == 0 and code.value == 0
    assert L.kami_selftest_bounded_wait(50_000_000, None) == 0  # 50 ms
    torch.cuda.synchronize()
    st = L.kami_device_status(ctypes.byref(code))
    assert st == -6 and code.value == 4  # KAMI_ERR_TIMEOUT
    assert L.kami_device_status(ctypes.byref(code)) == 0 and code.value == 0  # cleared
    # the context still computes correctly
    A = torch.tensor(np.ones((2, 64, 64)), dtype=torch.float16, device="cuda")
    C = api.gemm_batched(A, A)
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(np.ones((2, 64, 64)), np.ones((2, 64, 64))))


def test_selftest_rejects_unbounded_request(cuda):
    assert _lib.load().kami_selftest_bounded_wait(60_000_000_000, None) == -1
