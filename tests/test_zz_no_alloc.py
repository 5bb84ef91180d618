"""The allocation-free grouped GEMM entry point (kami_gemm_grouped_noalloc).

It exists for callers that may not allocate device memory -- work issued
while a CUDA graph is captured, allocators that forbid cudaMalloc after
start-up, hosts that preallocate everything -- and keeps its problem
descriptors in a fixed device array owned by the library instead of a
cudaMalloc'd plan.  This file is collected last so that a failing run that
stops at the first failure has already run every other test; it must pass
alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest
import torch

from kami_b200 import _lib, api

pytestmark = pytest.mark.gpu

F16, F32 = 0, 3


def _shapes(count, seed):
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(8), np.log(128), (count, 3)))
    return np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64)


def _call_noalloc(plan, A, B, C):
    sh = plan.shapes
    M, N, K = (np.ascontiguousarray(sh[:, i], dtype=np.int32) for i in range(3))
    ao, bo, co = plan.offsets
    st = _lib.load().kami_gemm_grouped_noalloc(F16, F32, len(sh), M.ctypes.data, N.ctypes.data, K.ctypes.data,
                                               ao.ctypes.data, bo.ctypes.data, co.ctypes.data, A.data_ptr(),
                                               B.data_ptr(), C.data_ptr(), 1.0, 0.0, 1,
                                               torch.cuda.current_stream().cuda_stream)
    _lib.check(st)


def test_noalloc_matches_plan_entry_point_twice(cuda):
    shapes = _shapes(700, 11)
    plan = api.GroupedPlan(shapes, torch.float16)
    for call in range(2):  # two calls in a row: the shared array is rewritten each time
        rng = np.random.default_rng(100 + call)
        A = torch.tensor(rng.uniform(-1, 1, plan.sizes[0]), dtype=torch.float16, device="cuda")
        B = torch.tensor(rng.uniform(-1, 1, plan.sizes[1]), dtype=torch.float16, device="cuda")
        C_ref = torch.zeros(plan.sizes[2], dtype=torch.float32, device="cuda")
        C_na = torch.full((plan.sizes[2],), float("nan"), dtype=torch.float32, device="cuda")
        plan.run(A, B, C_ref)
        _call_noalloc(plan, A, B, C_na)
        torch.cuda.synchronize()
        # same kernel, same partitions, same schedule order per problem: identical
        # results are expected; the tolerance is the suite's FP32 bound
        assert torch.isfinite(C_na).all()
        assert torch.allclose(C_na, C_ref, rtol=0, atol=1e-5), call


def test_noalloc_rejects_too_many_problems(cuda):
    n = 8193
    M = np.full(n, 8, dtype=np.int32)
    off = np.zeros(n, dtype=np.int64)
    buf = torch.zeros(64, dtype=torch.float16, device="cuda")
    out = torch.zeros(64, dtype=torch.float32, device="cuda")
    st = _lib.load().kami_gemm_grouped_noalloc(F16, F32, n, M.ctypes.data, M.ctypes.data, M.ctypes.data,
                                               off.ctypes.data, off.ctypes.data, off.ctypes.data, buf.data_ptr(),
                                               buf.data_ptr(), out.data_ptr(), 1.0, 0.0, 1, None)
    assert st == -2
    assert b"KAMI_NOALLOC_MAX_PROBLEMS" in _lib.load().kami_last_error_string()
