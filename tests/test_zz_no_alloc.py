"""The allocation-free grouped GEMM entry point (kami_gemm_grouped_noalloc).

Some callers cannot call cudaMalloc: a host whose device memory is carved up
once at start-up by its own allocator (a serving process, a real-time or
embedded controller) and that treats any later allocation as a fault, or a
plug-in that runs inside such a host.  A grouped plan keeps its problem
descriptors in cudaMalloc'd memory, so those callers cannot create one; this
entry point keeps them in a fixed device array owned by the library.

Every call is checked against the CPU oracle (exact on integer inputs) and
against the plan-based entry point (kami_gemm_grouped_plan_create + _run) on
the same problems, for FP16, BF16 and FP64 inputs, with single-warp problems
(M, N <= 32) in the mix and more problems than the kernel keeps CTAs.  The
second call of each pair has other shapes, so it also shows that what the
first call left in the shared array does not leak into the second.

This file is collected last so that a failing run that stops at the first
failure has already run every other test; it must pass alone in a fresh
process and after the rest of the suite.
"""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api

pytestmark = pytest.mark.gpu

_DT = {torch.float16: _lib.F16, torch.bfloat16: _lib.BF16, torch.float64: _lib.F64, torch.float32: _lib.F32}


def _shapes(count, seed):
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(8), np.log(128), (count, 3)))
    return np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64)


def _call_noalloc(plan, A, B, C):
    sh = plan.shapes
    M, N, K = (np.ascontiguousarray(sh[:, i], dtype=np.int32) for i in range(3))
    ao, bo, co = plan.offsets
    st = _lib.load().kami_gemm_grouped_noalloc(_DT[plan.dtype], _DT[plan.out_dtype], len(sh), M.ctypes.data,
                                               N.ctypes.data, K.ctypes.data, ao.ctypes.data, bo.ctypes.data,
                                               co.ctypes.data, A.data_ptr(), B.data_ptr(), C.data_ptr(), 1.0, 0.0, 1,
                                               torch.cuda.current_stream().cuda_stream)
    _lib.check(st)


def _oracle(plan, A, B):
    """C of every problem from the oracle, batched by shape."""
    ao, bo, co = plan.offsets
    out = np.zeros(plan.sizes[2])
    keys = plan.shapes @ np.array([1 << 20, 1 << 10, 1])
    for key in np.unique(keys):
        idx = np.nonzero(keys == key)[0]
        m, n, k = (int(v) for v in plan.shapes[idx[0]])
        As = np.stack([A[ao[i]:ao[i] + m * k].reshape(m, k) for i in idx])
        Bs = np.stack([B[bo[i]:bo[i] + n * k].reshape(n, k) for i in idx])
        Cs = oracle.gemm(As, Bs)
        for j, i in enumerate(idx):
            out[co[i]:co[i] + m * n] = Cs[j].ravel()
    return out


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float64])
def test_noalloc_matches_oracle_and_plan_twice(cuda, dtype):
    # first call: the largest request the array holds; second: other shapes
    for call, (count, seed) in enumerate([(8192, 11), (700, 12)]):
        shapes = _shapes(count, seed)
        assert (np.minimum(shapes[:, 0], shapes[:, 1]) <= 32).any()  # single-warp problems present
        plan = api.GroupedPlan(shapes, dtype)
        rng = np.random.default_rng(100 + call)
        A = rng.integers(-2, 3, plan.sizes[0]).astype(np.float64)
        B = rng.integers(-2, 3, plan.sizes[1]).astype(np.float64)
        dA = torch.tensor(A, dtype=dtype, device="cuda")
        dB = torch.tensor(B, dtype=dtype, device="cuda")
        C_plan = torch.full((plan.sizes[2],), float("nan"), dtype=plan.out_dtype, device="cuda")
        C_na = torch.full((plan.sizes[2],), float("nan"), dtype=plan.out_dtype, device="cuda")
        plan.run(dA, dB, C_plan)
        _call_noalloc(plan, dA, dB, C_na)
        torch.cuda.synchronize()
        got = C_na.double().cpu().numpy()
        # integer inputs: every product sum is exact in FP32 / FP64
        assert np.array_equal(got, _oracle(plan, A, B)), call
        assert np.array_equal(got, C_plan.double().cpu().numpy()), call


def test_noalloc_uniform_within_bound_of_plan(cuda):
    """uniform[-1, 1] FP16 inputs: the no-alloc launch (mma.sync warp grids)
    and the plan's default kernel (tcgen05) each stay within the FP32
    accumulation bound (K + 2) 2^-23 |A||B| of the oracle, so they agree
    within twice that bound."""
    shapes = _shapes(3000, 13)
    plan = api.GroupedPlan(shapes, torch.float16)
    rng = np.random.default_rng(14)
    A = rng.uniform(-1, 1, plan.sizes[0]).astype(np.float16).astype(np.float64)
    B = rng.uniform(-1, 1, plan.sizes[1]).astype(np.float16).astype(np.float64)
    dA = torch.tensor(A, dtype=torch.float16, device="cuda")
    dB = torch.tensor(B, dtype=torch.float16, device="cuda")
    C_plan = torch.empty(plan.sizes[2], dtype=torch.float32, device="cuda")
    C_na = torch.empty(plan.sizes[2], dtype=torch.float32, device="cuda")
    for _ in range(2):
        plan.run(dA, dB, C_plan)
        _call_noalloc(plan, dA, dB, C_na)
    ref = _oracle(plan, A, B)
    absref = _oracle(plan, np.abs(A), np.abs(B))
    kk = np.zeros(plan.sizes[2])
    for i, (m, n, k) in enumerate(plan.shapes):
        kk[plan.offsets[2][i]:plan.offsets[2][i] + m * n] = k
    bound = (kk + 2) * 2.0 ** -23 * absref
    got_na, got_plan = C_na.double().cpu().numpy(), C_plan.double().cpu().numpy()
    assert np.all(np.abs(got_na - ref) <= bound)
    assert np.all(np.abs(got_na - got_plan) <= 2 * bound)


def test_noalloc_rejects_too_many_problems(cuda):
    n = 8193
    M = np.full(n, 8, dtype=np.int32)
    off = np.zeros(n, dtype=np.int64)
    buf = torch.zeros(64, dtype=torch.float16, device="cuda")
    out = torch.zeros(64, dtype=torch.float32, device="cuda")
    st = _lib.load().kami_gemm_grouped_noalloc(_lib.F16, _lib.F32, n, M.ctypes.data, M.ctypes.data, M.ctypes.data,
                                               off.ctypes.data, off.ctypes.data, off.ctypes.data, buf.data_ptr(),
                                               buf.data_ptr(), out.data_ptr(), 1.0, 0.0, 1, None)
    assert st == -2
    assert b"KAMI_NOALLOC_MAX_PROBLEMS" in _lib.load().kami_last_error_string()
