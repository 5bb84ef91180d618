"""Uneven grouped GEMM (one persistent launch) against the CPU oracle, with
the static and the autotuned partition choice, FP16/BF16->FP32 and FP64, and
inside a captured CUDA graph."""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api

pytestmark = pytest.mark.gpu


def uneven_shapes(count, seed, lo=8, hi=128):
    # M, N, K each 8 * round(exp(U[ln 8, ln 128]) / 8), clamped to [8, 128]
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(lo), np.log(hi), (count, 3)))
    return np.clip(8 * np.round(x / 8), lo, hi).astype(np.int64)


def make_inputs(shapes, dtype, seed, integer=True):
    rng = np.random.default_rng(seed)
    As, Bs = [], []
    for (m, n, k) in shapes:
        if integer:
            As.append(rng.integers(-2, 3, (m, k)).astype(np.float64))
            Bs.append(rng.integers(-2, 3, (n, k)).astype(np.float64))
        else:
            As.append(rng.uniform(-1, 1, (m, k)))
            Bs.append(rng.uniform(-1, 1, (n, k)))
    A = torch.tensor(np.concatenate([a.ravel() for a in As]), dtype=dtype, device="cuda")
    B = torch.tensor(np.concatenate([b.ravel() for b in Bs]), dtype=dtype, device="cuda")
    return As, Bs, A, B


def check(plan, As, Bs, C, exact=True):
    Ch = C.double().cpu().numpy()
    co = plan.offsets[2]
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = oracle.gemm(As[i][None], Bs[i][None])[0]
        got = Ch[co[i]:co[i] + m * n].reshape(m, n)
        if exact:
            assert np.array_equal(got, ref), (i, m, n, k)
        else:
            assert np.max(np.abs(got - ref)) <= (k + 2) * 2.0 ** -52 * np.max(np.abs(As[i]) @ np.abs(Bs[i]).T)


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float64])
@pytest.mark.parametrize("autotune", [False, True])
def test_grouped_exact(cuda, dtype, autotune):
    shapes = uneven_shapes(600, 0)
    As, Bs, A, B = make_inputs(shapes, dtype, 1)
    plan = api.GroupedPlan(shapes, dtype, autotune=autotune)
    info = plan.info()
    assert info["problems"] == 600 and sum(info["partitions"]) == 600
    C = torch.empty(plan.sizes[2], dtype=plan.out_dtype, device="cuda")
    plan.run(A, B, C)
    torch.cuda.synchronize()
    check(plan, As, Bs, C)


def test_grouped_fp64_uniform(cuda):
    shapes = uneven_shapes(200, 5)
    As, Bs, A, B = make_inputs(shapes, torch.float64, 6, integer=False)
    plan = api.GroupedPlan(shapes, torch.float64)
    C = torch.empty(plan.sizes[2], dtype=torch.float64, device="cuda")
    plan.run(A, B, C)
    check(plan, As, Bs, C, exact=False)


def test_grouped_every_partition(cuda):
    # the same problems under every partition must give identical results
    shapes = np.array([[32, 32, 64], [64, 24, 128], [16, 64, 8], [8, 8, 8], [64, 64, 40]] * 20)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 2)
    plan = api.GroupedPlan(shapes, torch.float16, autotune=True)
    C = torch.empty(plan.sizes[2], dtype=torch.float32, device="cuda")
    plan.run(A, B, C, num_iter=3)
    Ch = C.double().cpu().numpy() / 3
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = oracle.gemm(As[i][None], Bs[i][None])[0]
        assert np.array_equal(Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n), ref)


def test_grouped_cuda_graph(cuda):
    shapes = uneven_shapes(300, 3)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 4)
    plan = api.GroupedPlan(shapes, torch.float16)
    C = torch.zeros(plan.sizes[2], dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.run(A, B, C, stream=s)  # warm up outside capture
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.run(A, B, C)
    As2, Bs2, A2, B2 = make_inputs(shapes, torch.float16, 9)
    A.copy_(A2)
    B.copy_(B2)
    C.zero_()
    g.replay()
    torch.cuda.synchronize()
    check(plan, As2, Bs2, C)


def test_grouped_alpha_beta_out_types(cuda):
    shapes = uneven_shapes(100, 7)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 8)
    plan = api.GroupedPlan(shapes, torch.float16, out_dtype=torch.float16)
    C = torch.full((plan.sizes[2],), 1.0, dtype=torch.float16, device="cuda")
    plan.run(A, B, C, alpha=2.0, beta=-1.0)
    Ch = C.double().cpu().numpy()
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = 2 * oracle.gemm(As[i][None], Bs[i][None])[0] - 1
        ref16 = ref.astype(np.float16).astype(np.float64)
        assert np.array_equal(Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n), ref16)


def test_grouped_rejects_bad_shapes(cuda):
    with pytest.raises(api.KamiError if hasattr(api, "KamiError") else Exception):
        api.GroupedPlan([[200, 8, 8]], torch.float16)
    with pytest.raises(Exception):
        api.GroupedPlan([[8, 8, 12]], torch.float16)
