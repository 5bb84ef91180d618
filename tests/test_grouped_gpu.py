"""Uneven grouped GEMM (one persistent launch) against the CPU oracle, with
the static and the autotuned partition choice, all three kernels (mma.sync
warp grids, tcgen05 for FP16/BF16, staged DMMA for FP64), FP16/BF16->FP32
and FP64, and inside a captured CUDA graph."""
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
    assert info["problems"] == 600
    default = "staged" if dtype == torch.float64 else "tcgen05"  # the uneven 8..128 mix
    assert info["kernel"] in ((default,) if not autotune else (default, "mma_sync"))
    if info["kernel"] == "mma_sync":
        assert sum(info["partitions"]) == 600
    elif info["kernel"] == "tcgen05":
        assert info["tcgen05_m64"] + info["tcgen05_m128"] == 600
    C = torch.empty(plan.sizes[2], dtype=plan.out_dtype, device="cuda")
    plan.run(A, B, C)
    torch.cuda.synchronize()
    check(plan, As, Bs, C)


@pytest.mark.parametrize("kernel", ["mma_sync", "staged"])
def test_grouped_fp64_uniform(cuda, kernel):
    shapes = uneven_shapes(200, 5)
    As, Bs, A, B = make_inputs(shapes, torch.float64, 6, integer=False)
    plan = api.GroupedPlan(shapes, torch.float64, kernel=kernel)
    assert plan.info()["kernel"] == kernel
    C = torch.empty(plan.sizes[2], dtype=torch.float64, device="cuda")
    plan.run(A, B, C)
    check(plan, As, Bs, C, exact=False)


def test_grouped_fp64_default_kernel_by_mix(cuda):
    """FP64 plans default to the staged kernel, and to the warp-grid kernel
    when problems of at most 32 x 32 carry most of the bytes."""
    assert api.GroupedPlan(uneven_shapes(300, 1), torch.float64).info()["kernel"] == "staged"
    assert api.GroupedPlan(np.full((300, 3), 32), torch.float64).info()["kernel"] == "mma_sync"
    assert api.GroupedPlan(np.full((300, 3), 32), torch.float64, kernel="staged").info()["kernel"] == "staged"


@pytest.mark.parametrize("num_iter", [1, 3])
def test_grouped_staged_fp64_edges(cuda, num_iter):
    """The staged DMMA kernel at the edges of its tiling: K of one partial
    k-step (2, 6), K across chunks with a partial last step (34, 98, 128),
    M and N not multiples of 16 (odd N too), a whole 128 x 128 C (five
    sub-tiles on some warps), single rows and columns; alpha / beta."""
    shapes = np.array([[8, 8, 2], [16, 16, 6], [17, 33, 34], [128, 128, 128], [1, 9, 98], [100, 1, 64],
                       [128, 120, 40], [64, 64, 32], [3, 127, 126], [48, 80, 96]] * 9)
    As, Bs, A, B = make_inputs(shapes, torch.float64, 17)
    plan = api.GroupedPlan(shapes, torch.float64, kernel="staged")
    C0 = np.random.default_rng(3).integers(-3, 4, plan.sizes[2]).astype(np.float64)
    C = torch.tensor(C0, device="cuda")
    plan.run(A, B, C, alpha=2.0, beta=-1.0, num_iter=num_iter)
    Ch = C.cpu().numpy()
    co = plan.offsets[2]
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = 2.0 * num_iter * oracle.gemm(As[i][None], Bs[i][None])[0] - C0[co[i]:co[i] + m * n].reshape(m, n)
        assert np.array_equal(Ch[co[i]:co[i] + m * n].reshape(m, n), ref), (i, m, n, k)


def test_grouped_staged_fp64_many_problems(cuda):
    """More problems per CTA than the staged kernel caches in shared memory."""
    rng = np.random.default_rng(18)
    count = 50000
    shapes = np.stack([rng.choice([8, 16, 24], count), rng.choice([8, 16], count), rng.choice([2, 8, 16], count)], 1)
    As, Bs, A, B = make_inputs(shapes, torch.float64, 19)
    plan = api.GroupedPlan(shapes, torch.float64, kernel="staged")
    assert plan.info()["problems"] // plan.info()["ctas"] > 256
    C = torch.empty(plan.sizes[2], dtype=torch.float64, device="cuda")
    plan.run(A, B, C)
    Ch = C.cpu().numpy()
    co = plan.offsets[2]
    for i in list(range(0, count, 499)) + [count - 1]:
        m, n, k = plan.shapes[i]
        assert np.array_equal(Ch[co[i]:co[i] + m * n].reshape(m, n), oracle.gemm(As[i][None], Bs[i][None])[0]), i


def test_grouped_every_partition(cuda):
    # the same problems under every partition must give identical results
    shapes = np.array([[32, 32, 64], [64, 24, 128], [16, 64, 8], [8, 8, 8], [64, 64, 40]] * 20)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 2)
    plan = api.GroupedPlan(shapes, torch.float16, autotune=True, kernel="mma_sync")
    assert plan.info()["kernel"] == "mma_sync"
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


@pytest.mark.parametrize("kernel", ["mma_sync", "tcgen05"])
@pytest.mark.parametrize("out_dtype", [torch.float16, torch.bfloat16, torch.float32])
def test_grouped_alpha_beta_out_types(cuda, kernel, out_dtype):
    shapes = uneven_shapes(100, 7)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 8)
    plan = api.GroupedPlan(shapes, torch.float16, out_dtype=out_dtype, kernel=kernel)
    assert plan.info()["kernel"] == kernel
    C = torch.full((plan.sizes[2],), 1.0, dtype=out_dtype, device="cuda")
    plan.run(A, B, C, alpha=2.0, beta=-1.0)
    Ch = C.double().cpu().numpy()
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = 2 * oracle.gemm(As[i][None], Bs[i][None])[0] - 1
        # exact integers in FP32; one rounding to the output type
        ref = torch.tensor(ref, dtype=torch.float32).to(out_dtype).double().numpy()
        assert np.array_equal(Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n), ref)


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("num_iter", [1, 3])
def test_grouped_tcgen05_edge_shapes(cuda, dtype, num_iter):
    """The tcgen05 kernel at the edges of its tiling: K of one partial k-step
    (8), K across two chunks with a partial last step (72, 120), M at the
    64 / 128 MMA boundary (64, 65), N not a multiple of 16, single rows."""
    shapes = np.array([[8, 8, 8], [64, 16, 72], [65, 24, 120], [128, 128, 128], [1, 8, 8], [17, 40, 64],
                       [64, 64, 64], [100, 8, 16], [8, 128, 24], [127, 121, 112]] * 7)
    As, Bs, A, B = make_inputs(shapes, dtype, 11)
    plan = api.GroupedPlan(shapes, dtype, kernel="tcgen05")
    info = plan.info()
    assert info["kernel"] == "tcgen05" and info["tcgen05_m64"] + info["tcgen05_m128"] == len(shapes)
    C = torch.full((plan.sizes[2],), -5.0, dtype=torch.float32, device="cuda")
    plan.run(A, B, C, num_iter=num_iter)
    torch.cuda.synchronize()
    Ch = C.double().cpu().numpy() / num_iter
    for i, (m, n, k) in enumerate(plan.shapes):
        ref = oracle.gemm(As[i][None], Bs[i][None])[0]
        assert np.array_equal(Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n), ref), (i, m, n, k)


def test_grouped_tcgen05_few_problems_and_offsets(cuda):
    """Fewer problems than SMs, and problems at caller offsets with gaps
    between them (the gaps must stay untouched)."""
    shapes = np.array([[40, 56, 32], [128, 8, 64], [8, 96, 104]])
    As, Bs, _, _ = make_inputs(shapes, torch.float16, 12)
    ao = np.array([0, 40 * 32 + 64, 40 * 32 + 64 + 128 * 64 + 8], dtype=np.int64)
    bo = np.array([16, 16 + 56 * 32 + 8, 16 + 56 * 32 + 8 + 8 * 64 + 32], dtype=np.int64)
    co = np.array([4, 4 + 40 * 56 + 13, 4 + 40 * 56 + 13 + 128 * 8 + 100], dtype=np.int64)
    A = torch.zeros(int(ao[-1]) + 8 * 104, dtype=torch.float16, device="cuda")
    B = torch.zeros(int(bo[-1]) + 96 * 104, dtype=torch.float16, device="cuda")
    for i, (m, n, k) in enumerate(shapes):
        A[ao[i]:ao[i] + m * k] = torch.tensor(As[i].ravel(), dtype=torch.float16)
        B[bo[i]:bo[i] + n * k] = torch.tensor(Bs[i].ravel(), dtype=torch.float16)
    C = torch.full((int(co[-1]) + 8 * 96 + 16,), 7.0, dtype=torch.float32, device="cuda")
    plan = api.GroupedPlan(shapes, torch.float16, offsets=(ao, bo, co), kernel="tcgen05")
    plan.run(A, B, C)
    Ch = C.double().cpu().numpy()
    mask = np.ones(Ch.size, bool)
    for i, (m, n, k) in enumerate(shapes):
        ref = oracle.gemm(As[i][None], Bs[i][None])[0]
        assert np.array_equal(Ch[co[i]:co[i] + m * n].reshape(m, n), ref)
        mask[co[i]:co[i] + m * n] = False
    assert np.all(Ch[mask] == 7.0)


def test_grouped_tcgen05_more_problems_than_cached(cuda):
    """More problems per CTA than the kernel's shared-memory descriptor cache
    holds (the rest are read from global memory)."""
    rng = np.random.default_rng(15)
    count = 90000
    shapes = np.stack([rng.choice([8, 16, 24], count), rng.choice([8, 16], count), rng.choice([8, 16], count)], 1)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 16)
    plan = api.GroupedPlan(shapes, torch.float16, kernel="tcgen05")
    assert plan.info()["problems"] // plan.info()["ctas"] > 224  # the cache holds at most 224
    C = torch.empty(plan.sizes[2], dtype=torch.float32, device="cuda")
    plan.run(A, B, C)
    Ch = C.double().cpu().numpy()
    co = plan.offsets[2]
    for i in list(range(0, count, 997)) + [count - 1]:
        m, n, k = plan.shapes[i]
        ref = oracle.gemm(As[i][None], Bs[i][None])[0]
        assert np.array_equal(Ch[co[i]:co[i] + m * n].reshape(m, n), ref), i


def test_grouped_kernels_agree_on_reals(cuda):
    """mma.sync and tcgen05 plans of the same uniform[-1, 1] problems agree
    within the FP32-accumulation bound of each against the oracle."""
    shapes = uneven_shapes(400, 13)
    As, Bs, A, B = make_inputs(shapes, torch.float16, 14, integer=False)
    A64 = [torch.tensor(a, dtype=torch.float16).double().numpy() for a in As]
    B64 = [torch.tensor(b, dtype=torch.float16).double().numpy() for b in Bs]
    for kernel in ("mma_sync", "tcgen05"):
        plan = api.GroupedPlan(shapes, torch.float16, kernel=kernel)
        C = torch.empty(plan.sizes[2], dtype=torch.float32, device="cuda")
        plan.run(A, B, C)
        Ch = C.double().cpu().numpy()
        for i, (m, n, k) in enumerate(plan.shapes):
            ref = A64[i] @ B64[i].T
            bound = (k + 2) * 2.0 ** -23 * (np.abs(A64[i]) @ np.abs(B64[i]).T) + 1e-30
            got = Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n)
            assert np.all(np.abs(got - ref) <= bound), (kernel, i)


def test_grouped_status_clean(cuda):
    import ctypes
    from kami_b200 import _lib
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0


def test_grouped_rejects_bad_shapes(cuda):
    with pytest.raises(api.KamiError if hasattr(api, "KamiError") else Exception):
        api.GroupedPlan([[200, 8, 8]], torch.float16)
    with pytest.raises(Exception):
        api.GroupedPlan([[8, 8, 12]], torch.float16)
    with pytest.raises(Exception):
        api.GroupedPlan([[8, 8, 8]], torch.float64, kernel="tcgen05")
    with pytest.raises(Exception):
        api.GroupedPlan([[8, 8, 8]], torch.float16, kernel="staged")


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("num_iter", [1, 2])
def test_grouped_tcgen05_packed_items(cuda, dtype, num_iter):
    """Small problems packed several to a work item (rows stacked in one A
    tile, 16-column groups of B, C on the accumulator's diagonal) give the
    oracle's results, as do the same problems unpacked: M, N up to 64 with
    odd sizes, K that differ inside an item (zero-filled), a single row,
    M = 64 and M = 128 items, and problems too large to pack between them."""
    rng = np.random.default_rng(30 + num_iter)
    shapes = np.stack([rng.choice([1, 8, 16, 17, 24, 33, 40, 64], 500), rng.choice([8, 16, 24, 40, 56, 64], 500),
                       rng.choice([8, 16, 24, 64, 72, 120, 128], 500)], 1)
    shapes[::37] = [128, 96, 64]
    As, Bs, A, B = make_inputs(shapes, dtype, 31)
    for pack in (True, False):
        plan = api.GroupedPlan(shapes, dtype, kernel="tcgen05", pack=pack)
        C = torch.full((plan.sizes[2],), float("nan"), dtype=torch.float32, device="cuda")
        plan.run(A, B, C, num_iter=num_iter)
        torch.cuda.synchronize()
        Ch = C.double().cpu().numpy() / num_iter
        for i, (m, n, k) in enumerate(plan.shapes):
            ref = oracle.gemm(As[i][None], Bs[i][None])[0]
            got = Ch[plan.offsets[2][i]:plan.offsets[2][i] + m * n].reshape(m, n)
            assert np.array_equal(got, ref), (pack, i, m, n, k)
    import ctypes
    from kami_b200 import _lib
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0
