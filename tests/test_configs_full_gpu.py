"""Parity at the full sizes of the benchmarked workloads, against the CPU
oracle, through the C ABI.

The other GPU tests run each kernel on small instances; the persistent
kernels' slot rings, mbarrier phases and longest-first schedules only reach
their steady state at the benchmark sizes, so every benchmarked configuration
is also checked here at exactly the size and seed that is timed:

1. FP64 32^3 x 1024, 2D partition, uniform[-1, 1] (seed 0), plus the
   reference's rand_r(i) % 3 inputs bit-exact (batched_gemm_2d_double_mma.cu:
   271-285, 338-358).
2. FP16 -> FP32 block GEMM, M = N = K in {16, 32, 64, 128} and 128 x 128 x
   {8, 16, 32}, batch 592 (4 x 148 SMs), every variant and partition; the
   timed launch (128^3, NUM_ITER 1000) with integer inputs (exact) and with
   uniform[-1, 1] inputs (FP32 bound over the 128000-term sums).
3. split-FP64 8192 x 64^3, sign * 10^u inputs: normwise error against the
   double-double oracle beside the native FP64 kernel on the same problems.
4. 20000 uneven problems (M, N, K log-uniform in [8, 128], multiples of 8,
   seed 0), FP16 and FP64, static and autotuned plans, and a graph-captured
   launch; exact on integer inputs.
5. block SpGEMM n = 16384 (1024^2 blocks of 16 x 16), 1 % block density,
   patterns from seeds 1 and 2: RowPtrC / ColIdxC exact, values exact on
   integer tiles and within the FP32 bound on uniform[-1, 1] tiles, by the
   host-synchronised and the on-device symbolic paths.
5b. BF16 batched GEMM forward + backward through the autograd function,
   4096 x 64^3: C, dA and dB against an FP64 torch.bmm of the same values.
"""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api
from kami_b200.autograd import bmm

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -23  # FP32 unit roundoff (round to nearest: 2^-24; 2^-23 covers truncating accumulation)
U64 = 2.0 ** -52


def _status_clean():
    import ctypes
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0


# ---------------------------------------------------------------------------
# config 1: FP64 32^3 x 1024, 2D
# ---------------------------------------------------------------------------
def test_config1_fp64_32cubed_x1024_uniform(cuda):
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, (1024, 32, 32))
    B = rng.uniform(-1, 1, (1024, 32, 32))  # the reference's N x K operand
    ref = oracle.gemm(A, B)
    bound = (32 + 2) * U64 * (np.abs(A) @ np.abs(B).transpose(0, 2, 1))
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    for part in ("2d", "1d", "3d", "auto"):
        C = api.gemm_batched(dA, dB, partition=part).cpu().numpy()
        assert np.all(np.abs(C - ref) <= bound), part
        assert np.linalg.norm(C - ref) / np.linalg.norm(ref) <= 1e-15, part
    _status_clean()


@pytest.mark.parametrize("part,P", [("2d", 1), ("2d", 2), ("1d", 2), ("3d", 2)])
def test_config1_fp64_reference_inputs_exact(cuda, part, P):
    # h_A[i] = rand_r(&i) % 3 over the whole batch, as the reference fills it
    A = oracle.fill_rand_r_mod(1024 * 32 * 32).reshape(1024, 32, 32)
    B = oracle.fill_rand_r_mod(1024 * 32 * 32).reshape(1024, 32, 32)
    C = api.gemm_batched(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), partition=part, P=P,
                         variant="mma_sync")
    assert np.array_equal(C.cpu().numpy(), oracle.gemm(A, B))


# ---------------------------------------------------------------------------
# config 2: FP16 -> FP32 block GEMM, batch 592
# ---------------------------------------------------------------------------
BATCH2 = 592
SHAPES2 = [(16, 16, 16), (32, 32, 32), (64, 64, 64), (128, 128, 128), (128, 128, 8), (128, 128, 16),
           (128, 128, 32)]
_ref2 = {}


def _inputs2(M, N, K, integer):
    key = (M, N, K, integer)
    if key not in _ref2:
        rng = np.random.default_rng(M * 1000 + K)
        if integer:
            A = rng.integers(-2, 3, (BATCH2, M, K)).astype(np.float16)
            B = rng.integers(-2, 3, (BATCH2, N, K)).astype(np.float16)
        else:
            A = rng.uniform(-1, 1, (BATCH2, M, K)).astype(np.float16)
            B = rng.uniform(-1, 1, (BATCH2, N, K)).astype(np.float16)
        ref = oracle.gemm(A, B)
        absref = oracle.gemm(np.abs(A), np.abs(B)) if not integer else None
        _ref2[key] = (torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), ref, absref)
    return _ref2[key]


def _variants(M, N, K):
    out = []
    for variant in ("mma_sync", "tcgen05", "tcgen05_ts", "auto"):
        for part in ("1d", "2d", "3d", "auto"):
            try:
                api.describe(M, N, K, BATCH2, torch.float16, variant=variant, partition=part)
            except Exception:
                continue
            out.append((variant, part))
    return out


@pytest.mark.parametrize("M,N,K", SHAPES2, ids=lambda v: str(v))
def test_config2_every_variant_num_iter_1000_exact(cuda, M, N, K):
    """NUM_ITER = 1000 on integer inputs in [-2, 2]: every partial sum is an
    integer below 2^24, so FP32 accumulation is exact in any order."""
    A, B, ref, _ = _inputs2(M, N, K, True)
    combos = _variants(M, N, K)
    assert combos, "no kernel for this shape"
    C = torch.empty((BATCH2, M, N), dtype=torch.float32, device="cuda")
    for variant, part in combos:
        C.fill_(float("nan"))
        api.gemm_batched(A, B, C, variant=variant, partition=part, num_iter=1000)
        got = C.double().cpu().numpy()
        assert np.array_equal(got, ref * 1000), (variant, part)
    _status_clean()


@pytest.mark.parametrize("M,N,K", SHAPES2, ids=lambda v: str(v))
def test_config2_every_variant_uniform(cuda, M, N, K):
    A, B, ref, absref = _inputs2(M, N, K, False)
    bound = (K + 2) * U32 * absref
    C = torch.empty((BATCH2, M, N), dtype=torch.float32, device="cuda")
    for variant, part in _variants(M, N, K):
        C.fill_(float("nan"))
        api.gemm_batched(A, B, C, variant=variant, partition=part)
        got = C.double().cpu().numpy()
        assert np.all(np.abs(got - ref) <= bound), (variant, part)
    _status_clean()


def test_config2_timed_launch_uniform_num_iter_1000(cuda):
    """The timed launch exactly: torch.rand inputs (seed 0) rounded to FP16,
    128^3 x 592, NUM_ITER 1000, the library's kernel choice.  Each C entry
    sums 128000 products in FP32."""
    g = torch.Generator(device="cpu").manual_seed(0)
    A_h = (torch.rand((BATCH2, 128, 128), generator=g) * 2 - 1).half()
    B_h = (torch.rand((BATCH2, 128, 128), generator=g) * 2 - 1).half()
    C = api.gemm_batched(A_h.cuda(), B_h.cuda(), num_iter=1000)
    got = C.double().cpu().numpy()
    A, B = A_h.numpy(), B_h.numpy()
    ref = oracle.gemm(A, B) * 1000
    absref = oracle.gemm(np.abs(A), np.abs(B)) * 1000
    assert np.all(np.abs(got - ref) <= (128 * 1000 + 2) * U32 * absref)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-3
    _status_clean()


def test_config2_host_buffer_call(cuda):
    """The end-to-end call on host buffers (kami_gemm_batched_host: chunked
    copies overlapping the products) gives the device call's result."""
    A, B, ref, _ = _inputs2(128, 128, 128, True)
    A_pin = A.cpu().pin_memory()
    B_pin = B.cpu().pin_memory()
    C_pin = torch.full((BATCH2, 128, 128), float("nan"), dtype=torch.float32).pin_memory()
    api.gemm_batched_host(A_pin, B_pin, C_pin, num_iter=1000)
    torch.cuda.synchronize()
    assert np.array_equal(C_pin.double().numpy(), ref * 1000)


# ---------------------------------------------------------------------------
# config 3: split-FP64, 8192 x 64^3, sign * 10^u
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def split_workload(cuda):
    rng = np.random.default_rng(0)
    A = rng.choice([-1.0, 1.0], size=(8192, 64, 64)) * 10.0 ** rng.uniform(-3, 3, size=(8192, 64, 64))
    B = rng.choice([-1.0, 1.0], size=(8192, 64, 64)) * 10.0 ** rng.uniform(-3, 3, size=(8192, 64, 64))
    hi, lo = oracle.gemm_dd(A, B)
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    native = api.gemm_batched(dA, dB).cpu().numpy()
    e_native = oracle.normwise_error_dd(native, hi, lo)
    return dA, dB, hi, lo, e_native


def test_config3_native_fp64_error(split_workload):
    _, _, _, _, e_native = split_workload
    assert 0 < e_native < 1e-15


@pytest.mark.parametrize("slice_dtype", [torch.float16, torch.bfloat16])
def test_config3_split_3_to_6_slices(split_workload, slice_dtype):
    """3-6 FP16 / BF16 slices with FP32 accumulation: each extra slice (9
    bits in binary16, 7 in bfloat16) cuts the normwise error by at least
    2^-7 / 2^-5 (two bits of slack) until the FP64 floor."""
    dA, dB, hi, lo, e_native = split_workload
    errs = []
    for s in (3, 4, 5, 6):
        C = api.split_f64_gemm(dA, dB, nslices=s, slice_dtype=slice_dtype).cpu().numpy()
        errs.append(oracle.normwise_error_dd(C, hi, lo))
    step = 2.0 ** -7 if slice_dtype == torch.float16 else 2.0 ** -5
    for a, b in zip(errs, errs[1:]):
        assert b <= max(a * step, 4 * e_native), errs
    # 3 slices carry 27 (binary16) / 21 (bfloat16) bits
    assert errs[0] < (1e-7 if slice_dtype == torch.float16 else 1e-5), errs


@pytest.mark.parametrize("slice_dtype,s", [(torch.float16, 7), (torch.bfloat16, 8), (torch.int8, 7),
                                           (torch.int8, 8)])
@pytest.mark.parametrize("num_iter", [1, 20])
def test_config3_split_within_2x_native_error(split_workload, slice_dtype, s, num_iter):
    """The FP64 target: normwise error no worse than 2x the native FP64
    kernel's on the same 8192 problems, streamed and with the products
    repeated on the resident digits (C / num_iter)."""
    dA, dB, hi, lo, e_native = split_workload
    C = api.split_f64_gemm(dA, dB, nslices=s, slice_dtype=slice_dtype, num_iter=num_iter).cpu().numpy() / num_iter
    e = oracle.normwise_error_dd(C, hi, lo)
    assert e <= 2.0 * e_native, (e, e_native)
    _status_clean()


# ---------------------------------------------------------------------------
# config 4: 20000 uneven problems
# ---------------------------------------------------------------------------
def _uneven20000():
    rng = np.random.default_rng(0)
    x = np.exp(rng.uniform(np.log(8), np.log(128), (20000, 3)))
    return np.clip(8 * np.round(x / 8), 8, 128).astype(np.int64)


def _uneven_inputs(shapes, dtype, seed):
    rng = np.random.default_rng(seed)
    a_sz = int((shapes[:, 0] * shapes[:, 2]).sum())
    b_sz = int((shapes[:, 1] * shapes[:, 2]).sum())
    A = rng.integers(-2, 3, a_sz).astype(np.float64)
    B = rng.integers(-2, 3, b_sz).astype(np.float64)
    return A, B, torch.tensor(A, dtype=dtype, device="cuda"), torch.tensor(B, dtype=dtype, device="cuda")


def _uneven_check(plan, A, B, C):
    """Every problem against the oracle, batched by shape."""
    Ch = C.double().cpu().numpy()
    ao, bo, co = plan.offsets
    shapes = plan.shapes
    keys = shapes[:, 0] * 1_000_000 + shapes[:, 1] * 1000 + shapes[:, 2]
    for key in np.unique(keys):
        idx = np.nonzero(keys == key)[0]
        m, n, k = (int(v) for v in shapes[idx[0]])
        As = np.stack([A[ao[i]:ao[i] + m * k].reshape(m, k) for i in idx])
        Bs = np.stack([B[bo[i]:bo[i] + n * k].reshape(n, k) for i in idx])
        got = np.stack([Ch[co[i]:co[i] + m * n].reshape(m, n) for i in idx])
        assert np.array_equal(got, oracle.gemm(As, Bs)), (m, n, k)


@pytest.mark.parametrize("dtype", [torch.float16, torch.float64])
@pytest.mark.parametrize("autotune", [False, True])
def test_config4_uneven_20000_exact(cuda, dtype, autotune):
    shapes = _uneven20000()
    A, B, dA, dB = _uneven_inputs(shapes, dtype, 1)
    plan = api.GroupedPlan(shapes, dtype, autotune=autotune)
    assert plan.info()["problems"] == 20000
    C = torch.full((plan.sizes[2],), float("nan"), dtype=plan.out_dtype, device="cuda")
    plan.run(dA, dB, C)
    _uneven_check(plan, A, B, C)
    _status_clean()


@pytest.mark.parametrize("dtype", [torch.float16, torch.float64])
def test_config4_uneven_20000_graph_replays(cuda, dtype):
    """One captured launch replayed on new inputs, as the benchmark runs it."""
    shapes = _uneven20000()
    A, B, dA, dB = _uneven_inputs(shapes, dtype, 2)
    plan = api.GroupedPlan(shapes, dtype)
    C = torch.zeros(plan.sizes[2], dtype=plan.out_dtype, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.run(dA, dB, C, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.run(dA, dB, C)
    for seed in (3, 4):
        A2, B2, dA2, dB2 = _uneven_inputs(shapes, dtype, seed)
        dA.copy_(dA2)
        dB.copy_(dB2)
        C.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        _uneven_check(plan, A2, B2, C)
    del g
    _status_clean()


def test_config4_uneven_20000_fp64_uniform(cuda):
    shapes = _uneven20000()
    rng = np.random.default_rng(5)
    a_sz = int((shapes[:, 0] * shapes[:, 2]).sum())
    b_sz = int((shapes[:, 1] * shapes[:, 2]).sum())
    A, B = rng.uniform(-1, 1, a_sz), rng.uniform(-1, 1, b_sz)
    plan = api.GroupedPlan(shapes, torch.float64)
    C = torch.empty(plan.sizes[2], dtype=torch.float64, device="cuda")
    plan.run(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), C)
    Ch = C.cpu().numpy()
    ao, bo, co = plan.offsets
    for i in range(0, 20000, 7):
        m, n, k = (int(v) for v in shapes[i])
        a = A[ao[i]:ao[i] + m * k].reshape(m, k)
        b = B[bo[i]:bo[i] + n * k].reshape(n, k)
        got = Ch[co[i]:co[i] + m * n].reshape(m, n)
        assert np.all(np.abs(got - a @ b.T) <= (k + 2) * U64 * (np.abs(a) @ np.abs(b).T)), i


# ---------------------------------------------------------------------------
# config 5: block SpGEMM n = 16384, 1 %
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def spgemm_patterns(cuda):
    nb = 1024
    rpa, cia = oracle.bsr_pattern(nb, nb, 0.01, 1)
    rpb, cib = oracle.bsr_pattern(nb, nb, 0.01, 2)
    return nb, (rpa, cia), (rpb, cib)


def _bsr_dev(rp, ci, vals, cols, dtype=torch.float16):
    return api.BSR(torch.tensor(rp, dtype=torch.int32, device="cuda"), torch.tensor(ci, dtype=torch.int32, device="cuda"),
                   torch.tensor(vals, dtype=dtype, device="cuda"), cols)


@pytest.mark.parametrize("values", ["integer", "uniform"])
def test_config5_spgemm_n16384_full(spgemm_patterns, values):
    nb, (rpa, cia), (rpb, cib) = spgemm_patterns
    rng = np.random.default_rng(0)
    if values == "integer":
        va = rng.integers(1, 4, (len(cia), 16, 16)).astype(np.float16)
        vb = rng.integers(1, 4, (len(cib), 16, 16)).astype(np.float16)
    else:
        va = rng.uniform(-1, 1, (len(cia), 16, 16)).astype(np.float16)
        vb = rng.uniform(-1, 1, (len(cib), 16, 16)).astype(np.float16)
    rpc_o, cic_o, vc_o = oracle.spgemm(nb, nb, (rpa, cia, va), (rpb, cib, vb), accum="double")
    A, B = _bsr_dev(rpa, cia, va, nb), _bsr_dev(rpb, cib, vb, nb)
    # host-synchronised sequence (the reference's), both numeric kernels
    C = api.spgemm(A, B, torch.float32, variant="mma_sync")
    C_tc = api.spgemm(A, B, torch.float32, variant="tcgen05")
    torch.cuda.synchronize()
    assert torch.equal(C_tc.row_ptr, C.row_ptr) and torch.equal(C_tc.col_idx, C.col_idx)
    assert np.array_equal(C.row_ptr.cpu().numpy(), rpc_o)
    assert np.array_equal(C.col_idx.cpu().numpy(), cic_o)
    got = C.values.double().cpu().numpy()
    got_tc = C_tc.values.double().cpu().numpy()
    if values == "integer":
        assert np.array_equal(got, vc_o)
        assert np.array_equal(got_tc, vc_o)
    else:
        absv = oracle.spgemm(nb, nb, (rpa, cia, np.abs(va)), (rpb, cib, np.abs(vb)), accum="double")[2]
        terms = 16 * int(np.max(np.diff(rpa)))
        assert np.all(np.abs(got - vc_o) <= (terms + 2) * U32 * absv)
        assert np.all(np.abs(got_tc - vc_o) <= (terms + 2) * U32 * absv)
    # on-device symbolic pass, capacity = nnzCub, numeric bounded by it
    cap = oracle.spgemm_nnzcub(cia, rpb)
    rpc, cic = api.spgemm_symbolic_device(A, B, cap)
    vals = torch.full((cap, 16, 16), float("nan"), dtype=torch.float32, device="cuda")
    api.spgemm_numeric_bound(A, B, rpc, cic, vals, variant="mma_sync")
    nnz = len(cic_o)
    assert int(rpc[-1]) == nnz
    assert np.array_equal(rpc.cpu().numpy(), rpc_o)
    assert np.array_equal(cic[:nnz].cpu().numpy(), cic_o)
    assert np.array_equal(vals[:nnz].double().cpu().numpy(), got)
    _status_clean()


# ---------------------------------------------------------------------------
# config 5b: BF16 fwd + bwd 4096 x 64^3
# ---------------------------------------------------------------------------
def test_config5b_bf16_fwd_bwd_4096(cuda):
    g = torch.Generator(device="cpu").manual_seed(0)
    A0 = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().cuda()
    B0 = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().cuda()
    G = (torch.rand((4096, 64, 64), generator=g) * 2 - 1).bfloat16().cuda()
    A, B = A0.clone().requires_grad_(), B0.clone().requires_grad_()
    C = bmm(A, B)
    C.backward(G)
    Ad, Bd, Gd = A0.double(), B0.double(), G.double()
    u16 = 2.0 ** -8  # bf16 rounding of the outputs
    checks = [(C, torch.bmm(Ad, Bd), torch.bmm(Ad.abs(), Bd.abs())),
              (A.grad, torch.bmm(Gd, Bd.transpose(1, 2)), torch.bmm(Gd.abs(), Bd.abs().transpose(1, 2))),
              (B.grad, torch.bmm(Ad.transpose(1, 2), Gd), torch.bmm(Ad.abs().transpose(1, 2), Gd.abs()))]
    for name, (got, ref, absref) in zip("C dA dB".split(), checks):
        assert got.dtype == torch.bfloat16
        err = (got.detach().double() - ref).abs()
        bound = u16 * ref.abs() + (1 + u16) * (64 + 2) * U32 * absref
        assert bool((err <= bound).all()), name
        assert float(err.norm() / ref.norm()) <= u16, name
    _status_clean()
