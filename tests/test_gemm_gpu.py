"""Parity of the batched block GEMM (mma.sync variant and AUTO) with the CPU
oracle, through the C ABI.  Integer-valued inputs must match exactly (the
reference's own check: |C/NUM_ITER - ref| <= 1e-6 on small integers);
uniform[-1,1] inputs must satisfy the FP32/FP64 accumulation bound
|C - C*| <= K * u * (|A||B|) elementwise (u = 2^-23 for FP32 accumulation of
16-bit products, 2^-52 for FP64), plus a normwise check."""
import glob
import os

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api
from kami_b200._lib import KamiError

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TDT = {"f16": torch.float16, "bf16": torch.bfloat16, "f64": torch.float64}


def _make(prec, batch, M, N, K, b_layout, a_layout, integer, seed=0):
    rng = np.random.default_rng(seed)
    if integer:
        A = rng.integers(0, 3, (batch, M, K)).astype(np.float64)
        Bt = rng.integers(0, 3, (batch, K, N)).astype(np.float64)  # K x N
    else:
        A = rng.uniform(-1, 1, (batch, M, K))
        Bt = rng.uniform(-1, 1, (batch, K, N))
    tA = torch.tensor(A, dtype=TDT[prec])
    tBt = torch.tensor(Bt, dtype=TDT[prec])
    # exact values the kernel sees
    A64 = tA.double().numpy()
    Bt64 = tBt.double().numpy()
    tA_dev = tA if a_layout == "row_mk" else tA.transpose(1, 2).contiguous()
    tB_dev = tBt.transpose(1, 2).contiguous() if b_layout == "ref_nk" else tBt
    return tA_dev.cuda(), tB_dev.cuda(), A64, Bt64


def _ref(A64, Bt64):
    return oracle.gemm(A64, np.ascontiguousarray(Bt64.transpose(0, 2, 1)), oracle.B_REF_NK)


def _bound(prec, A64, Bt64):
    u = 2.0 ** -52 if prec == "f64" else 2.0 ** -23
    K = A64.shape[2]
    return (K + 2) * u * (np.abs(A64) @ np.abs(Bt64)) + 1e-300


H16_INST = [(16, 16, 16, 1, "1d"), (16, 16, 16, 1, "2d"), (16, 16, 16, 1, "3d"),
            (32, 32, 32, 1, "1d"), (32, 32, 32, 2, "1d"), (32, 32, 32, 1, "2d"), (32, 32, 32, 2, "2d"),
            (32, 32, 32, 1, "3d"), (64, 64, 64, 2, "1d"), (64, 64, 64, 4, "1d"), (64, 64, 64, 2, "2d"),
            (64, 64, 64, 4, "2d"), (64, 64, 64, 2, "3d"), (128, 128, 128, 8, "1d"), (128, 128, 128, 4, "2d"),
            (128, 128, 128, 2, "3d"), (128, 128, 16, 4, "1d"), (128, 128, 16, 8, "1d"), (128, 128, 32, 4, "1d"),
            (128, 128, 32, 8, "1d"), (128, 128, 32, 2, "2d"), (128, 128, 64, 4, "1d"), (128, 128, 64, 4, "2d"),
            (128, 128, 8, 4, "1d")]
F64_INST = [(16, 16, 16, 1, "1d"), (16, 16, 16, 1, "2d"), (16, 16, 16, 1, "3d"), (32, 32, 32, 1, "1d"),
            (32, 32, 32, 2, "1d"), (32, 32, 32, 1, "2d"), (32, 32, 32, 2, "2d"), (32, 32, 32, 1, "3d"),
            (32, 32, 32, 2, "3d"), (64, 64, 64, 4, "1d"), (64, 64, 64, 2, "2d"), (64, 64, 64, 4, "2d"),
            (64, 64, 64, 2, "3d")]

CASES = [("f16",) + c for c in H16_INST] + [("bf16",) + c for c in H16_INST[::3]] + [("f64",) + c for c in F64_INST]


def _id(c):
    return f"{c[0]}-{c[1]}x{c[2]}x{c[3]}-P{c[4]}-{c[5]}"


@pytest.mark.parametrize("case", CASES, ids=_id)
def test_mma_parity_integer_exact(cuda, case):
    prec, M, N, K, P, part = case
    A, B, A64, Bt64 = _make(prec, 6, M, N, K, "ref_nk", "row_mk", integer=True)
    C = api.gemm_batched(A, B, variant="mma_sync", partition=part, P=P)
    torch.cuda.synchronize()
    assert np.array_equal(C.double().cpu().numpy(), _ref(A64, Bt64))


@pytest.mark.parametrize("case", CASES, ids=_id)
def test_mma_parity_uniform(cuda, case):
    prec, M, N, K, P, part = case
    A, B, A64, Bt64 = _make(prec, 5, M, N, K, "ref_nk", "row_mk", integer=False, seed=1)
    C = api.gemm_batched(A, B, variant="mma_sync", partition=part, P=P).double().cpu().numpy()
    ref = _ref(A64, Bt64)
    assert np.all(np.abs(C - ref) <= _bound(prec, A64, Bt64))
    rel = np.linalg.norm(C - ref) / np.linalg.norm(ref)
    assert rel <= (1e-14 if prec == "f64" else 2e-6)


@pytest.mark.parametrize("prec", ["f16", "bf16", "f64"])
@pytest.mark.parametrize("b_layout,a_layout", [("row_kn", "row_mk"), ("ref_nk", "col_mk"), ("row_kn", "col_mk")])
@pytest.mark.parametrize("part,P", [("1d", 2), ("2d", 2), ("3d", 2)])
def test_mma_layouts(cuda, prec, b_layout, a_layout, part, P):
    M = N = K = 32 if not (prec != "f64" and part == "3d") else 64
    A, B, A64, Bt64 = _make(prec, 3, M, N, K, b_layout, a_layout, integer=True, seed=3)
    C = api.gemm_batched(A, B, a_layout=a_layout, b_layout=b_layout, variant="mma_sync", partition=part, P=P)
    assert np.array_equal(C.double().cpu().numpy(), _ref(A64, Bt64))


@pytest.mark.parametrize("prec", ["f16", "f64"])
@pytest.mark.parametrize("num_iter", [1, 2, 7])
def test_num_iter_accumulates(cuda, prec, num_iter):
    # the reference's in-register repeat: C = NUM_ITER * A*B, checked as C / NUM_ITER
    for part, P in [("1d", 4), ("2d", 2), ("3d", 2)]:
        A, B, A64, Bt64 = _make(prec, 4, 64, 64, 64, "ref_nk", "row_mk", integer=True, seed=num_iter)
        C = api.gemm_batched(A, B, variant="mma_sync", partition=part, P=P, num_iter=num_iter)
        assert np.array_equal(C.double().cpu().numpy() / num_iter, _ref(A64, Bt64)), part


@pytest.mark.parametrize("prec", ["f16", "f64"])
def test_alpha_beta_and_out_types(cuda, prec):
    A, B, A64, Bt64 = _make(prec, 3, 32, 32, 32, "ref_nk", "row_mk", integer=True, seed=5)
    ref = _ref(A64, Bt64)
    C0 = torch.full((3, 32, 32), 2.0, dtype=torch.float64 if prec == "f64" else torch.float32, device="cuda")
    api.gemm_batched(A, B, C0, alpha=0.5, beta=3.0, variant="mma_sync")
    assert np.array_equal(C0.double().cpu().numpy(), 0.5 * ref + 6.0)
    if prec != "f64":
        for odt in (torch.float16, torch.bfloat16):
            C = api.gemm_batched(A, B, out_dtype=odt, variant="mma_sync")
            assert C.dtype == odt
            assert np.array_equal(C.double().cpu().numpy(), torch.tensor(ref).to(odt).double().numpy())


@pytest.mark.parametrize("prec", ["f16", "f64"])
@pytest.mark.parametrize("M,N,K", [(24, 40, 20), (1, 1, 4), (17, 9, 12), (100, 72, 36), (128, 120, 124)])
def test_ragged_shapes(cuda, prec, M, N, K):
    A, B, A64, Bt64 = _make(prec, 3, M, N, K, "ref_nk", "row_mk", integer=True, seed=M)
    C = api.gemm_batched(A, B)
    assert np.array_equal(C.double().cpu().numpy(), _ref(A64, Bt64))


@pytest.mark.parametrize("batch", [1, 3, 5, 1000, 70001])
def test_batch_sizes(cuda, batch):
    A, B, A64, Bt64 = _make("f16", batch, 16, 16, 16, "ref_nk", "row_mk", integer=True, seed=batch)
    C = api.gemm_batched(A, B, variant="mma_sync", partition="1d")
    assert np.array_equal(C.double().cpu().numpy(), _ref(A64, Bt64))


def test_empty_batch_is_noop(cuda):
    A = torch.zeros((0, 32, 32), dtype=torch.float16, device="cuda")
    B = torch.zeros((0, 32, 32), dtype=torch.float16, device="cuda")
    C = api.gemm_batched(A, B)
    assert C.shape == (0, 32, 32)


def test_alloc_warps_extra_warps_exit(cuda):
    A, B, A64, Bt64 = _make("f16", 4, 64, 64, 64, "ref_nk", "row_mk", integer=True)
    C = api.gemm_batched(A, B, variant="mma_sync", partition="2d", P=2, alloc_warps=8)
    assert np.array_equal(C.double().cpu().numpy(), _ref(A64, Bt64))


def test_unsupported_shape_raises(cuda):
    A = torch.zeros((1, 256, 256), dtype=torch.float16, device="cuda")
    with pytest.raises(KamiError):
        api.gemm_batched(A, A, variant="mma_sync")


def _dense_goldens():
    return sorted(glob.glob(os.path.join(GOLDEN, "dense_*.npz")))


@pytest.mark.parametrize("path", _dense_goldens(), ids=os.path.basename)
def test_reference_kernel_golden(cuda, path):
    """The reference's own kernel output (rand_r(i) % 3 inputs) is reproduced
    by the matching partition of this library."""
    z = np.load(path)
    M, N, K, P, num_iter, S, grid = (int(x) for x in z["cfg"])
    name = os.path.basename(path)
    part = "1d" if "1d_" in name else "2d" if "2d_" in name else "3d"
    dt = torch.float16 if "_f16_" in name else torch.float64
    A = torch.tensor(oracle.fill_rand_r_mod(grid * M * K).reshape(grid, M, K), dtype=dt, device="cuda")
    B = torch.tensor(oracle.fill_rand_r_mod(grid * N * K).reshape(grid, N, K), dtype=dt, device="cuda")
    C = api.gemm_batched(A, B, variant="mma_sync", partition=part, P=P, num_iter=num_iter)
    golden = oracle.reduce_slices(z["C"], S)
    assert np.array_equal(C.double().cpu().numpy(), golden)
