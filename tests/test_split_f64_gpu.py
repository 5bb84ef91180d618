"""FP64-accurate GEMM on the FP16/BF16 tensor cores (exact digit splitting)
against the double-double CPU oracle, beside the native FP64 (DMMA) kernel
of this library."""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api

pytestmark = pytest.mark.gpu


def wide_range(shape, rng):
    # sign * 10^u, u ~ U[-3, 3]: the wide-exponent workload of the FP64 target
    return rng.choice([-1.0, 1.0], size=shape) * 10.0 ** rng.uniform(-3, 3, size=shape)


def test_exact_on_integer_inputs(cuda):
    rng = np.random.default_rng(0)
    A = rng.integers(-1000, 1001, (16, 64, 64)).astype(np.float64)
    B = rng.integers(-1000, 1001, (16, 64, 64)).astype(np.float64)
    ref = oracle.gemm(A, B)
    for s in (2, 4, 6):
        C = api.split_f64_gemm(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), nslices=s)
        assert np.array_equal(C.cpu().numpy(), ref), s


@pytest.mark.parametrize("slice_dtype,s", [(torch.float16, 7), (torch.bfloat16, 8)])
def test_error_vs_double_double_and_native(cuda, slice_dtype, s):
    rng = np.random.default_rng(1)
    A = wide_range((64, 64, 64), rng)
    B = wide_range((64, 64, 64), rng)
    hi, lo = oracle.gemm_dd(A, B)
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    native = api.gemm_batched(dA, dB).cpu().numpy()
    split = api.split_f64_gemm(dA, dB, nslices=s, slice_dtype=slice_dtype).cpu().numpy()
    e_native = oracle.normwise_error_dd(native, hi, lo)
    e_split = oracle.normwise_error_dd(split, hi, lo)
    assert e_native < 1e-15
    # the target: no worse than 2x the native FP64 kernel's normwise error
    assert e_split <= 2.0 * e_native, (e_split, e_native)


@pytest.mark.parametrize("s", [2, 3, 4, 5])
def test_error_decreases_with_slices(cuda, s):
    """More digits, less error (down to the FP64 floor)."""
    rng = np.random.default_rng(2)
    A = wide_range((8, 64, 64), rng)
    B = wide_range((8, 64, 64), rng)
    hi, lo = oracle.gemm_dd(A, B)
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    e = [oracle.normwise_error_dd(api.split_f64_gemm(dA, dB, nslices=k).cpu().numpy(), hi, lo) for k in (s, s + 1)]
    # each extra 9-bit digit buys about 2^-9 until the FP64 floor
    assert e[1] <= max(e[0] * 2.0 ** -6, 1e-15)


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (17, 40, 33), (64, 1, 64), (1, 64, 2), (32, 32, 32)])
@pytest.mark.parametrize("b_layout", ["ref_nk", "row_kn"])
def test_shapes_layouts_alpha_beta(cuda, M, N, K, b_layout):
    rng = np.random.default_rng(M * N + K)
    A = rng.uniform(-1, 1, (5, M, K))
    Bt = rng.uniform(-1, 1, (5, K, N))
    B = np.ascontiguousarray(Bt.transpose(0, 2, 1)) if b_layout == "ref_nk" else Bt
    hi, lo = oracle.gemm_dd(A, np.ascontiguousarray(Bt.transpose(0, 2, 1)))
    C0 = rng.uniform(-1, 1, (5, M, N))
    dC = torch.tensor(C0, device="cuda")
    if K % 2 and b_layout == "ref_nk":
        pytest.skip("REF_NK rows must be 16-byte aligned")
    if K % 2:
        pytest.skip("A rows must be 16-byte aligned")
    api.split_f64_gemm(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), dC, nslices=6,
                       b_layout=b_layout, alpha=2.0, beta=0.5)
    ref = 2.0 * (hi + lo) + 0.5 * C0
    got = dC.cpu().numpy()
    # split error is relative to the row / column maxima: |err| <= c u K max|a_i| max|b_j|
    bound = 8 * K * 2.0 ** -53 * (np.abs(A).max(axis=2)[:, :, None] * np.abs(Bt).max(axis=1)[:, None, :] * 2
                                  + np.abs(C0))
    assert np.all(np.abs(got - ref) <= bound)


def test_num_iter_repeats_products(cuda):
    rng = np.random.default_rng(3)
    A = rng.integers(-50, 51, (4, 64, 64)).astype(np.float64)
    B = rng.integers(-50, 51, (4, 64, 64)).astype(np.float64)
    C = api.split_f64_gemm(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), nslices=3, num_iter=5)
    assert np.array_equal(C.cpu().numpy(), 5 * oracle.gemm(A, B))


@pytest.mark.parametrize("slice_dtype,s,b_layout,N", [(torch.float16, 3, "ref_nk", 64), (torch.float16, 6, "ref_nk", 64),
                                                       (torch.bfloat16, 8, "ref_nk", 64),
                                                       (torch.float16, 6, "row_kn", 63)])
def test_streamed_many_problems_exact(cuda, slice_dtype, s, b_layout, N):
    """Many problems per CTA (the persistent form's buffer rings and phases),
    staged (aligned rows) and unstaged (row_kn with an odd N) inputs; integer
    inputs make every digit product exact, so the result must be exact."""
    rng = np.random.default_rng(s + N)
    batch = 1500
    A = rng.integers(-2000, 2001, (batch, 64, 64)).astype(np.float64)
    Bt = rng.integers(-2000, 2001, (batch, 64, N)).astype(np.float64)
    B = np.ascontiguousarray(Bt.transpose(0, 2, 1)) if b_layout == "ref_nk" else Bt
    C = api.split_f64_gemm(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), nslices=s,
                           slice_dtype=slice_dtype, b_layout=b_layout)
    assert np.array_equal(C.cpu().numpy(), np.matmul(A, Bt))


@pytest.mark.parametrize("s", [2, 4, 7, 8])
def test_int8_digits_exact_on_integer_inputs(cuda, s):
    """int8 digits (kind::i8 MMAs, INT32 accumulation) on integer inputs:
    exact, per-problem (num_iter > 4) and streamed forms."""
    rng = np.random.default_rng(20 + s)
    A = rng.integers(-1000, 1001, (300, 64, 64)).astype(np.float64)
    B = rng.integers(-1000, 1001, (300, 64, 64)).astype(np.float64)
    ref = oracle.gemm(A, B)
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    C = api.split_f64_gemm(dA, dB, nslices=s, slice_dtype=torch.int8)
    assert np.array_equal(C.cpu().numpy(), ref)
    C5 = api.split_f64_gemm(dA[:8], dB[:8], nslices=s, slice_dtype=torch.int8, num_iter=5)
    assert np.array_equal(C5.cpu().numpy(), 5 * ref[:8])


def test_int8_eight_digits_error_vs_native(cuda):
    """8 int8 digits (62 bits): no worse than 2x the native FP64 kernel's
    normwise error against the double-double oracle, on the wide-exponent
    workload."""
    rng = np.random.default_rng(21)
    A = wide_range((64, 64, 64), rng)
    B = wide_range((64, 64, 64), rng)
    hi, lo = oracle.gemm_dd(A, B)
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    e_native = oracle.normwise_error_dd(api.gemm_batched(dA, dB).cpu().numpy(), hi, lo)
    for it in (1, 6):  # streamed and per-problem forms
        C = api.split_f64_gemm(dA, dB, nslices=8, slice_dtype=torch.int8, num_iter=it).cpu().numpy() / it
        e = oracle.normwise_error_dd(C, hi, lo)
        assert e <= 2.0 * e_native, (it, e, e_native)


@pytest.mark.parametrize("M,N,K,b_layout", [(17, 40, 34, "row_kn"), (64, 1, 64, "row_kn"), (33, 64, 2, "ref_nk")])
def test_int8_shapes_layouts(cuda, M, N, K, b_layout):
    rng = np.random.default_rng(M + N + K)
    A = rng.uniform(-1, 1, (5, M, K))
    Bt = rng.uniform(-1, 1, (5, K, N))
    B = np.ascontiguousarray(Bt.transpose(0, 2, 1)) if b_layout == "ref_nk" else Bt
    hi, lo = oracle.gemm_dd(A, np.ascontiguousarray(Bt.transpose(0, 2, 1)))
    C = api.split_f64_gemm(torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda"), nslices=8,
                           slice_dtype=torch.int8, b_layout=b_layout).cpu().numpy()
    bound = 8 * K * 2.0 ** -53 * (np.abs(A).max(axis=2)[:, :, None] * np.abs(Bt).max(axis=1)[:, None, :]) * 2
    assert np.all(np.abs(C - (hi + lo)) <= bound)
