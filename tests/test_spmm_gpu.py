"""Block SpMM (BSR or tiled-BSR A, dense B) through the C ABI, against the
CPU oracle (the reference programs' host check restated) and the golden
outputs of the reference's own kernels."""
import glob
import os

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dense_of(rp, ci, vals, mb, kb):
    D = np.zeros((mb * 16, kb * 16))
    for r in range(mb):
        for e in range(rp[r], rp[r + 1]):
            D[16 * r:16 * r + 16, 16 * ci[e]:16 * ci[e] + 16] = vals[e]
    return D


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "spmm_*.npz"))), ids=os.path.basename)
def test_reference_kernel_golden(cuda, path):
    """Exact against the reference kernels' outputs, in the index form each
    kernel takes (BSR for 1D, tiled BSR for 2D / 3D)."""
    g = np.load(path)
    M, N, K, P, tile_rows, tile_cols, ref_iter = (int(x) for x in g["cfg"])
    rp = torch.tensor(g["row_ptr"], dtype=torch.int32, device="cuda")
    ci = torch.tensor(g["col_idx"], dtype=torch.int32, device="cuda")
    vals = torch.tensor(g["vals"], device="cuda")
    B = torch.tensor(g["B"], device="cuda")
    for it in (1, ref_iter):
        C = api.spmm_batched(rp, ci, vals, K // 16, B, b_layout="ref_nk", num_iter=it, tile_rows=tile_rows,
                             tile_cols=tile_cols)
        assert np.array_equal(C[0].double().cpu().numpy(), it * g["C"]), it


def _bound(Aabs, Babs, K, out_dtype):
    u = {torch.float32: 2.0 ** -24, torch.float16: 2.0 ** -11, torch.bfloat16: 2.0 ** -8}[out_dtype]
    return (K + 2) * 2.0 ** -23 * (Aabs @ Babs) + u * (Aabs @ Babs) + 1e-30


@pytest.mark.parametrize("mb,kb,N,density", [(8, 8, 64, 0.3), (16, 4, 33, 0.5), (5, 20, 100, 0.2),
                                             (64, 64, 256, 0.02), (3, 1, 8, 1.0), (7, 9, 1, 0.4)])
@pytest.mark.parametrize("b_layout", ["ref_nk", "row_kn"])
@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_random_vs_oracle(cuda, mb, kb, N, density, b_layout, dtype):
    """Panel (K <= 256) and streamed (K > 256) forms, N not a multiple of 8 or
    64, both B layouts, FP16 and BF16, within the FP32-accumulation bound."""
    rng = np.random.default_rng(mb * 1000 + kb * 10 + N)
    rp, ci = oracle.bsr_pattern(mb, kb, density, mb + kb + N)
    vals = torch.tensor(rng.uniform(-1, 1, (max(ci.size, 1), 16, 16))[: ci.size]).to(dtype)
    Bk = torch.tensor(rng.uniform(-1, 1, (kb * 16, N))).to(dtype)
    Bop = Bk if b_layout == "row_kn" else Bk.t().contiguous()
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"), vals.cuda(), kb)
    C = api.spmm(A, Bop.cuda(), b_layout=b_layout).double().cpu().numpy()
    ref = oracle.spmm(rp, ci, vals.double().numpy(), kb, Bop.double().numpy(), b_layout)
    D = _dense_of(rp, ci, np.abs(vals.double().numpy()), mb, kb)
    assert np.all(np.abs(C - ref) <= _bound(D, np.abs(Bk.double().numpy()), kb * 16, torch.float32))


@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16, torch.bfloat16])
def test_integer_inputs_exact_alpha_beta(cuda, out_dtype):
    rng = np.random.default_rng(3)
    mb, kb, N = 12, 10, 72
    rp, ci = oracle.bsr_pattern(mb, kb, 0.3, 4)
    vals = rng.integers(-2, 3, (ci.size, 16, 16)).astype(np.float64)
    Bk = rng.integers(-2, 3, (kb * 16, N)).astype(np.float64)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), kb)
    C0 = rng.integers(-3, 4, (mb * 16, N)).astype(np.float64)
    dC = torch.tensor(C0, dtype=out_dtype, device="cuda")
    api.spmm(A, torch.tensor(Bk, dtype=torch.float16, device="cuda"), dC, alpha=2.0, beta=-1.0)
    ref = 2.0 * oracle.spmm(rp, ci, vals, kb, Bk, "row_kn") - C0
    # |values| stay below 2^8, exact in every output type
    assert np.array_equal(dC.double().cpu().numpy(), ref)


def test_num_iter_repeats_products(cuda):
    rng = np.random.default_rng(4)
    rp, ci = oracle.bsr_pattern(4, 4, 0.5, 9)
    vals = rng.integers(-1, 2, (ci.size, 16, 16)).astype(np.float64)
    B = rng.integers(-1, 2, (64, 64)).astype(np.float64)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), 4)
    C = api.spmm(A, torch.tensor(B, dtype=torch.float16, device="cuda"), b_layout="ref_nk", num_iter=1000)
    assert np.array_equal(C.double().cpu().numpy(), 1000 * oracle.spmm(rp, ci, vals, 4, B, "ref_nk"))


def test_batched_shared_and_distinct_operands(cuda):
    """batch problems: the pattern shared (stride 0, the reference's launch),
    values and B per problem, C per problem."""
    rng = np.random.default_rng(6)
    batch, mb, kb, N = 300, 4, 4, 64
    rp, ci = oracle.bsr_pattern(mb, kb, 0.5, 2)
    vals = rng.integers(-2, 3, (batch, ci.size, 16, 16)).astype(np.float64)
    B = rng.integers(-2, 3, (batch, N, kb * 16)).astype(np.float64)
    C = api.spmm_batched(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                         torch.tensor(vals, dtype=torch.float16, device="cuda"), kb,
                         torch.tensor(B, dtype=torch.float16, device="cuda"), b_layout="ref_nk")
    got = C.double().cpu().numpy()
    for b in (0, 1, 147, 148, 299):
        assert np.array_equal(got[b], oracle.spmm(rp, ci, vals[b], kb, B[b], "ref_nk")), b


def test_tilebsr_equals_bsr(cuda):
    """The tiled-BSR form (kami_bsr_to_tilebsr + values gathered through
    perm) multiplies the same matrix as the BSR form."""
    rng = np.random.default_rng(8)
    mb, kb, N = 8, 12, 96
    rp, ci = oracle.bsr_pattern(mb, kb, 0.4, 5)
    vals = rng.integers(-2, 3, (ci.size, 16, 16)).astype(np.float64)
    B = rng.integers(-2, 3, (kb * 16, N)).astype(np.float64)
    brp, bci, perm = api.bsr_to_tilebsr(rp, ci, kb, 2, 3)
    ref_brp, ref_bci = oracle.bsr2tilebsr(rp, ci, kb, mb // 2, 3)
    assert np.array_equal(brp, ref_brp) and np.array_equal(bci, ref_bci)
    dB = torch.tensor(B, dtype=torch.float16, device="cuda")
    Ct = api.spmm_batched(torch.tensor(brp, device="cuda"), torch.tensor(bci, device="cuda"),
                          torch.tensor(vals[perm], dtype=torch.float16, device="cuda"), kb, dB,
                          b_layout="row_kn", tile_rows=2, tile_cols=3)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), kb)
    Cb = api.spmm(A, dB)
    assert np.array_equal(Ct[0].cpu().numpy(), Cb.cpu().numpy())


def test_empty_rows_and_out_of_range_columns(cuda):
    """Rows without entries give zeros; a block column outside [0, kb) is
    skipped by the kernel's own bounds check."""
    rp = np.array([0, 0, 2, 2, 3], dtype=np.int32)
    ci = np.array([0, 5, 1], dtype=np.int32)  # 5 >= kb = 2: skipped
    vals = np.ones((3, 16, 16))
    B = np.ones((32, 16))
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), 2)
    C = api.spmm(A, torch.tensor(B, dtype=torch.float16, device="cuda")).cpu().numpy()
    ref = oracle.spmm(rp[:], np.array([0, 0, 1], dtype=np.int32), np.stack([vals[0], 0 * vals[1], vals[2]]), 2,
                      B, "row_kn")
    assert np.array_equal(C, ref)
    assert np.all(C[:16] == 0) and np.all(C[32:48] == 0)


def test_shared_operands_batched_output(cuda):
    """Every operand shared, C batched: each problem is the same product (the
    reference's launch of 16384 CTAs on one A and B)."""
    rp, ci, vals = oracle.bsr_generate(4, 4, 0.5, rule="spmm1d")
    rng = np.random.default_rng(1)
    B = rng.integers(0, 3, (64, 64)).astype(np.float64)
    C = torch.full((700, 64, 64), -1.0, device="cuda")
    api.spmm_batched(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                     torch.tensor(vals, device="cuda"), 4, torch.tensor(B, dtype=torch.float16, device="cuda"), C,
                     b_layout="ref_nk", num_iter=3)
    ref = 3 * oracle.spmm(rp, ci, vals.astype(np.float64), 4, B, "ref_nk")
    got = C.double().cpu().numpy()
    assert all(np.array_equal(got[b], ref) for b in (0, 1, 350, 699))


def _int_bsr(mb, kb, density, seed):
    rng = np.random.default_rng(seed)
    rp, ci = oracle.bsr_pattern(mb, kb, density, seed)
    vals = rng.integers(-2, 3, (ci.size, 16, 16)).astype(np.float64)
    return rp, ci, vals


@pytest.mark.parametrize("N", [1, 16, 100, 128, 129, 256, 300, 512, 600])
@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("b_layout", ["row_kn", "ref_nk"])
def test_tcgen05_form_exact(cuda, N, dtype, b_layout):
    """One problem with K beyond the staged panel: the tcgen05 kernel
    (C^T = B^T A^T per block-row) with N up to 512, for B K x N (its slices
    MN-major) and the reference's N x K (K-major); the mma.sync streamed form
    for N = 600; rows without entries included."""
    mb, kb = 40, 24
    rp, ci, vals = _int_bsr(mb, kb, 0.15, N)
    Bk = np.random.default_rng(N + 1).integers(-2, 3, (kb * 16, N)).astype(np.float64)
    B = Bk if b_layout == "row_kn" else np.ascontiguousarray(Bk.T)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=dtype, device="cuda"), kb)
    C = api.spmm(A, torch.tensor(B, dtype=dtype, device="cuda"), b_layout=b_layout)
    assert np.array_equal(C.double().cpu().numpy(), oracle.spmm(rp, ci, vals, kb, B, b_layout))


def test_tcgen05_both_layouts_full_size(cuda):
    """n = 16384 with 1 % of its 16 x 16 tiles, 256 dense columns (the
    bench's large SpMM): B as K x N and the same B transposed as N x K run
    the same MMAs in the same order (only the slice's shared-memory layout
    differs), so the two results are identical; the first 64 block-rows
    against the oracle within the FP32-accumulation bound."""
    nb, N = 1024, 256
    rp, ci = oracle.bsr_pattern(nb, nb, 0.01, 1)
    rng = np.random.default_rng(11)
    vals = rng.uniform(-1, 1, (ci.size, 16, 16)).astype(np.float16)
    Bk = rng.uniform(-1, 1, (nb * 16, N)).astype(np.float16)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, device="cuda"), nb)
    C_kn = api.spmm(A, torch.tensor(Bk, device="cuda"), b_layout="row_kn")
    C_nk = api.spmm(A, torch.tensor(np.ascontiguousarray(Bk.T), device="cuda"), b_layout="ref_nk")
    assert torch.equal(C_kn, C_nk)
    ref = oracle.spmm(rp[:65], ci[: rp[64]], vals[: rp[64]].astype(np.float64), nb, Bk.astype(np.float64), "row_kn")
    absref = oracle.spmm(rp[:65], ci[: rp[64]], np.abs(vals[: rp[64]].astype(np.float64)), nb,
                         np.abs(Bk.astype(np.float64)), "row_kn")
    got = C_kn[: 64 * 16].double().cpu().numpy()
    # FP32 accumulation over at most 16 * (tiles in a row) products per element
    kmax = 16 * int(np.diff(rp[:65]).max())
    assert np.all(np.abs(got - ref) <= (kmax + 2) * 2.0 ** -24 * absref + 1e-30)


@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16, torch.bfloat16])
def test_tcgen05_form_alpha_beta_repeats(cuda, out_dtype):
    mb, kb, N = 30, 20, 200
    rp, ci, vals = _int_bsr(mb, kb, 0.2, 5)
    B = np.random.default_rng(6).integers(-1, 2, (kb * 16, N)).astype(np.float64)
    C0 = np.random.default_rng(7).integers(-3, 4, (mb * 16, N)).astype(np.float64)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), kb)
    dC = torch.tensor(C0, dtype=out_dtype, device="cuda")
    api.spmm(A, torch.tensor(B, dtype=torch.float16, device="cuda"), dC, b_layout="row_kn", alpha=2.0, beta=-1.0,
             num_iter=3)
    ref = 2.0 * 3 * oracle.spmm(rp, ci, vals, kb, B, "row_kn") - C0
    ref = torch.tensor(ref, dtype=torch.float32).to(out_dtype).double().numpy()
    assert np.array_equal(dC.double().cpu().numpy(), ref)


@pytest.mark.parametrize("b_layout", ["row_kn", "ref_nk"])
def test_tcgen05_form_out_of_range_columns(cuda, b_layout):
    """A block column outside [0, kb) contributes nothing (zero-filled B
    slice in the tcgen05 kernel, skipped by the mma.sync kernels)."""
    mb, kb, N = 4, 20, 64
    rp = np.array([0, 2, 2, 4, 5], dtype=np.int32)
    ci = np.array([3, 25, 0, 19, -4], dtype=np.int32)
    vals = np.ones((5, 16, 16))
    Bk = np.random.default_rng(9).integers(-2, 3, (kb * 16, N)).astype(np.float64)
    B = Bk if b_layout == "row_kn" else np.ascontiguousarray(Bk.T)
    A = api.BSR(torch.tensor(rp, device="cuda"), torch.tensor(ci, device="cuda"),
                torch.tensor(vals, dtype=torch.float16, device="cuda"), kb)
    C = api.spmm(A, torch.tensor(B, dtype=torch.float16, device="cuda"), b_layout=b_layout).cpu().numpy()
    keep = np.array([True, False, True, True, False])
    ref = oracle.spmm(rp, np.where(keep, ci, 0).astype(np.int32), vals * keep[:, None, None], kb, B, b_layout)
    assert np.array_equal(C, ref)
