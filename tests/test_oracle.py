"""The CPU oracle, pinned against the reference (CPU only).

* SpGEMM: the restated generator and SPA match the reference's own
  generate_random_bsr_matrix / spgemm_spa bit for bit -- through the golden
  vectors in tests/golden (made by make_golden_spgemm.py from oracle/_ref),
  and directly against oracle/_ref when it is built.
* Dense: the restated check GEMM reproduces the golden outputs of the
  reference's own kernels (made on a GPU by make_golden_dense.py).
"""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _spgemm_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "spgemm_*.npz")))


def _dense_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "dense_*.npz")))


def test_golden_files_present():
    assert len(_spgemm_cases()) >= 5


@pytest.mark.parametrize("path", _spgemm_cases(), ids=os.path.basename)
def test_spgemm_oracle_matches_reference_golden(path):
    z = np.load(path)
    m, k, n = (int(x) for x in z["shape"])
    sp = float(z["sparsity"][0])
    A = oracle.bsr_generate(m, k, sp)
    B = oracle.bsr_generate(k, n, sp)
    for mine, key in zip(A, ["a_row_ptr", "a_col_idx", "a_vals"]):
        assert np.array_equal(np.asarray(mine).view(np.uint8), z[key].view(np.uint8)), key
    for mine, key in zip(B, ["b_row_ptr", "b_col_idx", "b_vals"]):
        assert np.array_equal(np.asarray(mine).view(np.uint8), z[key].view(np.uint8)), key
    rpc, cic, vc = oracle.spgemm(m, n, A, B, accum="half")
    assert np.array_equal(rpc, z["c_row_ptr"])
    assert np.array_equal(cic, z["c_col_idx"])
    assert np.array_equal(vc.view(np.uint16), z["c_vals"].view(np.uint16))
    # the double-accumulating mode agrees on these exactly-representable values
    rpc2, cic2, vc2 = oracle.spgemm(m, n, A, B, accum="double")
    assert np.array_equal(rpc2, rpc) and np.array_equal(cic2, cic)
    assert np.array_equal(vc2, vc.astype(np.float64))


@pytest.mark.skipif(not oracle.ref_available("spgemm2d_host"), reason="oracle/_ref not built")
@pytest.mark.parametrize("m,k,n,sp", [(5, 7, 3, 0.5), (32, 32, 32, 0.9), (1, 1, 1, 0.0), (20, 3, 9, 0.2)])
def test_spgemm_oracle_matches_reference_library(m, k, n, sp):
    L = oracle.ref_lib("spgemm2d_host")
    A = oracle.ref_bsr_generate(L, m, k, sp)
    B = oracle.ref_bsr_generate(L, k, n, sp)
    ref = oracle.ref_spgemm_spa(L, m, k, n, A, B)
    mine = oracle.spgemm(m, n, A, B, accum="half")
    for x, y in zip(ref, mine):
        assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


def test_spgemm_empty_rows_and_matrix():
    # an all-zero A gives an empty C with a zero row pointer
    A = (np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros((0, 16, 16), np.float16))
    B = oracle.bsr_generate(3, 5, 0.5)
    rpc, cic, vc = oracle.spgemm(3, 5, A, B)
    assert rpc.tolist() == [0, 0, 0, 0] and len(cic) == 0 and vc.shape[0] == 0


def test_nnzcub_counts_products():
    A = oracle.bsr_generate(8, 8, 0.5)
    B = oracle.bsr_generate(8, 8, 0.5)
    expect = sum(int(B[0][c + 1] - B[0][c]) for c in A[1])
    assert oracle.spgemm_nnzcub(A[1], B[0]) == expect


def test_fill_matches_libc_rand_r():
    libc = ctypes.CDLL("libc.so.6")
    libc.rand_r.argtypes = [ctypes.POINTER(ctypes.c_uint)]
    x = oracle.fill_rand_r_mod(1000, 3)
    for i in [0, 1, 2, 17, 999]:
        s = ctypes.c_uint(i)
        assert x[i] == libc.rand_r(ctypes.byref(s)) % 3


@pytest.mark.parametrize("path", _dense_cases(), ids=os.path.basename)
def test_dense_oracle_matches_reference_kernel_golden(path):
    z = np.load(path)
    M, N, K, P, num_iter, S, grid = (int(x) for x in z["cfg"])
    A = oracle.fill_rand_r_mod(grid * M * K).reshape(grid, M, K)
    B = oracle.fill_rand_r_mod(grid * N * K).reshape(grid, N, K)
    C = oracle.reduce_slices(z["C"], S) / num_iter
    ref = oracle.gemm(A, B, oracle.B_REF_NK)
    assert np.array_equal(C, ref)


@pytest.mark.parametrize("layout", [oracle.B_REF_NK, oracle.B_ROW_KN])
def test_gemm_oracle_against_numpy(layout):
    rng = np.random.default_rng(0)
    A = rng.uniform(-1, 1, (3, 17, 24))
    Bt = rng.uniform(-1, 1, (3, 24, 9))  # K x N
    B = np.ascontiguousarray(Bt.transpose(0, 2, 1)) if layout == oracle.B_REF_NK else Bt
    C = oracle.gemm(A, B, layout)
    assert np.allclose(C, A @ Bt, rtol=0, atol=1e-13)
    h = oracle.gemm(A.astype(np.float16), B.astype(np.float16), layout)
    assert np.allclose(h, A.astype(np.float16).astype(np.float64) @ Bt.astype(np.float16).astype(np.float64),
                       rtol=0, atol=1e-12)


def test_double_double_oracle_is_exact_on_cancellation():
    # (1 + 2^-40)(1 - 2^-40) + (-1) = -2^-80: lost entirely in double, kept in dd
    A = np.array([[[1 + 2.0 ** -40, 1.0]]])
    B = np.array([[[1 - 2.0 ** -40, -1.0]]])  # REF_NK: N=1, K=2
    hi, lo = oracle.gemm_dd(A, B)
    assert hi[0, 0, 0] + lo[0, 0, 0] == -(2.0 ** -80)
    err = oracle.normwise_error_dd(np.zeros((1, 1, 1)), hi, lo)
    assert err == pytest.approx(1.0)


def test_double_double_against_mpmath():
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    rng = np.random.default_rng(1)
    A = rng.uniform(-1, 1, (1, 4, 33)) * 10.0 ** rng.uniform(-3, 3, (1, 4, 33))
    B = rng.uniform(-1, 1, (1, 5, 33)) * 10.0 ** rng.uniform(-3, 3, (1, 5, 33))
    hi, lo = oracle.gemm_dd(A, B)
    for i in range(4):
        for j in range(5):
            exact = mpmath.fsum(mpmath.mpf(a) * mpmath.mpf(b) for a, b in zip(A[0, i], B[0, j]))
            got = mpmath.mpf(hi[0, i, j]) + mpmath.mpf(lo[0, i, j])
            scale = mpmath.fsum(abs(mpmath.mpf(a) * mpmath.mpf(b)) for a, b in zip(A[0, i], B[0, j]))
            assert abs(got - exact) <= scale * mpmath.mpf(2) ** -100


# --------------------------------------------------------------------------
# block SpMM
# --------------------------------------------------------------------------

def _spmm_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "spmm_*.npz")))


@pytest.mark.parametrize("path", _spmm_cases(), ids=os.path.basename)
def test_spmm_oracle_matches_reference_kernel_golden(path):
    """The restated SpMM host check reproduces the outputs of the
    reference's own block_spmm_{1d,2d,3d}_half_mma kernels (exact small
    integers; tiled-BSR indices for 2D / 3D)."""
    g = np.load(path)
    M, N, K, P, tile_rows, tile_cols, _ = (int(x) for x in g["cfg"])
    C = oracle.spmm(g["row_ptr"], g["col_idx"], g["vals"].astype(np.float64), K // 16, g["B"].astype(np.float64),
                    "ref_nk", tile_rows=tile_rows, tile_cols=tile_cols)
    assert np.array_equal(C, g["C"])


@pytest.mark.parametrize("lib,rule", [("spmm1d_64p4", "spmm1d"), ("spmm2d_64p2", "spmm2d"),
                                      ("spmm3d_64p2", "spmm2d")])
@pytest.mark.parametrize("rows,cols,sp", [(4, 4, 0.5), (8, 6, 0.3), (6, 8, 0.9)])
def test_spmm_generator_and_tiling_match_reference_library(lib, rule, rows, cols, sp):
    if not oracle.ref_available(lib):
        pytest.skip("oracle/_ref not built")
    L = oracle.ref_lib(lib)
    a = oracle.ref_bsr_generate(L, rows, cols, sp)
    b = oracle.bsr_generate(rows, cols, sp, rule=rule)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    cfg = oracle.ref_spmm_config(L)
    if cfg["tile_rows"] and (rows, cols) == (cfg["M"] // 16, cfg["K"] // 16):
        # bsr2tilebsr tiles with its compile-time geometry (BSR_ROWS, BSR_COLS,
        # NUMS_ROW, NUMS_COL), so it is compared at the compiled shape only
        r1 = oracle.ref_bsr2tilebsr(L, a[0], a[1], cols, cfg["P"], cfg["tile_cols"])
        r2 = oracle.bsr2tilebsr(a[0], a[1], cols, cfg["P"], cfg["tile_cols"])
        for x, y in zip(r1, r2):
            assert np.array_equal(x, y)


def test_spmm_oracle_against_numpy():
    rng = np.random.default_rng(5)
    rp, ci = oracle.bsr_pattern(6, 5, 0.4, 11)
    vals = rng.uniform(-1, 1, (ci.size, 16, 16))
    dense = np.zeros((96, 80))
    for r in range(6):
        for e in range(rp[r], rp[r + 1]):
            dense[16 * r:16 * r + 16, 16 * ci[e]:16 * ci[e] + 16] = vals[e]
    B = rng.uniform(-1, 1, (80, 33))
    assert np.allclose(oracle.spmm(rp, ci, vals, 5, B, "row_kn"), dense @ B, rtol=0, atol=1e-12)
    assert np.allclose(oracle.spmm(rp, ci, vals, 5, np.ascontiguousarray(B.T), "ref_nk"), dense @ B, rtol=0,
                       atol=1e-12)
