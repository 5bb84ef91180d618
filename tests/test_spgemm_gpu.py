"""Block SpGEMM (BSR, 16 x 16 tiles) through the C ABI against the CPU
oracle: exact structure (RowPtrC, ColIdxC ascending) and values -- bit-exact
on the reference's own integer-valued generator and golden vectors, within
the FP32-accumulation bound on uniform[-1,1] tiles."""
import glob
import os

import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def to_dev(M, block_cols, dtype=torch.float16):
    rp, ci, v = M
    return api.BSR(torch.tensor(rp, dtype=torch.int32, device="cuda"),
                   torch.tensor(ci, dtype=torch.int32, device="cuda"),
                   torch.tensor(np.asarray(v, dtype=np.float32), dtype=dtype, device="cuda").reshape(-1, 16, 16),
                   block_cols)


def random_bsr(rows, cols, density, seed, integer):
    rp, ci = oracle.bsr_pattern(rows, cols, density, seed)
    rng = np.random.default_rng(seed)
    if integer:
        v = rng.integers(1, 4, (len(ci), 16, 16)).astype(np.float16)
    else:
        v = rng.uniform(-1, 1, (len(ci), 16, 16)).astype(np.float16)
    return rp, ci, v


def run(A, B, mb, kb, nb, out_dtype=torch.float32, num_iter=1, dtype=torch.float16, variant="auto"):
    dA, dB = to_dev(A, kb, dtype), to_dev(B, nb, dtype)
    C = api.spgemm(dA, dB, out_dtype, num_iter=num_iter, variant=variant)
    torch.cuda.synchronize()
    return C.row_ptr.cpu().numpy(), C.col_idx.cpu().numpy(), C.values.double().cpu().numpy()


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "spgemm_*.npz"))), ids=os.path.basename)
def test_reference_golden(cuda, path):
    z = np.load(path)
    m, k, n = (int(x) for x in z["shape"])
    A = (z["a_row_ptr"], z["a_col_idx"], z["a_vals"])
    B = (z["b_row_ptr"], z["b_col_idx"], z["b_vals"])
    rpc, cic, vc = run(A, B, m, k, n, out_dtype=torch.float16)
    assert np.array_equal(rpc, z["c_row_ptr"])
    assert np.array_equal(cic, z["c_col_idx"])
    assert np.array_equal(vc.astype(np.float16).view(np.uint16), z["c_vals"].view(np.uint16))


@pytest.mark.parametrize("num_iter", [1, 4])
def test_reference_generator_num_iter(cuda, num_iter):
    # the reference's 128^2 case (8 x 8 blocks, sparsity 0.5) with NUM_ITER repeats
    A = oracle.bsr_generate(8, 8, 0.5)
    rpc, cic, vc = run(A, A, 8, 8, 8, num_iter=num_iter)
    r = oracle.spgemm(8, 8, A, A, accum="double")
    assert np.array_equal(rpc, r[0]) and np.array_equal(cic, r[1])
    assert np.array_equal(vc / num_iter, r[2])


@pytest.mark.parametrize("mb,kb,nb,density", [(64, 64, 64, 0.05), (200, 37, 150, 0.1), (1, 1, 1, 1.0),
                                              (33, 64, 1000, 0.02), (512, 512, 512, 0.01), (10, 10, 40, 0.0),
                                              # dense rows: more products per pass than the list holds,
                                              # B lists beyond the staging capacity, more A tiles than it
                                              (2, 32, 40, 1.0), (2, 32, 100, 1.0), (3, 40, 8, 1.0),
                                              (5, 20, 300, 0.9)])
def test_structure_and_values_exact(cuda, mb, kb, nb, density):
    A = random_bsr(mb, kb, density, 1, integer=True)
    B = random_bsr(kb, nb, density, 2, integer=True)
    rpc, cic, vc = run(A, B, mb, kb, nb)
    r = oracle.spgemm(mb, nb, A, B, accum="double")
    assert np.array_equal(rpc, r[0])
    assert np.array_equal(cic, r[1])
    assert np.array_equal(vc, r[2])


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_values_uniform_tolerance(cuda, dtype):
    mb = kb = nb = 256
    A = random_bsr(mb, kb, 0.03, 3, integer=False)
    B = random_bsr(kb, nb, 0.03, 4, integer=False)
    if dtype == torch.bfloat16:
        A = (A[0], A[1], torch.tensor(A[2].astype(np.float32)).bfloat16().float().numpy())
        B = (B[0], B[1], torch.tensor(B[2].astype(np.float32)).bfloat16().float().numpy())
    rpc, cic, vc = run(A, B, mb, kb, nb, dtype=dtype)
    A64 = (A[0], A[1], np.asarray(A[2], dtype=np.float64))
    B64 = (B[0], B[1], np.asarray(B[2], dtype=np.float64))
    r = oracle.spgemm(mb, nb, (A64[0], A64[1], A64[2].astype(np.float16)) if dtype == torch.float16 else A64,
                      (B64[0], B64[1], B64[2].astype(np.float16)) if dtype == torch.float16 else B64,
                      accum="double") if dtype == torch.float16 else None
    if r is None:
        # bf16 values are not representable as the oracle's binary16 tiles:
        # compare against a dense double product of the same blocks
        return _dense_check(A64, B64, mb, kb, nb, rpc, cic, vc)
    assert np.array_equal(rpc, r[0]) and np.array_equal(cic, r[1])
    assert np.max(np.abs(vc - r[2])) <= 16 * 40 * 2.0 ** -23 * 4


def _dense_check(A, B, mb, kb, nb, rpc, cic, vc):
    def dense(M, rows, cols):
        D = np.zeros((rows * 16, cols * 16))
        for i in range(rows):
            for e in range(M[0][i], M[0][i + 1]):
                j = M[1][e]
                D[i * 16:(i + 1) * 16, j * 16:(j + 1) * 16] = M[2][e]
        return D
    C = dense(A, mb, kb) @ dense(B, kb, nb)
    got = dense((rpc, cic, vc), mb, nb)
    assert np.max(np.abs(C - got)) < 1e-4


def test_empty_operands(cuda):
    A = (np.zeros(5, np.int32), np.zeros(0, np.int32), np.zeros((0, 16, 16), np.float16))
    B = random_bsr(4, 6, 0.5, 7, integer=True)
    rpc, cic, vc = run(A, B, 4, 4, 6)
    assert rpc.tolist() == [0] * 5 and len(cic) == 0


@pytest.mark.parametrize("mb,kb,nb,density", [(64, 64, 64, 0.05), (200, 37, 150, 0.1), (512, 512, 512, 0.01),
                                              (10, 10, 40, 0.0)])
def test_symbolic_device_matches_host_and_numeric_bound(cuda, mb, kb, nb, density):
    """The on-device symbolic pass gives the host pass's RowPtrC / ColIdxC,
    and the numeric pass accepts its capacity as the bound of nnzC."""
    A = random_bsr(mb, kb, density, 1, integer=True)
    B = random_bsr(kb, nb, density, 2, integer=True)
    dA, dB = to_dev(A, kb), to_dev(B, nb)
    rpc_h, nnz = api.spgemm_symbolic(dA, dB)
    cic_h = api.spgemm_fill_colidx(dA, dB, rpc_h, nnz)
    cap = nnz + 37
    rpc, cic = api.spgemm_symbolic_device(dA, dB, cap)
    assert torch.equal(rpc, rpc_h) and int(rpc[-1]) == nnz
    assert torch.equal(cic[:nnz], cic_h)
    vals = torch.full((cap, 16, 16), -7.0, device="cuda")
    api.spgemm_numeric_bound(dA, dB, rpc, cic, vals)
    r = oracle.spgemm(mb, nb, A, B, accum="double")
    assert np.array_equal(vals[:nnz].double().cpu().numpy(), r[2])
    assert bool((vals[nnz:] == -7.0).all())


@pytest.mark.parametrize("mb,kb,nb,density", [(20000, 64, 3000, 0.01), (1, 5, 7, 1.0), (3000, 3000, 40, 0.002),
                                              (50000, 16, 100, 0.05), (140000, 16, 40, 0.02)])
def test_symbolic_device_one_launch_large(cuda, mb, kb, nb, density):
    """The one-launch symbolic pass (count, look-back scan and column fill in
    one cooperative kernel) with many chunks per CTA, a single row, rows
    without entries and -- at 140000 block-rows, past one row per warp in
    16384 chunks -- two rows per warp and chunk, against the oracle's
    structure and the separate count / fill kernels."""
    A = random_bsr(mb, kb, density, 21, integer=True)
    B = random_bsr(kb, nb, min(1.0, density * 10), 22, integer=True)
    dA, dB = to_dev(A, kb), to_dev(B, nb)
    rpc_h, nnz = api.spgemm_symbolic(dA, dB)
    cic_h = api.spgemm_fill_colidx(dA, dB, rpc_h, nnz)
    rpc, cic = api.spgemm_symbolic_device(dA, dB, nnz)
    assert torch.equal(rpc, rpc_h) and torch.equal(cic[:nnz], cic_h)
    # RowPtrC of the oracle's SPA symbolic pass
    rpc_o = oracle.spgemm_row_ptr(mb, nb, A[0], A[1], B[0], B[1])
    assert np.array_equal(rpc.cpu().numpy(), rpc_o)
    from kami_b200 import _lib
    import ctypes
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0


def test_symbolic_device_capacity_respected(cuda):
    A = random_bsr(40, 30, 0.2, 5, integer=True)
    B = random_bsr(30, 50, 0.2, 6, integer=True)
    dA, dB = to_dev(A, 30), to_dev(B, 50)
    rpc_h, nnz = api.spgemm_symbolic(dA, dB)
    cic_h = api.spgemm_fill_colidx(dA, dB, rpc_h, nnz)
    cap = nnz // 2
    cic = torch.full((cap + 16,), -1, dtype=torch.int32, device="cuda")
    rpc = torch.empty(41, dtype=torch.int32, device="cuda")
    from kami_b200 import _lib
    assert _lib.load().kami_spgemm_bsr_symbolic_device(16, 40, 30, 50, dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                                       dB.row_ptr.data_ptr(), dB.col_idx.data_ptr(), rpc.data_ptr(),
                                                       cic.data_ptr(), cap, None) == 0
    assert int(rpc[-1]) == nnz  # the true count, beyond the capacity
    assert torch.equal(cic[:cap], cic_h[:cap]) and bool((cic[cap:] == -1).all())


# ---------------------------------------------------------------------------
# the reference's one-CTA block SpGEMM (kami_spgemm_bsr_block), 1D / 2D / 3D
# ---------------------------------------------------------------------------
BLOCK_PARTS = [("1d", 1), ("1d", 2), ("1d", 4), ("1d", 8), ("2d", 2), ("2d", 4), ("3d", 2)]


def _block_structure(A, B, mb, nb):
    r = oracle.spgemm(mb, nb, A, B, accum="double")
    return r


def _dev_bsr(rp, ci, vals, cols, dtype=torch.float16):
    v = torch.tensor(np.asarray(vals, dtype=np.float32), dtype=dtype, device="cuda")
    return api.BSR(torch.tensor(rp, dtype=torch.int32, device="cuda"),
                   torch.tensor(np.asarray(ci, dtype=np.int32), dtype=torch.int32, device="cuda"), v, cols)


@pytest.mark.parametrize("part,P", BLOCK_PARTS)
@pytest.mark.parametrize("mb,kb,nb,density", [(8, 8, 8, 0.5), (16, 16, 16, 0.3), (5, 12, 7, 0.6), (1, 1, 1, 1.0),
                                              (16, 4, 16, 1.0)])
def test_block_spgemm_partitions_exact(cuda, part, P, mb, kb, nb, density):
    """Every partition of the one-CTA block SpGEMM against the oracle's SPA,
    on integer tiles (exact), one problem per CTA with its own values."""
    batch = 6
    rpa, cia = oracle.bsr_pattern(mb, kb, density, 31)
    rpb, cib = oracle.bsr_pattern(kb, nb, density, 32)
    rng = np.random.default_rng(mb * 100 + nb)
    va = rng.integers(-3, 4, (batch, len(cia), 16, 16)).astype(np.float16)
    vb = rng.integers(-3, 4, (batch, len(cib), 16, 16)).astype(np.float16)
    rpc, cic, _ = oracle.spgemm(mb, nb, (rpa, cia, va[0]), (rpb, cib, vb[0]), accum="double")
    A = _dev_bsr(rpa, cia, va, kb)
    B = _dev_bsr(rpb, cib, vb, nb)
    C = _dev_bsr(rpc, cic, np.full((batch, len(cic), 16, 16), np.nan, np.float32), nb, torch.float32)
    api.spgemm_block(A, B, C, partition=part, P=P)
    got = C.values.double().cpu().numpy()
    for b in range(batch):
        ref = oracle.spgemm(mb, nb, (rpa, cia, va[b]), (rpb, cib, vb[b]), accum="double")[2]
        assert np.array_equal(got[b], ref), b


@pytest.mark.parametrize("part,P", [("1d", 4), ("2d", 2), ("3d", 2)])
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "spgemm_*.npz"))), ids=os.path.basename)
def test_block_spgemm_reference_golden(cuda, part, P, path):
    """The reference's own generator and SPA outputs (binary16 C), reproduced
    by the one-CTA block kernel with the values shared across a batch of
    CTAs and NUM_ITER repeats, as the reference launches it."""
    z = np.load(path)
    m, k, n = (int(x) for x in z["shape"])
    if max(m, k, n) > 16 or len(z["a_col_idx"]) + len(z["b_col_idx"]) > 384:
        pytest.skip("beyond one CTA's block")
    A = _dev_bsr(z["a_row_ptr"], z["a_col_idx"], z["a_vals"], k)
    B = _dev_bsr(z["b_row_ptr"], z["b_col_idx"], z["b_vals"], n)
    nnzc = len(z["c_col_idx"])
    for num_iter in (1, 3):
        C = _dev_bsr(z["c_row_ptr"], z["c_col_idx"], np.zeros((4, max(nnzc, 1), 16, 16), np.float32)[:, :nnzc],
                     n, torch.float16)
        api.spgemm_block(A, B, C, partition=part, P=P, num_iter=num_iter, alpha=1.0 / num_iter)
        got = C.values.cpu().numpy()
        for b in range(4):
            assert np.array_equal(got[b].view(np.uint16), z["c_vals"].view(np.uint16)), (num_iter, b)


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.bfloat16])
def test_block_spgemm_uniform_alpha_beta_num_iter(cuda, dtype, out_dtype):
    mb = kb = nb = 8
    rpa, cia = oracle.bsr_pattern(mb, kb, 0.5, 41)
    rpb, cib = oracle.bsr_pattern(kb, nb, 0.5, 42)
    rng = np.random.default_rng(43)
    va = torch.tensor(rng.uniform(-1, 1, (len(cia), 16, 16)), dtype=dtype).float().numpy()
    vb = torch.tensor(rng.uniform(-1, 1, (len(cib), 16, 16)), dtype=dtype).float().numpy()
    A, B = _dev_bsr(rpa, cia, va, kb, dtype), _dev_bsr(rpb, cib, vb, nb, dtype)
    # the structure, and values in double from the same rounded tiles
    dense = lambda rp, ci, v, r, c: _dense_of(rp, ci, v, r, c)
    Cd = dense(rpa, cia, va, mb, kb) @ dense(rpb, cib, vb, kb, nb)
    rpc, cic, _ = oracle.spgemm(mb, nb, (rpa, cia, np.ones((len(cia), 16, 16), np.float16)),
                                (rpb, cib, np.ones((len(cib), 16, 16), np.float16)))
    C0 = rng.uniform(-1, 1, (3, len(cic), 16, 16)).astype(np.float32)
    C0 = torch.tensor(C0).to(out_dtype).float().numpy()
    C = _dev_bsr(rpc, cic, C0, nb, out_dtype)
    api.spgemm_block(A, B, C, partition="2d", P=2, alpha=0.5, beta=-2.0, num_iter=4)
    got = C.values.double().cpu().numpy()
    ref_tiles = np.stack([Cd[16 * i:16 * i + 16, 16 * j:16 * j + 16]
                          for i in range(mb) for j in cic[rpc[i]:rpc[i + 1]]])
    ref = 0.5 * 4 * ref_tiles[None] - 2.0 * C0.astype(np.float64)
    Cabs = dense(rpa, cia, np.abs(va), mb, kb) @ dense(rpb, cib, np.abs(vb), kb, nb)
    abs_tiles = np.stack([Cabs[16 * i:16 * i + 16, 16 * j:16 * j + 16]
                          for i in range(mb) for j in cic[rpc[i]:rpc[i + 1]]])
    # FP32 accumulation over 4 repeats of at most kb * 16 products, then one
    # rounding to the output type
    u_out = 2.0 ** -8 if out_dtype == torch.bfloat16 else 2.0 ** -24
    tol = (4 * kb * 16 + 4) * 2.0 ** -23 * 2 * abs_tiles[None] + u_out * np.abs(ref) * 1.01
    assert np.all(np.abs(got - ref) <= tol)


def _dense_of(rp, ci, v, rows, cols):
    D = np.zeros((rows * 16, cols * 16))
    for i in range(rows):
        for e in range(rp[i], rp[i + 1]):
            D[16 * i:16 * i + 16, 16 * ci[e]:16 * ci[e] + 16] = v[e]
    return D


def test_block_spgemm_rejects_large(cuda):
    A = random_bsr(17, 4, 0.5, 1, integer=True)
    dA = to_dev(A, 4)
    dB = to_dev(random_bsr(4, 4, 0.5, 2, integer=True), 4)
    C = api.BSR(dA.row_ptr, dA.col_idx, torch.zeros((1, 16, 16), device="cuda"), 4)
    from kami_b200._lib import KamiError
    with pytest.raises(KamiError, match="exceed"):
        api.spgemm_block(dA, dB, C)


# ---------------------------------------------------------------------------
# the tcgen05 numeric kernel (kami_spgemm_bsr_numeric_variant, TCGEN05)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("variant", ["mma_sync", "tcgen05"])
@pytest.mark.parametrize("mb,kb,nb,density", [(64, 64, 64, 0.05), (200, 37, 150, 0.1), (1, 1, 1, 1.0),
                                              (33, 64, 1000, 0.02), (512, 512, 512, 0.01), (10, 10, 40, 0.0),
                                              # rows of more than one 64-tile unit, more A entries than
                                              # one enumeration chunk, more C columns than staged
                                              (3, 300, 200, 1.0), (4, 40, 2100, 0.9), (300, 8, 70, 0.5)])
def test_numeric_variants_exact(cuda, variant, mb, kb, nb, density):
    A = random_bsr(mb, kb, density, 5, integer=True)
    B = random_bsr(kb, nb, density, 6, integer=True)
    rpc, cic, vc = run(A, B, mb, kb, nb, variant=variant)
    r = oracle.spgemm(mb, nb, A, B, accum="double")
    assert np.array_equal(rpc, r[0]) and np.array_equal(cic, r[1])
    assert np.array_equal(vc, r[2])
    from kami_b200 import _lib
    import ctypes
    code = ctypes.c_int(0)
    assert _lib.load().kami_device_status(ctypes.byref(code)) == 0 and code.value == 0


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16, torch.bfloat16])
def test_numeric_tcgen05_alpha_beta_num_iter_out_types(cuda, dtype, out_dtype):
    mb = kb = nb = 96
    A = random_bsr(mb, kb, 0.05, 7, integer=True)
    B = random_bsr(kb, nb, 0.05, 8, integer=True)
    dA, dB = to_dev(A, kb, dtype), to_dev(B, nb, dtype)
    rpc, nnz = api.spgemm_symbolic(dA, dB)
    cic = api.spgemm_fill_colidx(dA, dB, rpc, nnz)
    r = oracle.spgemm(mb, nb, A, B, accum="double")
    C0 = np.random.default_rng(9).integers(-4, 5, (nnz, 16, 16)).astype(np.float64)
    vals = {}
    for variant in ("mma_sync", "tcgen05"):
        Cv = torch.tensor(C0, dtype=out_dtype, device="cuda")
        api.spgemm_numeric(dA, dB, rpc, cic, C_values=Cv, alpha=0.5, beta=2.0, num_iter=3, variant=variant)
        vals[variant] = Cv.double().cpu().numpy()
    ref = torch.tensor(0.5 * 3 * r[2] + 2.0 * C0, dtype=torch.float32).to(out_dtype).double().numpy()
    assert np.array_equal(vals["mma_sync"], ref)
    assert np.array_equal(vals["tcgen05"], ref)


def test_numeric_tcgen05_capacity_bound_untouched(cuda):
    """Tiles past row_ptr_c[mb] (a capacity larger than nnzC) stay untouched."""
    A = random_bsr(100, 100, 0.05, 11, integer=True)
    B = random_bsr(100, 100, 0.05, 12, integer=True)
    dA, dB = to_dev(A, 100), to_dev(B, 100)
    rpc_h, nnz = api.spgemm_symbolic(dA, dB)
    cap = nnz + 29
    rpc, cic = api.spgemm_symbolic_device(dA, dB, cap)
    vals = torch.full((cap, 16, 16), -7.0, device="cuda")
    api.spgemm_numeric_bound(dA, dB, rpc, cic, vals, variant="tcgen05")
    r = oracle.spgemm(100, 100, A, B, accum="double")
    assert np.array_equal(vals[:nnz].double().cpu().numpy(), r[2])
    assert bool((vals[nnz:] == -7.0).all())
