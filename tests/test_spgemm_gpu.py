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


def run(A, B, mb, kb, nb, out_dtype=torch.float32, num_iter=1, dtype=torch.float16):
    dA, dB = to_dev(A, kb, dtype), to_dev(B, nb, dtype)
    C = api.spgemm(dA, dB, out_dtype, num_iter=num_iter)
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
                                              (50000, 16, 100, 0.05)])
def test_symbolic_device_one_launch_large(cuda, mb, kb, nb, density):
    """The one-launch symbolic pass (count, scan, column fill as phases of a
    cooperative kernel) with many block-rows per CTA, a single row, and rows
    without entries, against the oracle's structure and the separate
    count / fill kernels."""
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
