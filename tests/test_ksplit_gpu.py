"""The register / shared-memory K split of the 1D mma.sync block GEMM and the
traced (communication / computation cycle) instances, through the C ABI,
against the CPU oracle: exact on integer-valued inputs for every compiled
split, shape edges, alpha / beta and output types, the measured choice of
split, and the trace's cycle counts."""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import api
from kami_b200._lib import KamiError

pytestmark = pytest.mark.gpu

# (tile, P, register k-steps) of the compiled splits; k-steps = tile / 16
SPLITS = [(128, 4, 0), (128, 4, 2), (128, 4, 4), (128, 8, 0), (128, 8, 4), (128, 8, 8), (64, 2, 0), (64, 2, 2),
          (64, 2, 4), (64, 4, 0), (64, 4, 2), (64, 4, 4)]


def ints(shape, seed, lo=-2, hi=3):
    return np.random.default_rng(seed).integers(lo, hi, shape).astype(np.float64)


@pytest.mark.parametrize("tile,P,rk", SPLITS)
@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_split_exact(cuda, tile, P, rk, dtype):
    batch = 300
    A = ints((batch, tile, tile), tile + P + rk)
    B = ints((batch, tile, tile), tile * P + rk + 1)
    C, used = api.gemm_batched_ksplit(torch.tensor(A, dtype=dtype, device="cuda"),
                                      torch.tensor(B, dtype=dtype, device="cuda"), P=P, reg_k_steps=rk)
    assert used == rk
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A, B))


@pytest.mark.parametrize("M,N,K,P,rk", [(100, 90, 120, 4, 2), (65, 128, 72, 4, 0), (33, 17, 40, 2, 2),
                                        (64, 64, 8, 4, 0), (1, 1, 16, 2, 0), (128, 1, 128, 8, 4)])
def test_split_edges_alpha_beta(cuda, M, N, K, P, rk):
    """Shapes below the tile (zero-filled loads, masked stores), K not a
    multiple of the k-step, alpha / beta, the repeats of num_iter."""
    batch = 150
    A = ints((batch, M, K), M + N)
    B = ints((batch, N, K), K + 7)
    C0 = ints((batch, M, N), 3)
    dC = torch.tensor(C0, dtype=torch.float32, device="cuda")
    api.gemm_batched_ksplit(torch.tensor(A, dtype=torch.float16, device="cuda"),
                            torch.tensor(B, dtype=torch.float16, device="cuda"), dC, P=P, reg_k_steps=rk,
                            num_iter=3, alpha=2.0, beta=-1.0)
    assert np.array_equal(dC.double().cpu().numpy(), 2.0 * 3 * oracle.gemm(A, B) - C0)


@pytest.mark.parametrize("out_dtype", [torch.float16, torch.bfloat16])
def test_split_out_types(cuda, out_dtype):
    A = ints((64, 128, 128), 5, -1, 2)
    B = ints((64, 128, 128), 6, -1, 2)
    C, _ = api.gemm_batched_ksplit(torch.tensor(A, dtype=torch.float16, device="cuda"),
                                   torch.tensor(B, dtype=torch.float16, device="cuda"), P=4, reg_k_steps=2,
                                   out_dtype=out_dtype)
    ref = torch.tensor(oracle.gemm(A, B), dtype=torch.float32).to(out_dtype).double().numpy()
    assert C.dtype == out_dtype and np.array_equal(C.double().cpu().numpy(), ref)


@pytest.mark.parametrize("P", [0, 4])
def test_split_measured_choice(cuda, P):
    A = ints((600, 128, 128), 8)
    B = ints((600, 128, 128), 9)
    dC = torch.full((600, 128, 128), 5.0, device="cuda")
    C, used = api.gemm_batched_ksplit(torch.tensor(A, dtype=torch.float16, device="cuda"),
                                      torch.tensor(B, dtype=torch.float16, device="cuda"), dC, P=P, reg_k_steps=-1,
                                      num_iter=10)
    allowed = {rk for (t, p, rk) in SPLITS if t == 128 and (P == 0 or p == P)}
    assert used in allowed
    assert np.array_equal(dC.double().cpu().numpy(), 10 * oracle.gemm(A, B))


def test_split_rejects(cuda):
    A = torch.zeros((4, 128, 128), dtype=torch.float16, device="cuda")
    with pytest.raises(KamiError):
        api.gemm_batched_ksplit(A, A, P=4, reg_k_steps=8)  # the all-register 1D 128^3 P=4 form is not compiled
    with pytest.raises(KamiError):
        api.gemm_batched_ksplit(A, A, P=3, reg_k_steps=0)
    with pytest.raises(KamiError):
        api.gemm_batched_ksplit(torch.zeros((4, 200, 16), dtype=torch.float16, device="cuda"),
                                torch.zeros((4, 8, 16), dtype=torch.float16, device="cuda"), P=4, reg_k_steps=0)


@pytest.mark.parametrize("partition,n,P,rk", [("1d", 128, 8, -1), ("2d", 128, 4, -1), ("3d", 128, 2, -1),
                                              ("1d", 64, 2, -1), ("1d", 64, 4, -1), ("2d", 64, 2, -1),
                                              ("3d", 64, 2, -1), ("1d", 128, 4, 4), ("1d", 128, 4, 0),
                                              ("1d", 128, 8, 4)])
def test_trace(cuda, partition, n, P, rk):
    A = ints((n, n), n + P)
    B = ints((n, n), n * P)
    C, cyc = api.gemm_trace(torch.tensor(A, dtype=torch.float16, device="cuda"),
                            torch.tensor(B, dtype=torch.float16, device="cuda"), partition=partition, P=P,
                            reg_k_steps=rk, num_iter=4)
    assert np.array_equal(C.double().cpu().numpy(), 4 * oracle.gemm(A[None], B[None])[0])
    nw = {"1d": P, "2d": P * P, "3d": P ** 3}[partition]
    assert cyc.shape == (nw, 2)
    assert np.all(cyc[:, 1] > 0)  # every warp computes
    assert np.all(cyc[:, 0] > 0)  # and communicates (publishes or waits)
