"""Parity of the tcgen05 (TMEM / TMA) block GEMM with the CPU oracle,
through the C ABI, for the three partition mappings, FP16 and BF16, the
output types, ragged shapes and the in-register repeat count."""
import numpy as np
import pytest
import torch

import oracle
from kami_b200 import _lib, api
from kami_b200._lib import KamiError

pytestmark = pytest.mark.gpu

TDT = {"f16": torch.float16, "bf16": torch.bfloat16}


def _inputs(prec, batch, M, N, K, integer, seed=0):
    rng = np.random.default_rng(seed)
    if integer:
        A = rng.integers(-2, 3, (batch, M, K)).astype(np.float64)
        B = rng.integers(-2, 3, (batch, N, K)).astype(np.float64)
    else:
        A = rng.uniform(-1, 1, (batch, M, K))
        B = rng.uniform(-1, 1, (batch, N, K))
    tA = torch.tensor(A, dtype=TDT[prec])
    tB = torch.tensor(B, dtype=TDT[prec])
    return tA.cuda(), tB.cuda(), tA.double().numpy(), tB.double().numpy()


def _status_clean():
    code = __import__("ctypes").c_int(0)
    st = _lib.load().kami_device_status(code)
    assert st == 0 and code.value == 0


SHAPES = [(128, 128, 128), (64, 64, 64), (128, 128, 16), (128, 128, 32), (128, 128, 8), (128, 256, 128),
          (64, 256, 64), (100, 72, 40), (128, 16, 64), (33, 48, 24), (128, 128, 256), (96, 200, 136)]


@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("M,N,K", SHAPES)
def test_tc05_1d_exact(cuda, prec, M, N, K):
    A, B, A64, B64 = _inputs(prec, 7, M, N, K, integer=True, seed=M + N + K)
    C = api.gemm_batched(A, B, variant="tcgen05", partition="1d")
    torch.cuda.synchronize()
    _status_clean()
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A64, B64))


@pytest.mark.parametrize("part,P", [("2d", 2), ("2d", 4), ("3d", 2), ("3d", 4)])
@pytest.mark.parametrize("M,N,K", [(128, 128, 128), (64, 64, 64), (128, 256, 64), (100, 72, 80)])
def test_tc05_partitions_exact(cuda, part, P, M, N, K):
    if part == "3d" and (K + 15) // 16 < P:
        pytest.skip("fewer k-steps than depth ranks")
    if part == "3d" and P * ((N + 15) // 16 * 16) > 512:
        pytest.skip("P accumulators of N columns exceed the 512 TMEM columns")
    A, B, A64, B64 = _inputs("f16", 5, M, N, K, integer=True, seed=P)
    C = api.gemm_batched(A, B, variant="tcgen05", partition=part, P=P)
    torch.cuda.synchronize()
    _status_clean()
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A64, B64))


@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("M,N,K", [(128, 128, 128), (64, 64, 64), (128, 128, 32)])
def test_tc05_uniform_tolerance(cuda, prec, M, N, K):
    A, B, A64, B64 = _inputs(prec, 9, M, N, K, integer=False, seed=11)
    C = api.gemm_batched(A, B, variant="tcgen05").double().cpu().numpy()
    ref = oracle.gemm(A64, B64)
    bound = (K + 2) * 2.0 ** -23 * (np.abs(A64) @ np.abs(B64).transpose(0, 2, 1))
    assert np.all(np.abs(C - ref) <= bound)
    assert np.linalg.norm(C - ref) / np.linalg.norm(ref) < 2e-6


@pytest.mark.parametrize("num_iter", [1, 3, 1000])
def test_tc05_num_iter(cuda, num_iter):
    A, B, A64, B64 = _inputs("f16", 4, 128, 128, 128, integer=True, seed=num_iter)
    C = api.gemm_batched(A, B, variant="tcgen05", num_iter=num_iter)
    ref = oracle.gemm(A64, B64) * num_iter
    # integer sums stay below 2^24, so FP32 accumulation is exact
    assert np.array_equal(C.double().cpu().numpy(), ref)


def test_tc05_out_types_alpha_beta(cuda):
    A, B, A64, B64 = _inputs("f16", 3, 128, 128, 64, integer=True, seed=2)
    ref = oracle.gemm(A64, B64)
    for odt in (torch.float16, torch.bfloat16):
        C = api.gemm_batched(A, B, variant="tcgen05", out_dtype=odt)
        assert np.array_equal(C.double().cpu().numpy(), torch.tensor(ref).to(odt).double().numpy())
    C0 = torch.full((3, 128, 128), 1.0, device="cuda")
    api.gemm_batched(A, B, C0, variant="tcgen05", alpha=2.0, beta=-1.0)
    assert np.array_equal(C0.double().cpu().numpy(), 2 * ref - 1)


def test_tc05_matches_mma_sync_large_batch(cuda):
    A, B, _, _ = _inputs("bf16", 4096, 64, 64, 64, integer=False, seed=5)
    C1 = api.gemm_batched(A, B, variant="tcgen05")
    C2 = api.gemm_batched(A, B, variant="mma_sync")
    assert torch.allclose(C1, C2, rtol=0, atol=1e-5)


def test_tc05_rejects_what_it_cannot_do(cuda):
    A = torch.zeros((2, 256, 64), dtype=torch.float16, device="cuda")
    with pytest.raises(KamiError):
        api.gemm_batched(A, A, variant="tcgen05")
    A = torch.zeros((2, 64, 60), dtype=torch.float16, device="cuda")  # K % 8 != 0: TMA rows misaligned
    with pytest.raises(KamiError):
        api.gemm_batched(A, A, variant="tcgen05")
    A = torch.zeros((2, 64, 64), dtype=torch.float64, device="cuda")  # FP64 has no tcgen05 kind
    with pytest.raises(KamiError):
        api.gemm_batched(A, A, variant="tcgen05")


def test_auto_picks_tcgen05_for_128(cuda):
    assert api.describe(128, 128, 128, 592)["variant"] == "tcgen05"
    A, B, A64, B64 = _inputs("f16", 8, 128, 128, 128, integer=True)
    assert np.array_equal(api.gemm_batched(A, B).double().cpu().numpy(), oracle.gemm(A64, B64))


@pytest.mark.parametrize("a_layout,b_layout", [("col_mk", "ref_nk"), ("row_mk", "row_kn"), ("col_mk", "row_kn")])
@pytest.mark.parametrize("M,N,K", [(128, 128, 128), (64, 64, 64), (104, 72, 40), (128, 256, 64), (64, 48, 136)])
def test_tc05_mn_major_layouts(cuda, a_layout, b_layout, M, N, K):
    """MN-major operands (A stored K x M, B stored K x N) staged by TMA in
    64-element swizzle boxes: the layouts of the backward pass."""
    rng = np.random.default_rng(M + 3 * N + 7 * K)
    A64 = rng.integers(-2, 3, (5, M, K)).astype(np.float64)
    B64 = rng.integers(-2, 3, (5, N, K)).astype(np.float64)
    A = torch.tensor(A64 if a_layout == "row_mk" else A64.transpose(0, 2, 1).copy(), dtype=torch.float16).cuda()
    B = torch.tensor(B64 if b_layout == "ref_nk" else B64.transpose(0, 2, 1).copy(), dtype=torch.float16).cuda()
    C = api.gemm_batched(A, B, a_layout=a_layout, b_layout=b_layout, variant="tcgen05")
    torch.cuda.synchronize()
    _status_clean()
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A64, B64))


@pytest.mark.parametrize("part,P", [("1d", 0), ("2d", 2), ("3d", 2)])
@pytest.mark.parametrize("M,N,K", [(128, 128, 128), (100, 72, 40), (128, 256, 64), (80, 128, 256), (128, 16, 8)])
@pytest.mark.parametrize("prec", ["f16", "bf16"])
def test_tc05_a_in_tmem(cuda, part, P, M, N, K, prec):
    """The TS form: A staged into tensor memory with tcgen05.st, B by TMA."""
    if part == "3d" and ((K + 15) // 16 < P or P * ((N + 15) // 16 * 16) + (K + 15) // 16 * 8 > 512):
        pytest.skip("does not fit")
    if part == "2d" and N % (16 * P):
        pytest.skip("2D panels")
    A, B, A64, B64 = _inputs(prec, 6, M, N, K, integer=True, seed=M + N + K + P)
    C = api.gemm_batched(A, B, variant="tcgen05_ts", partition=part, P=P)
    torch.cuda.synchronize()
    _status_clean()
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A64, B64))


def test_tc05_a_in_tmem_num_iter(cuda):
    A, B, A64, B64 = _inputs("f16", 4, 128, 128, 128, integer=True, seed=9)
    C = api.gemm_batched(A, B, variant="tcgen05_ts", num_iter=1000)
    assert np.array_equal(C.double().cpu().numpy(), oracle.gemm(A64, B64) * 1000)


@pytest.mark.parametrize("odt", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("M,N,K,batch", [(128, 128, 128, 600), (100, 128, 128, 300), (128, 120, 128, 300),
                                         (128, 192, 64, 200), (128, 96, 128, 300), (128, 100, 128, 150),
                                         (128, 128, 128, 1), (64, 128, 256, 300), (64, 64, 64, 1000),
                                         (128, 64, 64, 500), (64, 128, 64, 500), (56, 64, 64, 333),
                                         (128, 96, 64, 300), (128, 112, 64, 300)])
def test_tc05_streamed_store_paths(cuda, odt, M, N, K, batch):
    """The persistent streaming form (problems of at least 32 KB of operands,
    and 16-32 KB ones with two MMA issuers: 64^3, 128 x 64 x 64, 64 x 128 x
    64; 128 x 96 and 128 x 112 fall back to one CTA per problem) over its two
    C paths: bulk tensor stores of 128-byte boxes when C rows and problems
    are 16-byte aligned and the padded N is a whole number of boxes,
    per-thread stores otherwise (here N = 100 with 16-bit C, N = 96 with
    16-bit C).  C is a column slice of a wider buffer, so rows are padded:
    the padding must stay untouched and row tails clipped."""
    rng = np.random.default_rng(M * N + K + batch)
    A64 = rng.integers(-2, 3, (batch, M, K)).astype(np.float64)
    B64 = rng.integers(-2, 3, (batch, N, K)).astype(np.float64)
    A = torch.tensor(A64, dtype=torch.float16).cuda()
    B = torch.tensor(B64, dtype=torch.float16).cuda()
    ldc = N + 8
    big = torch.full((batch, M, ldc), 7.0, dtype=odt, device="cuda")
    C = big[:, :, :N]
    api.gemm_batched(A, B, C, variant="tcgen05")
    torch.cuda.synchronize()
    _status_clean()
    ref = oracle.gemm(A64, B64)
    assert np.array_equal(C.double().cpu().numpy(), torch.tensor(ref).to(odt).double().numpy())
    assert bool((big[:, :, N:] == 7.0).all())
    # contiguous C as well
    C2 = api.gemm_batched(A, B, variant="tcgen05", out_dtype=odt if odt != torch.float32 else None)
    assert np.array_equal(C2.double().cpu().numpy(), torch.tensor(ref).to(odt).double().numpy())


@pytest.mark.parametrize("odt", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("M,N,K,num_iter,part,P", [(128, 64, 64, 5, "1d", 0), (100, 64, 64, 5, "1d", 0),
                                                   (128, 96, 64, 1, "1d", 0), (64, 128, 64, 5, "1d", 0),
                                                   (50, 120, 32, 5, "1d", 0), (64, 48, 64, 1, "1d", 0),
                                                   (128, 128, 128, 8, "1d", 0),
                                                   (128, 128, 128, 1, "2d", 2), (128, 128, 64, 1, "3d", 2),
                                                   (64, 64, 64, 1, "3d", 4)])
def test_tc05_per_problem_store_paths(cuda, odt, M, N, K, num_iter, part, P):
    """The one-CTA-per-problem form (problems under 16 KB of operands or
    without a two-issuer streaming layout, the repeated-product mode beyond 4
    repeats, the 2D / 3D mappings) over its two C paths:
    bulk tensor stores staged in the dead operand tiles, or per-thread
    stores.  C rows are padded; the padding must stay untouched."""
    batch = 37
    rng = np.random.default_rng(M + 7 * N + K + num_iter)
    A64 = rng.integers(-2, 3, (batch, M, K)).astype(np.float64)
    B64 = rng.integers(-2, 3, (batch, N, K)).astype(np.float64)
    A = torch.tensor(A64, dtype=torch.float16).cuda()
    B = torch.tensor(B64, dtype=torch.float16).cuda()
    big = torch.full((batch, M, N + 8), 7.0, dtype=odt, device="cuda")
    C = big[:, :, :N]
    api.gemm_batched(A, B, C, variant="tcgen05", partition=part, P=P, num_iter=num_iter)
    torch.cuda.synchronize()
    _status_clean()
    ref = oracle.gemm(A64, B64) * num_iter
    assert np.array_equal(C.double().cpu().numpy(), torch.tensor(ref).to(odt).double().numpy())
    assert bool((big[:, :, N:] == 7.0).all())


@pytest.mark.parametrize("M,N,K", [(64, 256, 64), (128, 192, 64), (64, 64, 64), (128, 160, 64)])
def test_tc05_streamed_alpha_beta_many_per_cta(cuda, M, N, K):
    """alpha / beta (per-thread stores) with many problems per CTA in the
    streaming form, where wide N leaves few TMEM accumulators (2 for N >
    170): every epilogue group must drain an accumulator only after the
    product it waits for is complete."""
    batch = 900
    rng = np.random.default_rng(N + K)
    A64 = rng.integers(-2, 3, (batch, M, K)).astype(np.float64)
    B64 = rng.integers(-2, 3, (batch, N, K)).astype(np.float64)
    C64 = rng.integers(-3, 4, (batch, M, N)).astype(np.float64)
    A = torch.tensor(A64, dtype=torch.bfloat16).cuda()
    B = torch.tensor(B64, dtype=torch.bfloat16).cuda()
    C = torch.tensor(C64, dtype=torch.float32).cuda()
    api.gemm_batched(A, B, C, variant="tcgen05", alpha=2.0, beta=-1.0)
    torch.cuda.synchronize()
    _status_clean()
    assert np.array_equal(C.double().cpu().numpy(), 2 * oracle.gemm(A64, B64) - C64)


@pytest.mark.parametrize("K", [64, 32, 128, 40])
@pytest.mark.parametrize("batch", [2, 9, 1201])
@pytest.mark.parametrize("a_layout,b_layout", [("row_mk", "ref_nk"), ("row_mk", "row_kn"), ("col_mk", "row_kn")])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.bfloat16])
def test_tc05_stream_pairs_exact(cuda, K, batch, a_layout, b_layout, out_dtype):
    """Streamed 64 x 64 problems run two to a unit (one 128 x 128 MMA chain,
    C on the accumulator's diagonal): odd batches (a last unit of one problem),
    K of one, a partial and two K boxes, every operand layout; exact on
    integer inputs."""
    rng = np.random.default_rng(batch + K)
    A = rng.integers(-2, 3, (batch, 64, K)).astype(np.float64)
    Bt = rng.integers(-2, 3, (batch, K, 64)).astype(np.float64)  # K x N
    tA = torch.tensor(A, dtype=torch.bfloat16)
    tA = (tA if a_layout == "row_mk" else tA.transpose(1, 2).contiguous()).cuda()
    tB = torch.tensor(Bt, dtype=torch.bfloat16)
    tB = (tB.transpose(1, 2).contiguous() if b_layout == "ref_nk" else tB).cuda()
    C = api.gemm_batched(tA, tB, a_layout=a_layout, b_layout=b_layout, out_dtype=out_dtype)
    torch.cuda.synchronize()
    _status_clean()
    ref = np.matmul(A, Bt)
    assert np.array_equal(C.double().cpu().numpy(), torch.tensor(ref).to(out_dtype).double().numpy())
