"""The C ABI library: it loads, exports every function include/kami.h
declares, and validates arguments on the host (no GPU needed; nothing here
launches a kernel)."""
import ctypes
import os
import re

import pytest

from kami_b200 import _lib, api
from kami_b200._lib import KamiError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(kami_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_loads():
    L = _lib.load()
    assert L.kami_version() >= 100


def test_every_declared_symbol_is_exported():
    L = _lib.load()
    names = declared_functions()
    assert "kami_gemm_batched" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python signature table covers them all
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def _call(**kw):
    a = dict(in_type=_lib.F16, out_type=_lib.F32, part=0, var=0, M=64, N=64, K=64, P=0, alloc=0, batch=1,
             A=16, lda=64, sA=4096, al=0, B=16, ldb=64, sB=4096, bl=0, C=16, ldc=64, sC=4096,
             alpha=1.0, beta=0.0, it=1)
    a.update(kw)
    return _lib.load().kami_gemm_batched(a["in_type"], a["out_type"], a["part"], a["var"], a["M"], a["N"], a["K"],
                                         a["P"], a["alloc"], a["batch"], a["A"], a["lda"], a["sA"], a["al"],
                                         a["B"], a["ldb"], a["sB"], a["bl"], a["C"], a["ldc"], a["sC"],
                                         a["alpha"], a["beta"], a["it"], None, 0, None)


@pytest.mark.parametrize("kw,status", [
    (dict(batch=0), 0),
    (dict(M=0), -1),
    (dict(in_type=7), -1),
    (dict(in_type=_lib.F64, out_type=_lib.F32), -2),
    (dict(K=30, lda=30, ldb=30), -2),
    (dict(A=None), -1),
    (dict(A=18), -3),
    (dict(lda=63), -1),
    (dict(it=0), -1),
    (dict(al=5), -1),
])
def test_host_validation(kw, status):
    assert _call(**kw) == status
    if status:
        assert _lib.load().kami_last_error_string()


def test_describe_is_host_only():
    from kami_b200 import api
    import torch
    d = api.describe(128, 128, 128, 592, torch.float16, variant="mma_sync", partition="2d")
    assert d["variant"] == "mma_sync" and d["partition"] == "2d" and d["P"] == 4
    assert d["threads"] == 512 and d["grid"] == 592
    d = api.describe(32, 32, 32, 1024, torch.float64, partition="2d", P=2)
    assert d["threads"] == 128 and d["problems_per_cta"] == 1
    d = api.describe(16, 16, 16, 1000, torch.float16, partition="1d", variant="mma_sync")
    assert d["problems_per_cta"] == 4 and d["grid"] == 250
    with pytest.raises(KamiError):
        api.describe(200, 200, 200, 1, torch.float16, variant="mma_sync")


def _spmm(**kw):
    a = dict(it=_lib.F16, ot=_lib.F32, bsr=16, mb=4, kb=4, N=64, batch=1, rp=16, ci=16, srp=0, sci=0, v=16, sv=0,
             B=16, ldb=64, sB=0, bl=0, C=16, ldc=64, sC=0, alpha=1.0, beta=0.0, iters=1)
    a.update(kw)
    return _lib.load().kami_spmm_bsr(a["it"], a["ot"], a["bsr"], a["mb"], a["kb"], a["N"], a["batch"], a["rp"],
                                     a["ci"], a["srp"], a["sci"], a["v"], a["sv"], a["B"], a["ldb"], a["sB"],
                                     a["bl"], a["C"], a["ldc"], a["sC"], a["alpha"], a["beta"], a["iters"], None)


@pytest.mark.parametrize("kw,status", [
    (dict(batch=0), 0),
    (dict(N=0), 0),
    (dict(bsr=32), -2),
    (dict(it=_lib.F64), -2),
    (dict(ot=_lib.F64), -2),
    (dict(kb=0), -1),
    (dict(iters=0), -1),
    (dict(v=None), -1),
    (dict(v=18), -3),
    (dict(ldb=63), -1),
    (dict(bl=1, ldb=32), -1),
    (dict(ldc=8), -1),
])
def test_spmm_host_validation(kw, status):
    """Rejected before any launch (no GPU needed)."""
    assert _spmm(**kw) == status


def test_bsr_to_tilebsr_host_conversion():
    import numpy as np
    rp = np.array([0, 2, 3, 3, 5], dtype=np.int32)
    ci = np.array([0, 3, 2, 1, 2], dtype=np.int32)
    brp, bci, perm = api.bsr_to_tilebsr(rp, ci, 4, 2, 2)
    # row tile 0 (rows 0, 1): column tile 0 holds (0,0); tile 1 holds (0,3), (1,2)
    assert brp.tolist() == [0, 1, 1, 2, 3, 3, 4, 4, 5]
    assert bci.tolist() == [0, 1, 0, 1, 0]
    assert perm.tolist() == [0, 1, 2, 3, 4]
    with pytest.raises(Exception):
        api.bsr_to_tilebsr(rp, ci, 4, 3, 2)


@pytest.mark.parametrize("case", ["dims", "dtype", "mixed", "strided", "shape", "host"])
def test_bmm_forward_argument_checks(case):
    """api.bmm_forward (the autograd forward's launch) rejects what it cannot
    pass to kami_gemm_batched unchanged -- before any device work."""
    import torch
    A = torch.zeros((2, 8, 16), dtype=torch.float16)
    B = torch.zeros((2, 16, 8), dtype=torch.float16)
    if case == "dims":
        A = A[0]
    elif case == "dtype":
        A, B = A.float(), B.float()
    elif case == "mixed":
        B = B.bfloat16()
    elif case == "strided":
        A = torch.zeros((2, 16, 8), dtype=torch.float16).transpose(1, 2)
    elif case == "shape":
        B = torch.zeros((2, 12, 8), dtype=torch.float16)
    with pytest.raises((ValueError, TypeError)):
        api.bmm_forward(A, B)


@pytest.mark.parametrize("kw,status", [
    (dict(in_type=_lib.F32), -1),                         # FP32 inputs have no kernel
    (dict(out_type=_lib.F64), -2),                        # FP64 out only for FP64 in
    (dict(in_type=_lib.F64, out_type=_lib.F32), -2),
    (dict(M=0), -1),
    (dict(batch=-1), -1),
    (dict(A=None), -1),
    (dict(dC=None), -1),
    (dict(dA=None, dB=None), 0),                          # nothing asked: no work, no device call
    (dict(batch=0), 0),
])
def test_backward_host_validation(kw, status):
    """kami_gemm_backward_batched checks its request on the host before any
    device work (these calls need no GPU)."""
    a = dict(in_type=_lib.BF16, out_type=_lib.BF16, M=64, N=64, K=64, batch=4, A=16, B=16, dC=16, dA=16, dB=16)
    a.update(kw)
    st = _lib.load().kami_gemm_backward_batched(a["in_type"], a["out_type"], a["M"], a["N"], a["K"], a["batch"],
                                                a["A"], a["B"], a["dC"], a["dA"], a["dB"], None)
    assert st == status
    if status:
        assert _lib.load().kami_last_error_string()


@pytest.mark.parametrize("kw,status", [
    (dict(M=0), -1),
    (dict(batch=-1), -1),
    (dict(it=0), -1),
    (dict(A=None), -1),
    (dict(batch=0), 0),
])
def test_host_buffer_gemm_validation(kw, status):
    """kami_gemm_batched_host rejects bad requests before touching the device;
    an empty batch is a no-op."""
    a = dict(M=64, N=64, K=64, batch=4, A=16, B=16, C=16, it=1)
    a.update(kw)
    st = _lib.load().kami_gemm_batched_host(_lib.F16, _lib.F32, 0, 0, a["M"], a["N"], a["K"], a["batch"], a["A"],
                                            a["B"], a["C"], a["it"], None, 0, None)
    assert st == status


@pytest.mark.parametrize("batch,expect", [
    # 16 chunks of 37 problems, one buffer each: the whole batch's A, B, C
    (592, 592 * (128 * 128 * 2 * 2 + 128 * 128 * 4)),
    # one chunk
    (1, 128 * 128 * 2 * 2 + 128 * 128 * 4),
    # 16 chunks of 6250 problems would need 13 GB: a ring of two buffers
    (100000, 2 * 6250 * (128 * 128 * 2 * 2 + 128 * 128 * 4)),
])
def test_host_buffer_gemm_workspace_size(batch, expect):
    """The host-buffer GEMM's chunking, through the size it reports (no GPU
    needed; 148 SMs assumed when none answers, as on a B200): chunks of about
    one problem per four SMs, at most 16, each with its own device buffer
    unless all of them would exceed 1 GiB."""
    need = ctypes.c_size_t(0)
    L = _lib.load()
    assert L.kami_gemm_batched_host_workspace_size(_lib.F16, _lib.F32, 128, 128, 128, batch, ctypes.byref(need)) == 0
    assert need.value == expect
    assert L.kami_gemm_batched_host_workspace_size(_lib.F16, _lib.F32, 0, 128, 128, batch, ctypes.byref(need)) != 0


class _FakeCuda:
    """Stands for a CUDA tensor on a given device (no GPU needed)."""

    def __init__(self, index):
        import torch
        self.is_cuda = True
        self.device = torch.device("cuda", index)


def test_operands_on_different_devices_are_rejected():
    assert api._device_index(_FakeCuda(0), None, _FakeCuda(0)) == 0
    assert api._device_index(_FakeCuda(3)) == 3
    with pytest.raises(ValueError, match="different devices"):
        api._device_index(_FakeCuda(0), _FakeCuda(1))
    with pytest.raises(ValueError, match="different devices"):
        api._device_index(_FakeCuda(1), None, _FakeCuda(1), _FakeCuda(0))


def test_host_tensors_are_rejected_before_any_launch():
    import torch
    A = torch.zeros((2, 16, 16), dtype=torch.float16)
    with pytest.raises(ValueError, match="CUDA tensors"):
        api.gemm_batched(A, A)
    with pytest.raises(ValueError, match="CUDA tensors"):
        api.split_f64_gemm(A.double(), A.double())
    with pytest.raises(ValueError, match="CUDA tensors"):
        api._device_index(_FakeCuda(0), A)


def test_torch_operator_registers_without_gpu():
    """torch.ops.kami.bmm (the C++ autograd operator) loads, has the
    torch.bmm schema, and refuses host tensors (CUDA kernel only)."""
    import torch
    from kami_b200 import autograd
    if not autograd.ops_available():
        pytest.skip("libkami_torch_ops.so not built")
    assert str(torch.ops.kami.bmm.default._schema) == "kami::bmm(Tensor a, Tensor b) -> Tensor"
    A = torch.zeros((1, 8, 8), dtype=torch.float16)
    with pytest.raises(NotImplementedError):
        torch.ops.kami.bmm(A, A)
