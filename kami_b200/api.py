"""Python mirror of the C ABI (include/kami.h) over torch CUDA tensors.

torch provides device memory and streams only; every computation runs in
libkami_b200.so.  Argument meaning follows the reference kernels: A is the
M x K operand, B is the reference's N x K operand (``b_layout="ref_nk"``,
``h_B[j*K+k]`` in batched_gemm_2d_double_mma.cu:348) or K x N
(``b_layout="row_kn"``); ``P`` is NUM_RANK_BLOCK, ``alloc_warps`` is
NUM_ALLOC_RANK_BLOCK and ``num_iter`` is NUM_ITER.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check, load

_DT = {torch.float16: _lib.F16, torch.bfloat16: _lib.BF16, torch.float64: _lib.F64, torch.float32: _lib.F32}
_PART = {"auto": _lib.PARTITION_AUTO, "1d": _lib.PARTITION_1D, "2d": _lib.PARTITION_2D, "3d": _lib.PARTITION_3D}
_VAR = {"auto": _lib.VARIANT_AUTO, "mma_sync": _lib.VARIANT_MMA_SYNC, "tcgen05": _lib.VARIANT_TCGEN05,
        "tcgen05_ts": _lib.VARIANT_TCGEN05_TS}
_AL = {"row_mk": _lib.A_ROW_MK, "col_mk": _lib.A_COL_MK}
_BL = {"ref_nk": _lib.B_REF_NK, "row_kn": _lib.B_ROW_KN}


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_device = getattr(torch._C, "_cuda_getDevice", None)


def _stream_ptr(stream) -> int:
    """The CUDA stream handle to launch on: ``stream``, else the current
    stream of the current device (read without building a Stream object)."""
    if stream is None and _raw_stream is not None and _cur_device is not None:
        return _raw_stream(_cur_device())
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _device_index(*tensors) -> int:
    """The CUDA device every given tensor lives on (None entries are
    skipped).  Raises ValueError for a tensor off the GPU or operands on
    different devices: a kernel launched on one device with another
    device's pointers would fault or read through peer mappings."""
    idx = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError("operands must be CUDA tensors")
        d = t.device.index
        if idx is None:
            idx = d
        elif d != idx:
            raise ValueError(f"operands are on different devices (cuda:{idx} and cuda:{d})")
    return idx


class _OnDevice:
    """Makes `index` the current device for the duration of a call (so the
    launch and the default stream belong to the operands' device), at the
    cost of one device query when it already is."""
    __slots__ = ("index", "prev")

    def __init__(self, index):
        self.index = index
        self.prev = None

    def __enter__(self):
        if self.index is not None and _cur_device is not None:
            cur = _cur_device()
            if cur != self.index:
                self.prev = cur
                torch.cuda.set_device(self.index)
        return self

    def __exit__(self, *exc):
        if self.prev is not None:
            torch.cuda.set_device(self.prev)
        return False


def _on(*tensors) -> _OnDevice:
    return _OnDevice(_device_index(*tensors))


def _as3(x: torch.Tensor) -> torch.Tensor:
    return x.unsqueeze(0) if x.dim() == 2 else x


def _check_inner(x: torch.Tensor, name: str):
    if x.stride(-1) != 1 and x.shape[-1] > 1:
        raise ValueError(f"{name} must be contiguous in its last dimension")


def _ld(x: torch.Tensor) -> int:
    """Row stride of a [batch, rows, cols] operand; a single row has no
    meaningful stride (torch may report anything), so use the row length."""
    return x.stride(1) if x.shape[1] > 1 else x.shape[2]


def _bs(x: torch.Tensor) -> int:
    return x.stride(0) if x.shape[0] > 1 else 0


def gemm_batched(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *,
                 a_layout: str = "row_mk", b_layout: str = "ref_nk", partition: str = "auto",
                 variant: str = "auto", P: int = 0, alloc_warps: int = 0, num_iter: int = 1,
                 alpha: float = 1.0, beta: float = 0.0, out_dtype: torch.dtype | None = None,
                 stream=None) -> torch.Tensor:
    """C[b] = alpha * num_iter * A[b] op(B[b]) + beta * C[b] (kami_gemm_batched).

    A: [batch, M, K] (row_mk) or [batch, K, M] (col_mk).
    B: [batch, N, K] (ref_nk) or [batch, K, N] (row_kn).
    Returns C [batch, M, N]: float32 for 16-bit inputs unless ``out_dtype``
    (float16 / bfloat16) is given, float64 for float64 inputs."""
    squeeze = A.dim() == 2
    A3, B3 = _as3(A), _as3(B)
    if A3.dtype != B3.dtype:
        raise TypeError("A and B must have the same dtype")
    dev = _on(A3, B3, C)
    _check_inner(A3, "A")
    _check_inner(B3, "B")
    batch = A3.shape[0]
    if a_layout == "row_mk":
        M, K = A3.shape[1], A3.shape[2]
    else:
        K, M = A3.shape[1], A3.shape[2]
    N = B3.shape[1] if b_layout == "ref_nk" else B3.shape[2]
    if C is None:
        odt = out_dtype or (torch.float64 if A3.dtype == torch.float64 else torch.float32)
        C3 = torch.empty((batch, M, N), dtype=odt, device=A3.device)
    else:
        C3 = _as3(C)
        _check_inner(C3, "C")
    with dev:
        st = load().kami_gemm_batched(
            _DT[A3.dtype], _DT[C3.dtype], _PART[partition], _VAR[variant], M, N, K, P, alloc_warps, batch,
            A3.data_ptr(), _ld(A3), _bs(A3), _AL[a_layout],
            B3.data_ptr(), _ld(B3), _bs(B3), _BL[b_layout],
            C3.data_ptr(), _ld(C3), _bs(C3),
            float(alpha), float(beta), int(num_iter), None, 0, _stream_ptr(stream))
    check(st)
    if C is not None:
        return C
    return C3[0] if squeeze else C3


def bmm_forward(A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    """C = A @ B in torch.bmm layout (A [batch, M, K], B [batch, K, N], both
    contiguous CUDA tensors of one dtype: float16, bfloat16 or float64),
    returned in the input dtype: kami_gemm_batched with B as the K x N
    operand and the library's kernel choice, with the fewest host steps (the
    forward of the autograd function)."""
    if A.dim() != 3 or B.dim() != 3:
        raise ValueError("A and B must be 3-D: [batch, M, K] and [batch, K, N]")
    if A.dtype != B.dtype or A.dtype not in (torch.float16, torch.bfloat16, torch.float64):
        raise TypeError("A and B must both be float16, bfloat16 or float64")
    if not (A.is_contiguous() and B.is_contiguous()):
        raise ValueError("A and B must be contiguous")
    batch, M, K = A.shape
    N = B.shape[2]
    if B.shape[0] != batch or B.shape[1] != K:
        raise ValueError("shapes do not match C = A @ B")
    dev = _on(A, B)
    dt = _DT[A.dtype]
    C = torch.empty((batch, M, N), dtype=A.dtype, device=A.device)
    with dev:
        st = load().kami_gemm_batched(dt, dt, _lib.PARTITION_AUTO, _lib.VARIANT_AUTO, M, N, K, 0, 0, batch,
                                      A.data_ptr(), K, M * K, _lib.A_ROW_MK, B.data_ptr(), N, K * N, _lib.B_ROW_KN,
                                      C.data_ptr(), N, M * N, 1.0, 0.0, 1, None, 0, _stream_ptr(None))
    check(st)
    return C


def gemm_batched_host(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, *, partition: str = "auto",
                      variant: str = "auto", num_iter: int = 1, stream=None) -> torch.Tensor:
    """kami_gemm_batched_host: C = num_iter * A B^T for CPU tensors (pinned for
    overlap; contiguous A [batch, M, K], B [batch, N, K], C [batch, M, N]), the
    host copies pipelined with the product by chunks.  Returns C; it is
    complete once ``stream`` (default: the current stream) is synchronised."""
    for x, name in ((A, "A"), (B, "B"), (C, "C")):
        if x.is_cuda or not x.is_contiguous():
            raise ValueError(f"{name} must be a contiguous CPU tensor")
    A3, B3, C3 = _as3(A), _as3(B), _as3(C)
    batch, M, K = A3.shape
    N = B3.shape[1]
    check(load().kami_gemm_batched_host(_DT[A3.dtype], _DT[C3.dtype], _PART[partition], _VAR[variant], M, N, K,
                                        batch, A3.data_ptr(), B3.data_ptr(), C3.data_ptr(), int(num_iter), None, 0,
                                        _stream_ptr(stream)))
    return C


def gemm_backward(A: torch.Tensor, B: torch.Tensor, dC: torch.Tensor, *, need_dA: bool = True,
                  need_dB: bool = True, out_dtype: torch.dtype | None = None, stream=None):
    """Gradients of C = A @ B (torch.bmm layout: A [batch, M, K], B [batch,
    K, N], dC [batch, M, N], contiguous) by kami_gemm_backward_batched: one
    fused kernel for FP16 / BF16 64 / 128 shapes.  Returns (dA, dB), None for
    a gradient not asked for; outputs in ``out_dtype`` (default: the input
    dtype)."""
    A3, B3, G3 = _as3(A).contiguous(), _as3(B).contiguous(), _as3(dC).contiguous()
    if not (A3.dtype == B3.dtype == G3.dtype):
        raise TypeError("A, B and dC must have the same dtype")
    batch, M, K = A3.shape
    N = B3.shape[2]
    if B3.shape[1] != K or G3.shape[1:] != (M, N) or B3.shape[0] != batch or G3.shape[0] != batch:
        raise ValueError("shapes do not match C = A @ B")
    dev = _on(A3, B3, G3)
    odt = out_dtype or A3.dtype
    dA = torch.empty((batch, M, K), dtype=odt, device=A3.device) if need_dA else None
    dB = torch.empty((batch, K, N), dtype=odt, device=A3.device) if need_dB else None
    with dev:
        st = load().kami_gemm_backward_batched(_DT[A3.dtype], _DT[odt], M, N, K, batch, A3.data_ptr(),
                                               B3.data_ptr(), G3.data_ptr(), dA.data_ptr() if dA is not None else None,
                                               dB.data_ptr() if dB is not None else None, _stream_ptr(stream))
    check(st)
    if A.dim() == 2:
        dA = dA[0] if dA is not None else None
        dB = dB[0] if dB is not None else None
    return dA, dB


def gemm_batched_ksplit(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *, P: int = 0,
                        reg_k_steps: int = -1, num_iter: int = 1, alpha: float = 1.0, beta: float = 0.0,
                        out_dtype: torch.dtype | None = None, stream=None):
    """1D block GEMM with K split between registers and shared memory
    (kami_gemm_batched_ksplit).  A: [batch, M, K], B: [batch, N, K] (the
    reference's layout), FP16 or BF16.  reg_k_steps -1 measures the compiled
    splits and keeps the fastest.  Returns (C, reg_k_steps used)."""
    A3, B3 = _as3(A), _as3(B)
    if A3.dtype != B3.dtype or A3.dtype not in (torch.float16, torch.bfloat16):
        raise TypeError("A and B must both be float16 or both bfloat16")
    _check_inner(A3, "A")
    _check_inner(B3, "B")
    batch, M, K = A3.shape
    N = B3.shape[1]
    if C is None:
        C3 = torch.empty((batch, M, N), dtype=out_dtype or torch.float32, device=A3.device)
    else:
        C3 = _as3(C)
        _check_inner(C3, "C")
    used = ctypes.c_int(-2)
    with _on(A3, B3, C3):
        st = load().kami_gemm_batched_ksplit(_DT[A3.dtype], _DT[C3.dtype], M, N, K, P, batch,
                                             A3.data_ptr(), _ld(A3), _bs(A3), B3.data_ptr(), _ld(B3), _bs(B3),
                                             C3.data_ptr(), _ld(C3), _bs(C3), float(alpha), float(beta),
                                             int(num_iter), int(reg_k_steps), ctypes.byref(used), _stream_ptr(stream))
    check(st)
    out = C if C is not None else (C3[0] if A.dim() == 2 else C3)
    return out, used.value


def gemm_trace(A: torch.Tensor, B: torch.Tensor, *, partition: str = "1d", P: int, reg_k_steps: int = -1,
               num_iter: int = 10, stream=None):
    """Per-warp communication / computation clock64 cycles of one FP16 block
    GEMM (kami_gemm_trace).  A: [M, K], B: [N, K] float16 on the device.
    Returns (C [M, N] float32, cycles [nwarps, 2] int64 numpy array)."""
    import numpy as np
    if A.dtype != torch.float16 or B.dtype != torch.float16:
        raise TypeError("the traced instances take float16 A and B")
    A, B = A.contiguous(), B.contiguous()
    M, K = A.shape
    N = B.shape[0]
    C = torch.empty((M, N), dtype=torch.float32, device=A.device)
    cyc = torch.zeros(64, dtype=torch.int64, device=A.device)
    nw = ctypes.c_int(0)
    with _on(A, B):
        st = load().kami_gemm_trace(_PART[partition], M, N, K, P, reg_k_steps, A.data_ptr(), B.data_ptr(),
                                    C.data_ptr(), int(num_iter), cyc.data_ptr(), ctypes.byref(nw), _stream_ptr(stream))
    check(st)
    return C, cyc.cpu().numpy()[: 2 * nw.value].reshape(nw.value, 2)


def describe(M: int, N: int, K: int, batch: int, dtype=torch.float16, out_dtype=None, *, partition="auto",
             variant="auto", P=0, alloc_warps=0, a_layout="row_mk", b_layout="ref_nk") -> dict:
    """The kernel kami_gemm_batched would launch for this request."""
    out = (ctypes.c_int * 8)()
    odt = out_dtype or (torch.float64 if dtype == torch.float64 else torch.float32)
    check(load().kami_gemm_describe(_DT[dtype], _DT[odt], _PART[partition], _VAR[variant], M, N, K, P,
                                    alloc_warps, batch, _AL[a_layout], _BL[b_layout], out))
    keys = ["variant", "partition", "P", "threads", "smem", "problems_per_cta", "grid"]
    d = dict(zip(keys, list(out)[:7]))
    d["variant"] = {1: "mma_sync", 2: "tcgen05", 3: "tcgen05_ts"}[d["variant"]]
    d["partition"] = {1: "1d", 2: "2d", 3: "3d"}[d["partition"]]
    return d


class GroupedPlan:
    """A persistent-launch plan for uneven problems (kami_gemm_grouped_*).

    shapes: sequence of (M, N, K).  Problems are packed back to back in the
    A, B and C buffers (A_i M x K, B_i N x K, C_i M x N, row-major) unless
    explicit element offsets are given.  kernel: None (the library's choice:
    tcgen05 for FP16 / BF16, staged DMMA for FP64, measured against mma.sync
    when autotuned), "mma_sync", "tcgen05" or "staged" (KAMI_PLAN_MMA_SYNC /
    KAMI_PLAN_TCGEN05 / KAMI_PLAN_STAGED)."""

    def __init__(self, shapes, dtype=torch.float16, out_dtype=None, *, autotune=False, offsets=None, kernel=None,
                 pack=False):
        import numpy as np
        sh = np.asarray(shapes, dtype=np.int64).reshape(-1, 3)
        self.count = len(sh)
        self.dtype = dtype
        self.out_dtype = out_dtype or (torch.float64 if dtype == torch.float64 else torch.float32)
        M, N, K = (np.ascontiguousarray(sh[:, i], dtype=np.int32) for i in range(3))
        if offsets is None:
            a = np.concatenate([[0], np.cumsum(sh[:, 0] * sh[:, 2])])
            b = np.concatenate([[0], np.cumsum(sh[:, 1] * sh[:, 2])])
            c = np.concatenate([[0], np.cumsum(sh[:, 0] * sh[:, 1])])
            offsets = (a[:-1], b[:-1], c[:-1])
            self.sizes = (int(a[-1]), int(b[-1]), int(c[-1]))
        ao, bo, co = (np.ascontiguousarray(o, dtype=np.int64) for o in offsets)
        self.shapes, self.offsets = sh, (ao, bo, co)
        # the plan's descriptors live on the device current at creation
        self.device_index = _cur_device() if _cur_device is not None and torch.cuda.is_available() else None
        h = ctypes.c_void_p()
        check(load().kami_gemm_grouped_plan_create(_DT[dtype], _DT[self.out_dtype], self.count,
                                                   M.ctypes.data, N.ctypes.data, K.ctypes.data, ao.ctypes.data,
                                                   bo.ctypes.data, co.ctypes.data,
                                                   (1 if autotune else 0) | (16 if pack else 0)
                                                   | {None: 0, "mma_sync": 2, "tcgen05": 4, "staged": 8}[kernel],
                                                   ctypes.byref(h)))
        self._h = h

    def info(self) -> dict:
        out = (ctypes.c_int64 * 16)()
        check(load().kami_gemm_grouped_plan_info(self._h, out))
        v = list(out)
        return {"problems": v[0], "ctas": v[1], "smem": v[2], "flops": v[3], "bytes": v[4],
                "partitions": v[5:13], "kernel": {0: "mma_sync", 1: "tcgen05", 2: "staged"}[v[13]],
                "tcgen05_m64": v[14], "tcgen05_m128": v[15]}

    def run(self, A: torch.Tensor, B: torch.Tensor, C: torch.Tensor, *, alpha=1.0, beta=0.0, num_iter=1,
            stream=None) -> torch.Tensor:
        idx = _device_index(A, B, C)
        if self.device_index is not None and idx != self.device_index:
            raise ValueError(f"the plan was built on cuda:{self.device_index}, the operands are on cuda:{idx}")
        with _OnDevice(idx):
            st = load().kami_gemm_grouped_run(self._h, A.data_ptr(), B.data_ptr(), C.data_ptr(), float(alpha),
                                              float(beta), int(num_iter), _stream_ptr(stream))
        check(st)
        return C

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                load().kami_gemm_grouped_plan_destroy(h)
            except Exception:
                pass
            self._h = None


def split_f64_gemm(A: torch.Tensor, B: torch.Tensor, C: torch.Tensor | None = None, *, nslices: int = 6,
                   slice_dtype=torch.float16, b_layout: str = "ref_nk", alpha: float = 1.0, beta: float = 0.0,
                   num_iter: int = 1, stream=None) -> torch.Tensor:
    """FP64 C = A op(B) via exact digit slices on the tensor cores
    (kami_split_f64_gemm_batched): slice_dtype torch.float16 (2-7 slices),
    torch.bfloat16 (2-8) or torch.int8 (2-8; 8 slices carry 62 bits).
    A: [batch, M, K] float64; B: [batch, N, K] (ref_nk) or [batch, K, N]
    (row_kn)."""
    squeeze = A.dim() == 2
    A3, B3 = _as3(A), _as3(B)
    if A3.dtype != torch.float64 or B3.dtype != torch.float64:
        raise TypeError("split_f64_gemm takes float64 operands")
    _check_inner(A3, "A")
    _check_inner(B3, "B")
    batch, M, K = A3.shape
    N = B3.shape[1] if b_layout == "ref_nk" else B3.shape[2]
    C3 = torch.empty((batch, M, N), dtype=torch.float64, device=A3.device) if C is None else _as3(C)
    with _on(A3, B3, C3):
        st = load().kami_split_f64_gemm_batched(
            int(nslices), _lib.S8 if slice_dtype == torch.int8 else _DT[slice_dtype], M, N, K, batch,
            A3.data_ptr(), _ld(A3), _bs(A3),
            B3.data_ptr(), _ld(B3), _bs(B3), _BL[b_layout], C3.data_ptr(), _ld(C3), _bs(C3),
            float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    check(st)
    if C is not None:
        return C
    return C3[0] if squeeze else C3


# ---------------------------------------------------------------------------
# block SpGEMM (BSR, 16 x 16 tiles)
# ---------------------------------------------------------------------------
class BSR:
    """A block-sparse matrix on the device: row_ptr (int32, rows+1), col_idx
    (int32, ascending per block-row) and values [nnz, 16, 16]."""

    def __init__(self, row_ptr: torch.Tensor, col_idx: torch.Tensor, values: torch.Tensor, block_cols: int):
        self.row_ptr, self.col_idx, self.values = row_ptr, col_idx, values
        self.block_rows = row_ptr.numel() - 1
        self.block_cols = block_cols

    @property
    def nnz_blocks(self) -> int:
        return self.col_idx.numel()


def spgemm_symbolic(A: BSR, B: BSR, stream=None):
    """RowPtrC and nnzC (host int; synchronises like the reference's D2H)."""
    if A.block_cols != B.block_rows:
        raise ValueError("inner block dimensions differ")
    rpc = torch.empty(A.block_rows + 1, dtype=torch.int32, device=A.row_ptr.device)
    nnz = ctypes.c_int(0)
    with _on(*_bsr_tensors(A, B)):
        st = load().kami_spgemm_bsr_symbolic(16, A.block_rows, A.block_cols, B.block_cols, A.row_ptr.data_ptr(),
                                             _ptr(A.col_idx), B.row_ptr.data_ptr(), _ptr(B.col_idx),
                                             rpc.data_ptr(), ctypes.byref(nnz), _stream_ptr(stream))
    check(st)
    return rpc, nnz.value


def spgemm_fill_colidx(A: BSR, B: BSR, row_ptr_c: torch.Tensor, nnz_c: int, stream=None) -> torch.Tensor:
    cic = torch.empty(max(nnz_c, 1), dtype=torch.int32, device=A.row_ptr.device)
    with _on(*_bsr_tensors(A, B), row_ptr_c):
        st = load().kami_spgemm_bsr_fill_colidx(16, A.block_rows, A.block_cols, B.block_cols, A.row_ptr.data_ptr(),
                                                _ptr(A.col_idx), B.row_ptr.data_ptr(), _ptr(B.col_idx),
                                                row_ptr_c.data_ptr(), cic.data_ptr(), _stream_ptr(stream))
    check(st)
    return cic[:nnz_c]


def spgemm_numeric(A: BSR, B: BSR, row_ptr_c, col_idx_c, out_dtype=torch.float32, C_values=None, *,
                   alpha=1.0, beta=0.0, num_iter=1, variant: str = "auto", stream=None) -> torch.Tensor:
    """Numeric pass (kami_spgemm_bsr_numeric_variant): variant "auto",
    "mma_sync" or "tcgen05"."""
    nnz_c = col_idx_c.numel()
    if C_values is None:
        C_values = torch.empty((max(nnz_c, 1), 16, 16), dtype=out_dtype, device=A.row_ptr.device)
    with _on(*_bsr_tensors(A, B), row_ptr_c, col_idx_c, C_values):
        st = load().kami_spgemm_bsr_numeric_variant(_VAR[variant], _DT[A.values.dtype], _DT[C_values.dtype], 16,
                                            A.block_rows,
                                            A.block_cols, B.block_cols, A.row_ptr.data_ptr(), _ptr(A.col_idx),
                                            _ptr(A.values), B.row_ptr.data_ptr(), _ptr(B.col_idx), _ptr(B.values),
                                            row_ptr_c.data_ptr(), _ptr(col_idx_c), _ptr(C_values), nnz_c,
                                            float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    check(st)
    return C_values[:nnz_c]


def spgemm_symbolic_device(A: BSR, B: BSR, capacity: int, stream=None):
    """RowPtrC and ColIdxC (capacity entries) without a host round trip
    (kami_spgemm_bsr_symbolic_device); nnzC is row_ptr_c[-1] on the device."""
    if A.block_cols != B.block_rows:
        raise ValueError("inner block dimensions differ")
    dev = A.row_ptr.device
    rpc = torch.empty(A.block_rows + 1, dtype=torch.int32, device=dev)
    cic = torch.empty(max(int(capacity), 1), dtype=torch.int32, device=dev)
    with _on(*_bsr_tensors(A, B)):
        st = load().kami_spgemm_bsr_symbolic_device(16, A.block_rows, A.block_cols, B.block_cols,
                                                    A.row_ptr.data_ptr(), _ptr(A.col_idx), B.row_ptr.data_ptr(),
                                                    _ptr(B.col_idx), rpc.data_ptr(), cic.data_ptr(), int(capacity),
                                                    _stream_ptr(stream))
    check(st)
    return rpc, cic


def spgemm_numeric_bound(A: BSR, B: BSR, row_ptr_c, col_idx_c, C_values, *, alpha=1.0, beta=0.0, num_iter=1,
                         variant: str = "auto", stream=None) -> torch.Tensor:
    """Numeric pass into C_values [capacity, 16, 16] with the capacity as the
    bound of nnzC (no host synchronisation)."""
    cap = C_values.shape[0]
    with _on(*_bsr_tensors(A, B), row_ptr_c, col_idx_c, C_values):
        st = load().kami_spgemm_bsr_numeric_variant(_VAR[variant], _DT[A.values.dtype], _DT[C_values.dtype], 16,
                                            A.block_rows,
                                            A.block_cols, B.block_cols, A.row_ptr.data_ptr(), _ptr(A.col_idx),
                                            _ptr(A.values), B.row_ptr.data_ptr(), _ptr(B.col_idx), _ptr(B.values),
                                            row_ptr_c.data_ptr(), _ptr(col_idx_c), _ptr(C_values), cap,
                                            float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    check(st)
    return C_values


def spgemm(A: BSR, B: BSR, out_dtype=torch.float32, *, num_iter=1, variant: str = "auto", stream=None) -> BSR:
    """C = A * B: symbolic, column fill, numeric (the reference's sequence)."""
    rpc, nnz = spgemm_symbolic(A, B, stream)
    cic = spgemm_fill_colidx(A, B, rpc, nnz, stream)
    vals = spgemm_numeric(A, B, rpc, cic, out_dtype, num_iter=num_iter, variant=variant, stream=stream)
    return BSR(rpc, cic, vals, B.block_cols)


def spgemm_block(A: BSR, B: BSR, C: BSR, *, partition: str = "1d", P: int = 0, alpha: float = 1.0,
                 beta: float = 0.0, num_iter: int = 1, stream=None) -> torch.Tensor:
    """The reference's one-CTA block SpGEMM (kami_spgemm_bsr_block): C.values
    = alpha * num_iter * A * B + beta * C.values for small BSR matrices (at
    most 16 x 16 blocks) whose structure is shared by a batch: A.values
    [batch, nnzA, 16, 16] or [nnzA, 16, 16] (shared), B likewise, C.values
    [batch, nnzC, 16, 16] or [nnzC, 16, 16]; C.row_ptr / C.col_idx from the
    symbolic pass.  The batch is the largest leading dimension."""
    def _split(v):
        return (v.shape[0], v.stride(0)) if v.dim() == 4 else (1, 0)
    ba, sa = _split(A.values)
    bb, sb = _split(B.values)
    bc, sc = _split(C.values)
    batch = max(ba, bb, bc)
    if bc != batch:
        raise ValueError("C.values must hold one tile set per problem")
    with _on(*_bsr_tensors(A, B, C)):
        st = load().kami_spgemm_bsr_block(
            _DT[A.values.dtype], _DT[C.values.dtype], _PART[partition], int(P), 16, A.block_rows, A.block_cols,
            B.block_cols, batch, A.row_ptr.data_ptr(), _ptr(A.col_idx), _ptr(A.values), sa, A.nnz_blocks,
            B.row_ptr.data_ptr(), _ptr(B.col_idx), _ptr(B.values), sb, B.nnz_blocks,
            C.row_ptr.data_ptr(), _ptr(C.col_idx), _ptr(C.values), sc, C.nnz_blocks,
            float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    check(st)
    return C.values


def spmm(A: BSR, B: torch.Tensor, C: torch.Tensor | None = None, *, b_layout: str = "row_kn",
         out_dtype=torch.float32, alpha: float = 1.0, beta: float = 0.0, num_iter: int = 1,
         stream=None) -> torch.Tensor:
    """Block SpMM (kami_spmm_bsr): C [16 mb, N] = A * B for a BSR matrix A and
    a dense B, [K, N] (row_kn, torch's A @ B) or [N, K] (ref_nk, the
    reference's layout: C = A * B^T).  FP16/BF16 operands, FP32 accumulation."""
    K = A.block_cols * 16
    if B.dim() != 2:
        raise ValueError("B must be 2-D")
    N = B.shape[1] if b_layout == "row_kn" else B.shape[0]
    if (B.shape[0] if b_layout == "row_kn" else B.shape[1]) != K:
        raise ValueError(f"B does not match K = {K}")
    if B.stride(1) != 1:
        B = B.contiguous()
    if C is None:
        C = torch.empty((A.block_rows * 16, N), dtype=out_dtype, device=B.device)
    with _on(A.row_ptr, A.col_idx, A.values, B, C):
        st = load().kami_spmm_bsr(_DT[A.values.dtype], _DT[C.dtype], 16, A.block_rows, A.block_cols, N, 1,
                                  A.row_ptr.data_ptr(), _ptr(A.col_idx), 0, 0, _ptr(A.values), 0,
                                  B.data_ptr(), _ld(B[None]), 0, _BL[b_layout], C.data_ptr(), _ld(C[None]), 0,
                                  float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    check(st)
    return C


def spmm_batched(row_ptr: torch.Tensor, col_idx: torch.Tensor, values: torch.Tensor, block_cols: int,
                 B: torch.Tensor, C: torch.Tensor | None = None, *, b_layout: str = "ref_nk",
                 out_dtype=torch.float32, alpha: float = 1.0, beta: float = 0.0, num_iter: int = 1,
                 tile_rows: int = 0, tile_cols: int = 0, stream=None) -> torch.Tensor:
    """Batched block SpMM (kami_spmm_bsr / kami_spmm_tilebsr).  row_ptr
    [batch, rows+1] or [rows+1] (shared), col_idx [batch, e] or [e], values
    [batch, e, 16, 16] or [e, 16, 16]; B [batch, N, K] (ref_nk) or
    [batch, K, N] (row_kn), or 2-D (shared); the batch is the largest
    leading dimension among them and C [batch, 16 rows, N] (when given), so
    fully shared operands with a batched C repeat one problem, as the
    reference's 16384-CTA launch does.  tile_rows / tile_cols > 0 select the
    reference's tiled-BSR index form."""
    def _b(t, nd):
        return (t.shape[0], t.stride(0)) if t.dim() == nd else (1, 0)
    nb_r, s_r = _b(row_ptr, 2)
    nb_c, s_c = _b(col_idx, 2)
    nb_v, s_v = _b(values, 4)
    nb_b, s_b = _b(B, 3)
    batch = max(nb_r, nb_c, nb_v, nb_b, C.shape[0] if C is not None and C.dim() == 3 else 1)
    if not (tile_rows and tile_cols):
        tile_rows = tile_cols = 0
    mb = row_ptr.shape[-1] - 1
    B2 = B if B.dim() == 2 else B[0]
    N = B2.shape[0] if b_layout == "ref_nk" else B2.shape[1]
    if tile_rows:
        nct = block_cols // tile_cols
        mb = (row_ptr.shape[-1] - 1) // nct
    if C is None:
        C = torch.empty((batch, mb * 16, N), dtype=out_dtype, device=B.device)
    s_cc = _bs(C) if C.dim() == 3 else 0
    ldc = _ld(C if C.dim() == 3 else C[None])
    ldb = _ld(B if B.dim() == 3 else B[None])
    L = load()
    dev = _on(row_ptr, col_idx, values, B, C)
    common_tail = (_ptr(values), s_v, B.data_ptr(), ldb, s_b, _BL[b_layout], C.data_ptr(), ldc, s_cc,
                   float(alpha), float(beta), int(num_iter), _stream_ptr(stream))
    with dev:
        if tile_rows:
            st = L.kami_spmm_tilebsr(_DT[values.dtype], _DT[C.dtype], 16, mb, block_cols, N, batch, tile_rows,
                                     tile_cols, row_ptr.data_ptr(), _ptr(col_idx), s_r, s_c, *common_tail)
        else:
            st = L.kami_spmm_bsr(_DT[values.dtype], _DT[C.dtype], 16, mb, block_cols, N, batch,
                                 row_ptr.data_ptr(), _ptr(col_idx), s_r, s_c, *common_tail)
    check(st)
    return C


def bsr_to_tilebsr(row_ptr, col_idx, block_cols: int, tile_rows: int, tile_cols: int):
    """The reference's bsr2tilebsr on host arrays (numpy int32): returns
    (blk_row_ptr, blk_col_idx, perm) with perm[e] = the BSR entry of tiled
    entry e."""
    import numpy as np
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    mb = rp.size - 1
    nct = block_cols // tile_cols
    brp = np.zeros((mb // tile_rows) * nct * tile_rows + 1, dtype=np.int32)
    bci = np.zeros(max(ci.size, 1), dtype=np.int32)
    perm = np.zeros(max(ci.size, 1), dtype=np.int32)
    n = load().kami_bsr_to_tilebsr(mb, block_cols, tile_rows, tile_cols, rp.ctypes.data, ci.ctypes.data,
                                   brp.ctypes.data, bci.ctypes.data, perm.ctypes.data)
    check(n if n < 0 else 0)
    return brp, bci[:n], perm[:n]


def _bsr_tensors(*mats):
    return [t for m in mats for t in (m.row_ptr, m.col_idx, m.values)]


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr() if t.numel() else 0
