"""Differentiable batched block GEMM: a torch.autograd.Function whose forward
and backward both run the library's partitioned block-GEMM kernels through
the C ABI (no torch matmul on the path).

    C  = A @ B            A: [batch, M, K], B: [batch, K, N]   (torch.bmm)
    dA = dC @ B^T         B [K, N] row-major is the reference's N x K operand
                          of this product (b_layout="ref_nk")
    dB = A^T @ dC         A read transposed (a_layout="col_mk"), dC as the
                          K x N operand (b_layout="row_kn")

With the library's default kernel choice the backward is one call of
kami_gemm_backward_batched: for FP16 / BF16 64 / 128 shapes a single fused
kernel reads A, B and dC once and writes both gradients.

All three products accumulate in FP32 (FP16/BF16 inputs) or FP64 and are
returned in the input dtype, as torch.bmm does.

The default path (the library's kernel choice) is the C++ operator
torch.ops.kami.bmm (kami_b200/torch_ops/kami_torch_ops.cpp): the same two
launches with its forward, backward node and argument handling in C++, so
the host time per step stays below the kernels' time.
"""
from __future__ import annotations

import os

import torch

from . import _lib, api

_OPS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkami_torch_ops.so")
_ops_state = None


def ops_available() -> bool:
    """Load torch.ops.kami (the C++ operator library) once; False when it was
    not built, in which case bmm runs the Python autograd.Function (the same
    kernels, more host time per step)."""
    global _ops_state
    if _ops_state is None:
        _ops_state = False
        if os.path.exists(_OPS_PATH):
            _lib.load()  # the kernels' library first, so both loaders share one copy
            torch.ops.load_library(_OPS_PATH)
            _ops_state = True
    return _ops_state


def _out_dtype(dt):
    return dt if dt in (torch.float16, torch.bfloat16, torch.float64) else None


class KamiBmm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A: torch.Tensor, B: torch.Tensor, partition: str = "auto", variant: str = "auto"):
        if A.dtype != B.dtype or A.dtype not in (torch.float16, torch.bfloat16, torch.float64):
            raise TypeError("KamiBmm takes two float16, bfloat16 or float64 tensors of the same dtype")
        A = A.contiguous()
        B = B.contiguous()
        ctx.save_for_backward(A, B)
        ctx.partition, ctx.variant = partition, variant
        if partition == "auto" and variant == "auto" and A.dim() == 3 and B.dim() == 3 and A.is_cuda and B.is_cuda:
            return api.bmm_forward(A, B)
        return api.gemm_batched(A, B, b_layout="row_kn", partition=partition, variant=variant,
                                out_dtype=_out_dtype(A.dtype))

    @staticmethod
    def backward(ctx, dC: torch.Tensor):
        A, B = ctx.saved_tensors
        dC = dC.contiguous()
        dA = dB = None
        if ctx.partition == "auto" and ctx.variant == "auto" and A.dim() == 3:
            # both gradients in one launch (kami_gemm_backward_batched)
            dA, dB = api.gemm_backward(A, B, dC, need_dA=ctx.needs_input_grad[0], need_dB=ctx.needs_input_grad[1])
            return dA, dB, None, None
        if ctx.needs_input_grad[0]:
            dA = api.gemm_batched(dC, B, b_layout="ref_nk", partition=ctx.partition, variant=ctx.variant,
                                  out_dtype=_out_dtype(A.dtype))
        if ctx.needs_input_grad[1]:
            dB = api.gemm_batched(A, dC, a_layout="col_mk", b_layout="row_kn", partition=ctx.partition,
                                  variant=ctx.variant, out_dtype=_out_dtype(B.dtype))
        return dA, dB, None, None


_OP_DTYPES = (torch.float16, torch.bfloat16, torch.float64)


def bmm(A: torch.Tensor, B: torch.Tensor, partition: str = "auto", variant: str = "auto") -> torch.Tensor:
    """torch.bmm semantics, computed by the KAMI block-GEMM kernels.  With the
    library's kernel choice (partition and variant "auto") on 3-D CUDA
    operands it is the C++ operator torch.ops.kami.bmm (forward and backward
    dispatched without Python); otherwise the Python KamiBmm function."""
    if (partition == "auto" and variant == "auto" and A.dim() == 3 and B.dim() == 3 and A.is_cuda
            and A.dtype in _OP_DTYPES and ops_available()):
        return torch.ops.kami.bmm(A, B)
    return KamiBmm.apply(A, B, partition, variant)
