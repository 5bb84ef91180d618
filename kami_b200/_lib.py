"""Loader of libkami_b200.so (the C ABI declared in include/kami.h).

The library is built in-tree by ``kami_b200.build``.  There is no fallback:
when the library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# $KAMI_B200_LIB selects another build of the library (A/B timing of kernel variants)
LIB_PATH = os.environ.get("KAMI_B200_LIB") or os.path.join(HERE, "libkami_b200.so")

# enums of include/kami.h
KAMI_OK = 0
F16, BF16, F64, F32, S8 = 0, 1, 2, 3, 4
PARTITION_AUTO, PARTITION_1D, PARTITION_2D, PARTITION_3D = 0, 1, 2, 3
VARIANT_AUTO, VARIANT_MMA_SYNC, VARIANT_TCGEN05, VARIANT_TCGEN05_TS = 0, 1, 2, 3
A_ROW_MK, A_COL_MK = 0, 1
B_REF_NK, B_ROW_KN = 0, 1

STATUS_NAMES = {
    0: "KAMI_OK", -1: "KAMI_ERR_INVALID_VALUE", -2: "KAMI_ERR_UNSUPPORTED", -3: "KAMI_ERR_MISALIGNED",
    -4: "KAMI_ERR_WORKSPACE", -5: "KAMI_ERR_CUDA", -6: "KAMI_ERR_TIMEOUT", -7: "KAMI_ERR_INTERNAL",
}

# every exported symbol, with ctypes signatures (kept in step with kami.h)
_i = ctypes.c_int
_i64 = ctypes.c_int64
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_d = ctypes.c_double
SIGNATURES = {
    "kami_last_error_string": ([], ctypes.c_char_p),
    "kami_version": ([], _i),
    "kami_device_status": ([ctypes.POINTER(_i)], _i),
    "kami_selftest_bounded_wait": ([ctypes.c_uint64, _vp], _i),
    "kami_gemm_batched": ([_i, _i, _i, _i, _i, _i, _i, _i, _i, _i64,
                           _vp, _i64, _i64, _i,
                           _vp, _i64, _i64, _i,
                           _vp, _i64, _i64,
                           _d, _d, _i, _vp, _sz, _vp], _i),
    "kami_gemm_batched_host": ([_i, _i, _i, _i, _i, _i, _i, _i64, _vp, _vp, _vp, _i, _vp, _sz, _vp], _i),
    "kami_gemm_batched_host_workspace_size": ([_i, _i, _i, _i, _i, _i64, ctypes.POINTER(_sz)], _i),
    "kami_gemm_backward_batched": ([_i, _i, _i, _i, _i, _i64, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "kami_gemm_batched_ksplit": ([_i, _i, _i, _i, _i, _i, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64,
                                  _d, _d, _i, _i, ctypes.POINTER(_i), _vp], _i),
    "kami_gemm_trace": ([_i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _i, _vp, ctypes.POINTER(_i), _vp], _i),
    "kami_gemm_workspace_size": ([_i, _i, _i, _i, _i, _i, _i, _i64, ctypes.POINTER(_sz)], _i),
    "kami_gemm_describe": ([_i, _i, _i, _i, _i, _i, _i, _i, _i, _i64, _i, _i, ctypes.POINTER(_i)], _i),
    "kami_gemm_grouped_plan_create": ([_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i, ctypes.POINTER(_vp)], _i),
    "kami_gemm_grouped_run": ([_vp, _vp, _vp, _vp, _d, _d, _i, _vp], _i),
    "kami_gemm_grouped_plan_info": ([_vp, ctypes.POINTER(_i64)], _i),
    "kami_gemm_grouped_plan_destroy": ([_vp], _i),
    "kami_gemm_grouped_noalloc": ([_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _i, _vp], _i),
    "kami_split_f64_gemm_batched": ([_i, _i, _i, _i, _i, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _i,
                                     _vp, _i64, _i64, _d, _d, _i, _vp], _i),
    "kami_spgemm_bsr_symbolic": ([_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_i), _vp], _i),
    "kami_spgemm_bsr_fill_colidx": ([_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "kami_spgemm_bsr_numeric_variant": ([_i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                         _i64, _d, _d, _i, _vp], _i),
    "kami_spgemm_bsr_block": ([_i, _i, _i, _i, _i, _i, _i, _i, _i64, _vp, _vp, _vp, _i64, _i, _vp, _vp, _vp, _i64, _i,
                               _vp, _vp, _vp, _i64, _i, _d, _d, _i, _vp], _i),
    "kami_spgemm_bsr_symbolic_device": ([_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp], _i),
    "kami_spgemm_bsr_numeric": ([_i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                                 _d, _d, _i, _vp], _i),
    "kami_spmm_bsr": ([_i, _i, _i, _i, _i, _i, _i64, _vp, _vp, _i64, _i64, _vp, _i64,
                       _vp, _i64, _i64, _i, _vp, _i64, _i64, _d, _d, _i, _vp], _i),
    "kami_spmm_tilebsr": ([_i, _i, _i, _i, _i, _i, _i64, _i, _i, _vp, _vp, _i64, _i64, _vp, _i64,
                           _vp, _i64, _i64, _i, _vp, _i64, _i64, _d, _d, _i, _vp], _i),
    "kami_bsr_to_tilebsr": ([_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp], _i),
}


class KamiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m kami_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != KAMI_OK:
        raise KamiError(status, load().kami_last_error_string().decode())
