"""ctypes wrapper over ``oracle/libkami_oracle.so`` (the CPU restatement of the
reference's host-side checks) and over the reference libraries that
``oracle/Makefile.ref`` builds into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY -- see ``oracle/__init__.py``.  Every function cites
the reference code it restates (paths inside the KAMI project).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkami_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

B_REF_NK = 0  # B stored N x K row-major: the reference's layout
B_ROW_KN = 1  # B stored K x N row-major

_lib = None

_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u16p = ctypes.POINTER(ctypes.c_uint16)


def build(force: bool = False) -> None:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def reference_root() -> str:
    """The reference checkout: $KAMI_REFERENCE_ROOT, else /root/reference."""
    return os.environ.get("KAMI_REFERENCE_ROOT") or "/root/reference"


def build_reference(ref_root: str | None = None) -> bool:
    """Compile the reference pieces into ``oracle/_ref`` when the reference
    sources are present (``ref_root``, default :func:`reference_root`).
    Returns True when the libraries exist afterwards."""
    ref_root = ref_root or reference_root()
    if os.path.isdir(ref_root):
        subprocess.run(["make", "-s", "-C", HERE, "-f", "Makefile.ref", "-j8", f"REF={ref_root}"],
                       check=True)
    return os.path.exists(os.path.join(REF_DIR, "libref_spgemm2d_host.so"))


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.kami_oracle_fill_rand_r_mod.argtypes = [_dp, _i64, _i32]
        L.kami_oracle_bsr_generate.argtypes = [_i32, _i32, ctypes.c_float, _i32, _i32, _ip, _ip, _u16p]
        L.kami_oracle_bsr_generate.restype = _i32
        L.kami_oracle_bsr_generate_rule.argtypes = [_i32, _i32, ctypes.c_float, _i32, _i32, _i32, _i32, _ip, _ip,
                                                    _u16p]
        L.kami_oracle_bsr_generate_rule.restype = _i32
        L.kami_oracle_bsr2tilebsr.argtypes = [_i32, _i32, _i32, _i32, _ip, _ip, _ip, _ip]
        L.kami_oracle_bsr2tilebsr.restype = _i32
        L.kami_oracle_spmm.argtypes = [_i32, _i32, _i32, _i32, _i32, _ip, _ip, _dp, _dp, _i64, _i32, _dp, _i64]
        L.kami_oracle_gemm_f64.argtypes = [_i64, _i32, _i32, _i32, _dp, _i64, _i64, _dp, _i64, _i64, _i32,
                                           _dp, _i64, _i64]
        L.kami_oracle_gemm_h16.argtypes = [_i64, _i32, _i32, _i32, _u16p, _i64, _i64, _u16p, _i64, _i64, _i32,
                                           _i32, _dp, _i64, _i64]
        L.kami_oracle_reduce_slices_f64.argtypes = [_i64, _i32, _i32, _i32, _dp, _dp]
        L.kami_oracle_gemm_dd.argtypes = [_i64, _i32, _i32, _i32, _dp, _i64, _i64, _dp, _i64, _i64, _i32,
                                          _dp, _dp, _i64, _i64]
        L.kami_oracle_normwise_error_dd.argtypes = [_i64, _dp, _dp, _dp]
        L.kami_oracle_normwise_error_dd.restype = ctypes.c_double
        L.kami_oracle_spgemm_symbolic.argtypes = [_i32, _i32, _ip, _ip, _ip, _ip, _ip]
        L.kami_oracle_spgemm_symbolic.restype = _i32
        L.kami_oracle_spgemm_numeric.argtypes = [_i32, _i32, _i32, _ip, _ip, _u16p, _ip, _ip, _u16p, _ip, _ip,
                                                 _i32, _u16p, _dp]
        L.kami_oracle_spgemm_nnzcub.argtypes = [_i32, _ip, _ip]
        L.kami_oracle_spgemm_nnzcub.restype = _i64
        L.kami_oracle_bsr_pattern.argtypes = [_i32, _i32, ctypes.c_double, ctypes.c_uint64, _ip, _ip, _i32]
        L.kami_oracle_bsr_pattern.restype = _i32
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------

def fill_rand_r_mod(n: int, mod: int = 3) -> np.ndarray:
    """x[i] = rand_r(&i) % mod (batched_gemm_2d_double_mma.cu:271-285)."""
    x = np.empty(n, dtype=np.float64)
    lib().kami_oracle_fill_rand_r_mod(_p(x, _dp), n, mod)
    return x


# value rules of the reference's generate_random_bsr_matrix copies
BSR_RULES = {
    "spgemm": (3, 1),  # block_spgemm_2d_half_mma.cu:648-673: rand() % 3 + 1
    "spmm1d": (3, 0),  # spmm/1d/block_spmm_1d_half_mma.cu:197-222: rand() % 3
    "spmm2d": (2, 1),  # spmm/2d/...:236-262 and spmm/3d/...:241-266: rand() % 2 + 1
}


def bsr_generate(rows: int, cols: int, sparsity: float, bsr: int = 16, rule: str = "spgemm"):
    """generate_random_bsr_matrix of the reference's sparse programs (srand(0),
    one rand() per block position, values by `rule`): returns (row_ptr int32,
    col_idx int32, values float16 [nnz, bsr, bsr])."""
    mod, add = BSR_RULES[rule]
    row_ptr = np.zeros(rows + 1, dtype=np.int32)
    col_idx = np.zeros(max(rows * cols, 1), dtype=np.int32)
    vals = np.zeros(max(rows * cols, 1) * bsr * bsr, dtype=np.uint16)
    nnz = lib().kami_oracle_bsr_generate_rule(rows, cols, sparsity, bsr, bsr, mod, add, _p(row_ptr, _ip),
                                              _p(col_idx, _ip), _p(vals, _u16p))
    return row_ptr, col_idx[:nnz].copy(), vals[: nnz * bsr * bsr].view(np.float16).reshape(nnz, bsr, bsr).copy()


def bsr2tilebsr(row_ptr, col_idx, cols: int, row_tiles: int, tile_cols: int):
    """bsr2tilebsr (spmm/2d/block_spmm_2d_half_mma.cu:264-293): returns
    (blk_row_ptr, blk_col_idx) for row_tiles row tiles of
    (rows / row_tiles) block-rows and column tiles of tile_cols columns."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    rows = rp.size - 1
    tile_rows = rows // row_tiles
    brp = np.zeros(row_tiles * (cols // tile_cols) * tile_rows + 1, dtype=np.int32)
    bci = np.zeros(max(ci.size, 1), dtype=np.int32)
    if ci.size == 0:
        ci = np.zeros(1, dtype=np.int32)
    n = lib().kami_oracle_bsr2tilebsr(row_tiles, tile_rows, cols, tile_cols, _p(rp, _ip), _p(ci, _ip),
                                      _p(brp, _ip), _p(bci, _ip))
    return brp, bci[:n].copy()


def spmm(row_ptr, col_idx, values, block_cols: int, B, b_layout: str = "ref_nk", tile_rows: int = 1,
         tile_cols: int = 0) -> np.ndarray:
    """Host check of the block SpMM programs (spmm/1d/...:305-326; tiled form
    spmm/2d/...:385-408): C [16 rows, N] in double, values as given (tiles in
    entry order), B [N, K] (ref_nk) or [K, N] (row_kn)."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    if ci.size == 0:
        ci = np.zeros(1, dtype=np.int32)
    v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
    if v.size == 0:
        v = np.zeros(256)
    Bd = np.ascontiguousarray(np.asarray(B, dtype=np.float64))
    N = Bd.shape[0] if b_layout == "ref_nk" else Bd.shape[1]
    ntiles = block_cols // tile_cols if tile_cols else 1
    mb = (rp.size - 1) // ntiles
    C = np.zeros((mb * 16, N))
    lib().kami_oracle_spmm(mb, block_cols, N, tile_rows, tile_cols, _p(rp, _ip), _p(ci, _ip), _p(v, _dp),
                           _p(Bd, _dp), Bd.shape[1], 0 if b_layout == "ref_nk" else 1, _p(C, _dp), N)
    return C


def bsr_pattern(rows: int, cols: int, density: float, seed: int):
    """Independent Bernoulli(density) block pattern from a seeded LCG."""
    cap = max(int(rows * cols * density * 1.5) + 64, 64)
    while True:
        row_ptr = np.zeros(rows + 1, dtype=np.int32)
        col_idx = np.zeros(cap, dtype=np.int32)
        n = lib().kami_oracle_bsr_pattern(rows, cols, density, seed, _p(row_ptr, _ip), _p(col_idx, _ip), cap)
        if n >= 0:
            return row_ptr, col_idx[:n].copy()
        cap *= 2


# --------------------------------------------------------------------------
# dense GEMM
# --------------------------------------------------------------------------

def gemm(A: np.ndarray, B: np.ndarray, b_layout: int = B_REF_NK) -> np.ndarray:
    """Batched C = A * op(B) with a double accumulator, i-j-k order
    (batched_gemm_2d_double_mma.cu:338-352; block_gemm_1d_half_mma.cu:269-279).

    A: [batch, M, K]; B: [batch, N, K] (REF_NK) or [batch, K, N] (ROW_KN).
    float64, float16 or bfloat16-as-uint16 (pass dtype np.uint16 and
    ``bf16=True`` via :func:`gemm_bf16`).  Returns float64 [batch, M, N]."""
    return _gemm(A, B, b_layout, bf16=False)


def gemm_bf16(A_bits: np.ndarray, B_bits: np.ndarray, b_layout: int = B_REF_NK) -> np.ndarray:
    return _gemm(A_bits, B_bits, b_layout, bf16=True)


def _gemm(A, B, b_layout, bf16):
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    if A.ndim == 2:
        A = A[None]
    if B.ndim == 2:
        B = B[None]
    batch, M, K = A.shape
    if b_layout == B_REF_NK:
        N = B.shape[1]
        ldb = K
    else:
        N = B.shape[2]
        ldb = N
    C = np.zeros((batch, M, N), dtype=np.float64)
    if A.dtype == np.float64:
        lib().kami_oracle_gemm_f64(batch, M, N, K, _p(A, _dp), K, M * K, _p(B, _dp), ldb, N * K, b_layout,
                                   _p(C, _dp), N, M * N)
    else:
        a16 = A.view(np.uint16)
        b16 = B.view(np.uint16)
        lib().kami_oracle_gemm_h16(batch, M, N, K, _p(a16, _u16p), K, M * K, _p(b16, _u16p), ldb, N * K,
                                   b_layout, 1 if bf16 else 0, _p(C, _dp), N, M * N)
    return C


def reduce_slices(Cp: np.ndarray, P: int) -> np.ndarray:
    """Host reduction of P partial C slices per problem
    (batched_gemm_3d_double_mma.cu:361-373).  Cp: [batch, P, M, N]."""
    Cp = np.ascontiguousarray(Cp, dtype=np.float64)
    batch, P2, M, N = Cp.shape
    assert P2 == P
    out = np.empty((batch, M, N), dtype=np.float64)
    lib().kami_oracle_reduce_slices_f64(batch, P, M, N, _p(Cp, _dp), _p(out, _dp))
    return out


def gemm_dd(A: np.ndarray, B: np.ndarray, b_layout: int = B_REF_NK):
    """Double-double C = A * op(B) (TwoSum/TwoProd, Dot2).  Returns (hi, lo)."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    batch, M, K = A.shape
    N = B.shape[1] if b_layout == B_REF_NK else B.shape[2]
    ldb = K if b_layout == B_REF_NK else N
    hi = np.empty((batch, M, N))
    lo = np.empty((batch, M, N))
    lib().kami_oracle_gemm_dd(batch, M, N, K, _p(A, _dp), K, M * K, _p(B, _dp), ldb, N * K, b_layout,
                              _p(hi, _dp), _p(lo, _dp), N, M * N)
    return hi, lo


def normwise_error_dd(C: np.ndarray, hi: np.ndarray, lo: np.ndarray) -> float:
    C = np.ascontiguousarray(C, dtype=np.float64)
    return float(lib().kami_oracle_normwise_error_dd(C.size, _p(C, _dp), _p(hi, _dp), _p(lo, _dp)))


# --------------------------------------------------------------------------
# block SpGEMM
# --------------------------------------------------------------------------

def spgemm(mA, nB, A, B, accum: str = "double"):
    """spgemm_spa (block_spgemm_2d_half_mma.cu:557-646).

    A = (row_ptr, col_idx, vals[nnz, bsr, bsr] float16), B likewise.
    accum="half" reproduces the reference's binary16 dense row exactly;
    accum="double" accumulates in double (the FP32-accumulating kernels are
    checked against it).  Returns (RowPtrC, ColIdxC, ValC[nnzC, bsr, bsr])."""
    rpa, cia, va = (np.ascontiguousarray(x) for x in A)
    rpb, cib, vb = (np.ascontiguousarray(x) for x in B)
    rpa = rpa.astype(np.int32)
    cia = cia.astype(np.int32)
    rpb = rpb.astype(np.int32)
    cib = cib.astype(np.int32)
    bsr = va.shape[-1] if va.size else vb.shape[-1]
    rpc = np.zeros(mA + 1, dtype=np.int32)
    L = lib()
    nnzc = L.kami_oracle_spgemm_symbolic(mA, nB, _p(rpa, _ip), _p(cia, _ip), _p(rpb, _ip), _p(cib, _ip),
                                         _p(rpc, _ip))
    cic = np.zeros(max(nnzc, 1), dtype=np.int32)
    va16 = np.ascontiguousarray(va, dtype=np.float16).view(np.uint16)
    vb16 = np.ascontiguousarray(vb, dtype=np.float16).view(np.uint16)
    if accum == "half":
        vc16 = np.zeros(max(nnzc, 1) * bsr * bsr, dtype=np.uint16)
        vc64 = np.zeros(1)
        mode = 0
    else:
        vc16 = np.zeros(1, dtype=np.uint16)
        vc64 = np.zeros(max(nnzc, 1) * bsr * bsr)
        mode = 1
    L.kami_oracle_spgemm_numeric(mA, nB, bsr, _p(rpa, _ip), _p(cia, _ip), _p(va16, _u16p), _p(rpb, _ip),
                                 _p(cib, _ip), _p(vb16, _u16p), _p(rpc, _ip), _p(cic, _ip), mode,
                                 _p(vc16, _u16p), _p(vc64, _dp))
    if mode == 0:
        vals = vc16[: nnzc * bsr * bsr].view(np.float16).reshape(nnzc, bsr, bsr)
    else:
        vals = vc64[: nnzc * bsr * bsr].reshape(nnzc, bsr, bsr)
    return rpc, cic[:nnzc].copy(), vals.copy()


def spgemm_row_ptr(mA, nB, row_ptr_a, col_idx_a, row_ptr_b, col_idx_b):
    """RowPtrC of the SPA symbolic pass alone (block_spgemm_2d_half_mma.cu:557-600)."""
    rpa, cia, rpb, cib = (np.ascontiguousarray(x, dtype=np.int32) for x in (row_ptr_a, col_idx_a, row_ptr_b,
                                                                            col_idx_b))
    rpc = np.zeros(mA + 1, dtype=np.int32)
    lib().kami_oracle_spgemm_symbolic(mA, nB, _p(rpa, _ip), _p(cia, _ip), _p(rpb, _ip), _p(cib, _ip), _p(rpc, _ip))
    return rpc


def spgemm_nnzcub(col_idx_a: np.ndarray, row_ptr_b: np.ndarray) -> int:
    """nnzCub (block_spgemm_2d_half_mma.cu:763-768)."""
    cia = np.ascontiguousarray(col_idx_a, dtype=np.int32)
    rpb = np.ascontiguousarray(row_ptr_b, dtype=np.int32)
    return int(lib().kami_oracle_spgemm_nnzcub(len(cia), _p(cia, _ip), _p(rpb, _ip)))


# --------------------------------------------------------------------------
# reference libraries (oracle/_ref)
# --------------------------------------------------------------------------

def ref_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{name}.so"))


def ref_lib(name: str):
    L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_{name}.so"))
    if hasattr(L, "kami_ref_launch"):
        L.kami_ref_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i32]
        L.kami_ref_launch.restype = _i32
        L.kami_ref_config.argtypes = [_ip]
    if hasattr(L, "kami_ref_spmm_launch"):
        L.kami_ref_spmm_launch.argtypes = [ctypes.c_void_p] * 5 + [_i32]
        L.kami_ref_spmm_launch.restype = _i32
        L.kami_ref_spmm_config.argtypes = [_ip]
        L.kami_ref_bsr_generate.argtypes = [_i32, _i32, ctypes.c_float, _ip, _ip, _u16p]
        L.kami_ref_bsr_generate.restype = _i32
        L.kami_ref_bsr_size.restype = _i32
        if hasattr(L, "kami_ref_bsr2tilebsr"):
            L.kami_ref_bsr2tilebsr.argtypes = [_i32, _i32, _i32, _ip, _ip, _ip, _ip]
    if hasattr(L, "kami_ref_spgemm_spa"):
        L.kami_ref_bsr_generate.argtypes = [_i32, _i32, ctypes.c_float, _ip, _ip, _u16p]
        L.kami_ref_bsr_generate.restype = _i32
        L.kami_ref_spgemm_spa.argtypes = [_i32, _i32, _ip, _ip, _u16p, _i32, _ip, _ip, _u16p, _ip, _ip, _u16p]
        L.kami_ref_spgemm_spa.restype = _i32
        L.kami_ref_bsr_size.restype = _i32
    return L


def ref_config(L) -> dict:
    cfg = (ctypes.c_int * 8)()
    L.kami_ref_config(cfg)
    keys = ["M", "N", "K", "P", "num_iter", "threads", "slices", "smem"]
    return dict(zip(keys, list(cfg)))


def ref_spmm_config(L) -> dict:
    cfg = (ctypes.c_int * 9)()
    L.kami_ref_spmm_config(cfg)
    keys = ["M", "N", "K", "P", "num_iter", "threads", "slices", "tile_rows", "tile_cols"]
    return dict(zip(keys, list(cfg)))


def ref_bsr2tilebsr(L, row_ptr, col_idx, cols: int, row_tiles: int, tile_cols: int):
    """The reference's own bsr2tilebsr (compiled from its 2D/3D SpMM file)."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    rows = rp.size - 1
    tile_rows = rows // row_tiles
    brp = np.zeros(row_tiles * (cols // tile_cols) * tile_rows + 1, dtype=np.int32)
    bci = np.zeros(max(ci.size, 1), dtype=np.int32)
    if ci.size == 0:
        ci = np.zeros(1, dtype=np.int32)
    L.kami_ref_bsr2tilebsr(rows, cols, int(rp[-1]) * 256, _p(rp, _ip), _p(ci, _ip), _p(brp, _ip), _p(bci, _ip))
    return brp, bci[: int(brp[-1])].copy()


def ref_bsr_generate(L, rows, cols, sparsity):
    bsr = L.kami_ref_bsr_size()
    row_ptr = np.zeros(rows + 1, dtype=np.int32)
    col_idx = np.zeros(max(rows * cols, 1), dtype=np.int32)
    vals = np.zeros(max(rows * cols, 1) * bsr * bsr, dtype=np.uint16)
    nnz = L.kami_ref_bsr_generate(rows, cols, sparsity, _p(row_ptr, _ip), _p(col_idx, _ip), _p(vals, _u16p))
    return row_ptr, col_idx[:nnz].copy(), vals[: nnz * bsr * bsr].view(np.float16).reshape(nnz, bsr, bsr).copy()


def ref_spgemm_spa(L, mA, nA, nB, A, B):
    bsr = L.kami_ref_bsr_size()
    rpa, cia, va = A
    rpb, cib, vb = B
    rpa = np.ascontiguousarray(rpa, dtype=np.int32)
    cia = np.ascontiguousarray(cia, dtype=np.int32)
    rpb = np.ascontiguousarray(rpb, dtype=np.int32)
    cib = np.ascontiguousarray(cib, dtype=np.int32)
    va16 = np.ascontiguousarray(va, dtype=np.float16).view(np.uint16).ravel()
    vb16 = np.ascontiguousarray(vb, dtype=np.float16).view(np.uint16).ravel()
    if va16.size == 0:
        va16 = np.zeros(1, dtype=np.uint16)
    if vb16.size == 0:
        vb16 = np.zeros(1, dtype=np.uint16)
    if cia.size == 0:
        cia = np.zeros(1, dtype=np.int32)
    if cib.size == 0:
        cib = np.zeros(1, dtype=np.int32)
    cap = max(mA * nB, 1)
    rpc = np.zeros(mA + 1, dtype=np.int32)
    cic = np.zeros(cap, dtype=np.int32)
    vc = np.zeros(cap * bsr * bsr, dtype=np.uint16)
    nnzc = L.kami_ref_spgemm_spa(mA, nA, _p(rpa, _ip), _p(cia, _ip), _p(va16, _u16p), nB, _p(rpb, _ip),
                                 _p(cib, _ip), _p(vb16, _u16p), _p(rpc, _ip), _p(cic, _ip), _p(vc, _u16p))
    return rpc, cic[:nnzc].copy(), vc[: nnzc * bsr * bsr].view(np.float16).reshape(nnzc, bsr, bsr).copy()
