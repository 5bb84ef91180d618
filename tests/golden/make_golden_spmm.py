"""Generate the block-SpMM golden vectors from the reference's own kernels.

Runs on a machine with a GPU.  The kernels are the reference's
block_spmm_{1d,2d,3d}_half_mma, compiled from its sources by
oracle/Makefile.ref into oracle/_ref/ at M = N = K = 64 (1D with P = 4 and
its fixed NUM_ITER = 1000; 2D and 3D with P = 2 and NUM_ITER = 1).  They
accumulate in FP16, so the inputs keep every partial sum an exact integer:

* 2D / 3D: exactly the reference programs' inputs -- generate_random_bsr_matrix
  (srand(0), sparsity 0.5, values rand() % 2 + 1), then B[i] = rand() % 2 + 1
  continuing the same C-library rand() stream (spmm/2d/...:311-318), then
  bsr2tilebsr; values stay in BSR order, as the reference passes them.
  Partial sums are at most 64 * 4.
* 1D (NUM_ITER = 1000 repeats): the reference generator's block pattern,
  with tile values chosen so that every row of A has at most two ones, and
  B in {0, 1}: every C entry is at most 2, so 1000 repeats stay below 2048.
  The golden C is the kernel's output divided by 1000.

Each case is stored as tests/golden/spmm_<name>.npz = {row_ptr, col_idx,
vals (float16 [e, 16, 16]), B (float16 [N, K]), C (float64 [M, N]), cfg}.

Usage: python tests/golden/make_golden_spmm.py OUTDIR
"""
import ctypes
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402


def run(L, rp, ci, vals, B, M, N, slices):
    d_rp = torch.tensor(rp, dtype=torch.int32, device="cuda")
    d_ci = torch.tensor(ci if ci.size else np.zeros(1, np.int32), dtype=torch.int32, device="cuda")
    d_v = torch.tensor(vals.astype(np.float32), device="cuda").half().contiguous()
    d_B = torch.tensor(B.astype(np.float32), device="cuda").half().contiguous()
    d_C = torch.zeros(slices * M * N, dtype=torch.float16, device="cuda")
    rc = L.kami_ref_spmm_launch(d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), d_B.data_ptr(), d_C.data_ptr(), 1)
    if rc != 0:
        raise RuntimeError(f"reference launch returned cudaError {rc}")
    return d_C.double().cpu().numpy().reshape(slices, M, N).sum(axis=0)


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    libc = ctypes.CDLL(None)

    # 1D: fixed NUM_ITER = 1000, exact-by-construction inputs
    L = oracle.ref_lib("spmm1d_64p4")
    cfg = oracle.ref_spmm_config(L)
    M, N, K = cfg["M"], cfg["N"], cfg["K"]
    rp, ci, _ = oracle.ref_bsr_generate(L, M // 16, K // 16, 0.5)
    rng = np.random.default_rng(7)
    vals = np.zeros((ci.size, 16, 16))
    for r in range(M):
        br, rr = divmod(r, 16)
        ents = list(range(rp[br], rp[br + 1]))
        for _ in range(min(2, len(ents))):
            e = ents[rng.integers(len(ents))]
            vals[e, rr, rng.integers(16)] = 1.0
    B = rng.integers(0, 2, (N, K)).astype(np.float64)
    C = run(L, rp, ci, vals, B, M, N, cfg["slices"]) / cfg["num_iter"]
    np.savez_compressed(os.path.join(outdir, "spmm_1d_64p4.npz"), row_ptr=rp, col_idx=ci,
                        vals=vals.astype(np.float16), B=B.astype(np.float16), C=C,
                        cfg=np.array([M, N, K, cfg["P"], 1, 0, cfg["num_iter"]], dtype=np.int64))
    print("1d", cfg, "max", C.max())

    # 2D / 3D: the reference programs' own inputs
    for name in ("spmm2d_64p2", "spmm3d_64p2"):
        L = oracle.ref_lib(name)
        cfg = oracle.ref_spmm_config(L)
        M, N, K = cfg["M"], cfg["N"], cfg["K"]
        rows, cols = M // 16, K // 16
        rp, ci, vals = oracle.ref_bsr_generate(L, rows, cols, 0.5)
        B = np.array([libc.rand() % 2 + 1.0 for _ in range(K * N)]).reshape(N, K)
        brp, bci = oracle.ref_bsr2tilebsr(L, rp, ci, cols, rows // cfg["tile_rows"], cfg["tile_cols"])
        C = run(L, brp, bci, vals.astype(np.float64), B, M, N, cfg["slices"])
        np.savez_compressed(os.path.join(outdir, f"spmm_{name[4:]}.npz"), row_ptr=brp, col_idx=bci,
                            vals=vals.astype(np.float16), B=B.astype(np.float16), C=C,
                            cfg=np.array([M, N, K, cfg["P"], cfg["tile_rows"], cfg["tile_cols"], cfg["num_iter"]],
                                         dtype=np.int64))
        print(name, cfg, "max", C.max())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
