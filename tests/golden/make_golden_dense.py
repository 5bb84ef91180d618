"""Generate the dense golden vectors from the reference's own kernels.

Runs on a machine with a GPU.  The kernels are the reference's, compiled from
its sources by oracle/Makefile.ref into oracle/_ref/ (one library per kernel
and compile-time shape).  Inputs are filled exactly as the reference's
batched programs fill them: x[i] = rand_r(&i) % 3 over the flat index
(batched_gemm_2d_double_mma.cu:271-285), for A and then for B, so every
product is an exact small integer.  Each output is stored as
tests/golden/dense_<name>.npz = {C (float64, [grid, slices, M, N]), cfg}.

Usage: python tests/golden/make_golden_dense.py OUTDIR
"""
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

NAMES = ["batched1d_f64_32p2", "batched1d_f64_64p4", "batched2d_f64_32p2", "batched2d_f64_64p2",
         "batched3d_f64_32p2", "block1d_f64_32p2", "block2d_f16_64p2", "block3d_f16_64p2"]
BATCH = 4


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name in NAMES:
        L = oracle.ref_lib(name)
        cfg = oracle.ref_config(L)
        M, N, K, S = cfg["M"], cfg["N"], cfg["K"], cfg["slices"]
        grid = BATCH if name.startswith("batched") else 1
        A = oracle.fill_rand_r_mod(grid * M * K)
        B = oracle.fill_rand_r_mod(grid * N * K)
        dt = torch.float16 if "_f16_" in name else torch.float64
        dA = torch.tensor(A, dtype=dt, device="cuda")
        dB = torch.tensor(B, dtype=dt, device="cuda")
        dC = torch.zeros(grid * S * M * N, dtype=dt, device="cuda")
        rc = L.kami_ref_launch(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), grid)
        if rc != 0:
            raise RuntimeError(f"{name}: reference launch returned cudaError {rc}")
        C = dC.double().cpu().numpy().reshape(grid, S, M, N)
        np.savez_compressed(os.path.join(outdir, f"dense_{name}.npz"), C=C,
                            cfg=np.array([M, N, K, cfg["P"], cfg["num_iter"], S, grid], dtype=np.int64))
        print(name, cfg, "max", C.max())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
