"""Generate the SpGEMM golden vectors from the reference's own host code.

generate_random_bsr_matrix and spgemm_spa of
src/sparse/spgemm/2d/block_spgemm_2d_half_mma.cu (compiled from the reference
sources by oracle/Makefile.ref into oracle/_ref/libref_spgemm2d_host.so) are
run on the CPU exactly as the reference's main() runs them: A and B from the
generator (srand(0) each time, so square patterns coincide), then the SPA
symbolic and numeric passes with the binary16 dense row.  Each case is
stored as tests/golden/spgemm_<rows>x<cols>_s<sparsity>.npz.

Usage: python tests/golden/make_golden_spgemm.py [OUTDIR]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

# (block rows of A, block cols of A = block rows of B, block cols of B, sparsity)
CASES = [(8, 8, 8, 0.5), (12, 8, 12, 0.3), (8, 8, 8, 0.0), (4, 4, 4, 0.9), (16, 16, 16, 0.7)]


def main(outdir):
    L = oracle.ref_lib("spgemm2d_host")
    for (m, k, n, sp) in CASES:
        A = oracle.ref_bsr_generate(L, m, k, sp)
        B = oracle.ref_bsr_generate(L, k, n, sp)
        C = oracle.ref_spgemm_spa(L, m, k, n, A, B)
        fn = os.path.join(outdir, f"spgemm_{m}x{k}x{n}_s{sp}.npz")
        np.savez_compressed(fn, shape=np.array([m, k, n]), sparsity=np.array([sp]),
                            a_row_ptr=A[0], a_col_idx=A[1], a_vals=A[2],
                            b_row_ptr=B[0], b_col_idx=B[1], b_vals=B[2],
                            c_row_ptr=C[0], c_col_idx=C[1], c_vals=C[2])
        print(fn, "nnzA", len(A[1]), "nnzB", len(B[1]), "nnzC", len(C[1]))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
