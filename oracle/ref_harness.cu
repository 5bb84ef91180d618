// ref_harness.cu -- builds pieces of the KAMI reference, from its own sources
// where they lie, into small shared libraries under oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: these libraries pin the CPU oracle
// (oracle/kami_oracle.c) against the reference's own code.  Nothing in the
// product library links or loads them.
//
// The reference is a set of stand-alone benchmark programs, each one .cu file
// with one kernel, a main() and compile-time -D macros.  This harness renames
// the program's main() out of the way, includes the .cu file named by
// KAMI_REF_SOURCE, and exports C entry points around the reference's own
// functions:
//   * KAMI_REF_KERNEL set: a launcher for the dense kernel of that file with
//     the file's own dynamic shared-memory size and block size
//     (the launch of batched_gemm_2d_double_mma.cu:303-307 and friends);
//   * KAMI_REF_SPGEMM_HOST set: the host functions generate_random_bsr_matrix
//     and spgemm_spa of the block SpGEMM files (CPU only);
//   * KAMI_REF_SPMM set: a launcher for the block SpMM kernel of that file
//     (block_spmm_{1d,2d,3d}_half_mma) with the file's own launch geometry,
//     plus its generate_random_bsr_matrix and (2D/3D) bsr2tilebsr.
// Oracle/Makefile.ref lists the variants and their -D macros.
#include <cstdint>
#include <cuda_runtime.h>

#define main kami_reference_program_main
#include KAMI_REF_SOURCE
#undef main

#ifndef KAMI_REF_SLICES
#define KAMI_REF_SLICES 1
#endif

#if defined(KAMI_REF_KERNEL)

#ifndef KAMI_REF_T
#error "KAMI_REF_T (the element type of the kernel) must be defined"
#endif

extern "C" int kami_ref_launch(const void *A, const void *B, void *C, int grid)
{
    cudaError_t e = cudaFuncSetAttribute(KAMI_REF_KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         shmem_size_block_gemm);
    if (e != cudaSuccess)
        return (int)e;
    KAMI_REF_KERNEL<<<grid, NUM_ALLOC_RANK_BLOCK * WARP_SIZE, shmem_size_block_gemm>>>(
        (const KAMI_REF_T *)A, (const KAMI_REF_T *)B, (KAMI_REF_T *)C, (KAMI_REF_T)1.0, (KAMI_REF_T)0.0);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return (int)e;
    return (int)cudaDeviceSynchronize();
}

// {M, N, K, P, NUM_ITER, threads per block, C slices per problem, smem bytes}
extern "C" void kami_ref_config(int *cfg)
{
    cfg[0] = M_BLOCK;
    cfg[1] = N_BLOCK;
    cfg[2] = K_BLOCK;
    cfg[3] = NUM_RANK_BLOCK;
    cfg[4] = NUM_ITER;
    cfg[5] = NUM_ALLOC_RANK_BLOCK * WARP_SIZE;
    cfg[6] = KAMI_REF_SLICES;
    cfg[7] = shmem_size_block_gemm;
}

#elif defined(KAMI_REF_SPGEMM_HOST)

// Values cross this boundary as binary16 bit patterns (the reference's half).
extern "C" int kami_ref_bsr_generate(int rows, int cols, float sparsity, int *row_ptr, int *col_idx,
                                     uint16_t *values)
{
    int nnz = 0;
    generate_random_bsr_matrix(rows, cols, sparsity, row_ptr, col_idx, reinterpret_cast<half *>(values), &nnz);
    return nnz / (BSR_M * BSR_K);
}

// Symbolic then numeric spgemm_spa, exactly as the reference's main() calls
// it (block_spgemm_2d_half_mma.cu:749-761).  RowPtrC has mA + 1 entries;
// ColIdxC / ValC must hold the worst case (mA * nB blocks).  Returns nnzC in
// blocks.
extern "C" int kami_ref_spgemm_spa(int mA, int nA, const int *RowPtrA, const int *ColIdxA, const uint16_t *ValA,
                                   int nB, const int *RowPtrB, const int *ColIdxB, const uint16_t *ValB,
                                   int *RowPtrC, int *ColIdxC, uint16_t *ValC)
{
    int nnzA = RowPtrA[mA] * BSR_M * BSR_K;
    int nnzB = RowPtrB[nA] * BSR_K * BSR_N;
    int nnzC = 0;
    spgemm_spa(RowPtrA, ColIdxA, reinterpret_cast<const half *>(ValA), mA, nA, nnzA, RowPtrB, ColIdxB,
               reinterpret_cast<const half *>(ValB), nA, nB, nnzB, RowPtrC, ColIdxC,
               reinterpret_cast<half *>(ValC), mA, nB, &nnzC, 1);
    spgemm_spa(RowPtrA, ColIdxA, reinterpret_cast<const half *>(ValA), mA, nA, nnzA, RowPtrB, ColIdxB,
               reinterpret_cast<const half *>(ValB), nA, nB, nnzB, RowPtrC, ColIdxC,
               reinterpret_cast<half *>(ValC), mA, nB, &nnzC, 0);
    return nnzC / (BSR_M * BSR_N);
}

extern "C" int kami_ref_bsr_size(void) { return BSR_M; }

#elif defined(KAMI_REF_SPMM)

// The file's kernel on its own launch geometry (e.g. spmm/1d/...:283-285):
// index arrays as the kernel takes them (BSR for 1D, tiled BSR for 2D/3D).
extern "C" int kami_ref_spmm_launch(const int *rowptr, const int *colidx, const void *vals, const void *B, void *C,
                                    int grid)
{
    cudaError_t e =
        cudaFuncSetAttribute(KAMI_REF_SPMM, cudaFuncAttributeMaxDynamicSharedMemorySize, shmem_size_block_spmm);
    if (e != cudaSuccess)
        return (int)e;
    KAMI_REF_SPMM<<<grid, KAMI_REF_SPMM_THREADS, shmem_size_block_spmm>>>(
        rowptr, colidx, (const half *)vals, (const half *)B, (half *)C, (half)1.0, (half)0.0);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return (int)e;
    return (int)cudaDeviceSynchronize();
}

// {M, N, K, P, NUM_ITER, threads per block, C slices, tile rows, tile cols}
extern "C" void kami_ref_spmm_config(int *cfg)
{
    cfg[0] = M_BLOCK;
    cfg[1] = N_BLOCK;
    cfg[2] = K_BLOCK;
    cfg[3] = NUM_RANK_BLOCK;
    cfg[4] = NUM_ITER;
    cfg[5] = KAMI_REF_SPMM_THREADS;
    cfg[6] = KAMI_REF_SLICES;
#ifdef NUMS_ROW
    cfg[7] = NUMS_ROW;
    cfg[8] = NUMS_COL;
#else
    cfg[7] = 0;
    cfg[8] = 0;
#endif
}

extern "C" int kami_ref_bsr_generate(int rows, int cols, float sparsity, int *row_ptr, int *col_idx,
                                     uint16_t *values)
{
    int nnz = 0;
    generate_random_bsr_matrix(rows, cols, sparsity, row_ptr, col_idx, reinterpret_cast<half *>(values), &nnz);
    return nnz / (BSR_M * BSR_K);
}

extern "C" int kami_ref_bsr_size(void) { return BSR_M; }

#ifdef NUMS_ROW
extern "C" void kami_ref_bsr2tilebsr(int rows, int cols, int bsr_nnz, const int *bsr_rowptr, const int *bsr_colidx,
                                     int *blk_rowptr, int *blk_colidx)
{
    bsr2tilebsr(rows, cols, bsr_nnz, 0.5f, const_cast<int *>(bsr_rowptr), const_cast<int *>(bsr_colidx), blk_rowptr,
                blk_colidx);
}
#endif

#else
#error "define KAMI_REF_KERNEL, KAMI_REF_SPGEMM_HOST or KAMI_REF_SPMM"
#endif
