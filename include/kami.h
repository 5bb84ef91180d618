/*
 * kami.h -- C ABI of kami_b200, a B200-native (sm_100a) implementation of the
 * KAMI block-GEMM / block-SpGEMM path.
 *
 * The reference (KAMI) has no library ABI: each benchmark program owns one
 * __global__ kernel whose shape and partition are compile-time -D macros and
 * whose launch is <<<batch, NUM_ALLOC_RANK_BLOCK*32, smem>>> on the default
 * stream.  Every entry point below replaces one of those kernel launches
 * (cited per function, paths inside the KAMI project) and keeps the
 * reference's knobs as run-time arguments: precision, M/N/K, partition
 * (1D/2D/3D), warp-rank count P (NUM_RANK_BLOCK), allocated warps
 * (NUM_ALLOC_RANK_BLOCK) and in-register repeat count (NUM_ITER).
 *
 * Conventions
 *   - Every function returns int: 0 (KAMI_OK) or a negative kami_status.
 *     No C++ exception crosses this boundary.
 *   - All pointers to matrix data are DEVICE pointers.  Index arrays
 *     (row_ptr/col_idx) are device int32.  The caller allocates every device
 *     buffer, as in the reference.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls are stream-ordered and do not synchronise the host,
 *     except where a function says so.
 *   - Leading dimensions (ld*) are row strides in elements; stride* are
 *     per-problem strides in elements.
 *   - Layouts: A is M x K row-major (KAMI_A_ROW_MK) or stored transposed
 *     (K x M row-major, KAMI_A_COL_MK).  B is the reference's N x K
 *     row-major operand (KAMI_B_REF_NK: h_B[j*K+k], batched_gemm_2d_double_
 *     mma.cu:348) or K x N row-major (KAMI_B_ROW_KN).  C is M x N row-major.
 */
#ifndef KAMI_B200_H
#define KAMI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum kami_status {
    KAMI_OK = 0,
    KAMI_ERR_INVALID_VALUE = -1, /* bad shape, null pointer, bad enum     */
    KAMI_ERR_UNSUPPORTED = -2,   /* valid request with no kernel for it    */
    KAMI_ERR_MISALIGNED = -3,    /* pointer / leading-dimension alignment  */
    KAMI_ERR_WORKSPACE = -4,     /* workspace missing or too small         */
    KAMI_ERR_CUDA = -5,          /* a CUDA runtime call failed             */
    KAMI_ERR_TIMEOUT = -6,       /* a bounded device wait gave up          */
    KAMI_ERR_INTERNAL = -7
} kami_status_t;

typedef enum kami_dtype {
    KAMI_F16 = 0,
    KAMI_BF16 = 1,
    KAMI_F64 = 2,
    KAMI_F32 = 3,
    KAMI_S8 = 4 /* signed 8-bit integer: digit slices of kami_split_f64_gemm_batched only */
} kami_dtype_t;

typedef enum kami_partition {
    KAMI_PARTITION_AUTO = 0,
    KAMI_PARTITION_1D = 1, /* warps split M; B slices broadcast per stage            */
    KAMI_PARTITION_2D = 2, /* P x P warps; A along rows, B along columns (SUMMA)     */
    KAMI_PARTITION_3D = 3  /* P x P x P warps; K split in depth, reduced on device   */
} kami_partition_t;

typedef enum kami_variant {
    KAMI_VARIANT_AUTO = 0,
    KAMI_VARIANT_MMA_SYNC = 1, /* warp mma.sync, register-resident operands        */
    KAMI_VARIANT_TCGEN05 = 2,  /* tcgen05.mma, TMA-staged operands, TMEM accumulators */
    KAMI_VARIANT_TCGEN05_TS = 3 /* tcgen05.mma with A resident in tensor memory (M 65..128) */
} kami_variant_t;

typedef enum kami_a_layout { KAMI_A_ROW_MK = 0, KAMI_A_COL_MK = 1 } kami_a_layout_t;
typedef enum kami_b_layout { KAMI_B_REF_NK = 0, KAMI_B_ROW_KN = 1 } kami_b_layout_t;

/* ------------------------------------------------------------------------ */
/* Library                                                                  */
/* ------------------------------------------------------------------------ */

/* Human-readable text of the last error raised on the calling host thread. */
const char *kami_last_error_string(void);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int kami_version(void);

/* Read and clear the device-side status word that kernels with bounded
 * waits set when a wait gives up instead of hanging (no counterpart in the
 * reference, whose kernels have no waits).  *code receives 0 when no wait
 * timed out; the return value is KAMI_ERR_TIMEOUT when one did.  Synchronises
 * with the device. */
int kami_device_status(int *code);

/* Failure-detection self test (no counterpart in the reference): launch a
 * one-thread kernel that waits, with the library's bounded wait, on an
 * mbarrier that nothing arrives at.  The wait gives up after timeout_ns
 * (<= 10 s) and records a timeout, which the next kami_device_status call
 * reports as KAMI_ERR_TIMEOUT (code 4); the context stays usable. */
int kami_selftest_bounded_wait(uint64_t timeout_ns, void *stream);

/* ------------------------------------------------------------------------ */
/* Batched block GEMM                                                       */
/* ------------------------------------------------------------------------ */

/*
 * C[b] = alpha * sum_{iter < num_iter} A[b] * op(B[b]) + beta * C[b],
 * for b < batch, one problem per CTA (one CTA may also hold several small
 * problems).  With num_iter > 1 the product is accumulated num_iter times in
 * the accumulator -- the reference's in-register repeat methodology
 * (NUM_ITER, block_gemm_1d_half_mma.cu:130), whose host check divides C by
 * NUM_ITER.
 *
 * Replaces the launches of
 *   block_gemm_{1d,2d,3d}_half_mma   (src/block_gemm/KAMI/{1d,2d,3d}/fp16/<file>.cu:61/64/61)
 *   block_gemm_{1d,2d,3d}_double_mma (src/block_gemm/KAMI/{1d,2d,3d}/fp64/<file>.cu:55/61/62)
 *   batched_gemm_{1d,2d,3d}_double_mma (src/batched_gemm/KAMI/{1d,2d,3d}/<file>.cu:59/65/64)
 * whose signature is (const T *A, const T *B, T *C, T alpha, T beta).  The
 * reference ignores alpha and beta; here they are applied.  The 3D partition
 * reduces its P partial C slices on the device instead of writing a P-times
 * larger C for a host reduction (batched_gemm_3d_double_mma.cu:361-373).
 *
 * in_type : KAMI_F16, KAMI_BF16 (FP32 accumulation) or KAMI_F64.
 * out_type: KAMI_F32, KAMI_F16 or KAMI_BF16 for 16-bit inputs; KAMI_F64
 *           for KAMI_F64 inputs.
 * P       : ranks per partition dimension (NUM_RANK_BLOCK); 0 = choose.
 * alloc_warps: warps launched per CTA (NUM_ALLOC_RANK_BLOCK); 0 = exactly
 *           the warps the partition uses.  Extra warps exit at once.
 * workspace / ws_bytes: device scratch; see kami_gemm_workspace_size (the
 *           current kernels need none; pass NULL, 0).
 */
int kami_gemm_batched(kami_dtype_t in_type, kami_dtype_t out_type,
                      kami_partition_t partition, kami_variant_t variant,
                      int M, int N, int K, int P, int alloc_warps,
                      int64_t batch,
                      const void *A, int64_t lda, int64_t strideA, kami_a_layout_t a_layout,
                      const void *B, int64_t ldb, int64_t strideB, kami_b_layout_t b_layout,
                      void *C, int64_t ldc, int64_t strideC,
                      double alpha, double beta, int num_iter,
                      void *workspace, size_t ws_bytes, void *stream);

/*
 * kami_gemm_batched on HOST buffers (C = num_iter * A B^T per problem, A
 * packed M x K row-major, B the reference's N x K row-major, C M x N; alpha 1,
 * beta 0): the reference's host sequence -- copy in, launch, copy out
 * (e.g. batched_gemm_2d_double_mma.cu) -- as one call, with the batch cut
 * into chunks of about one problem per four SMs (16 at most): the input
 * copies run back to back on one stream, the result copies on another, and
 * each chunk's product starts on one of the library's compute streams as
 * soon as its inputs have landed (one device buffer per chunk, a ring of
 * buffers above 1 GiB in all).  Host buffers should be pinned
 * (pageable memory works, without overlap) and stay valid until the work on
 * `stream` completes; `stream` waits for the last result copy.  workspace:
 * device memory of kami_gemm_batched_host_workspace_size bytes, or NULL for a
 * library-owned buffer (allocated on first use, grown as needed).  Calls are
 * serialised by a process-wide lock.
 */
int kami_gemm_batched_host(kami_dtype_t in_type, kami_dtype_t out_type,
                           kami_partition_t partition, kami_variant_t variant,
                           int M, int N, int K, int64_t batch,
                           const void *A, const void *B, void *C, int num_iter,
                           void *workspace, size_t ws_bytes, void *stream);
int kami_gemm_batched_host_workspace_size(kami_dtype_t in_type, kami_dtype_t out_type,
                                          int M, int N, int K, int64_t batch, size_t *bytes);

/* Bytes of device workspace kami_gemm_batched needs for this request. */
int kami_gemm_workspace_size(kami_dtype_t in_type, kami_partition_t partition,
                             kami_variant_t variant, int M, int N, int K, int P,
                             int64_t batch, size_t *bytes);

/*
 * Backward of the batched GEMM C = A B in the torch.bmm layout (A M x K,
 * B K x N, C M x N, row-major, problems packed at strides M K, K N, M N):
 * given dC, dA = dC B^T (M x K) and dB = A^T dC (K x N) in out_type; dA or
 * dB may be NULL to skip that gradient.  No counterpart in the reference (it
 * has no backward pass); this is the library's differentiation path.  FP16 /
 * BF16 with M, N, K in {64, 128} (and 16-byte aligned buffers) run ONE
 * tcgen05 kernel per problem that reads A, B and dC once and serves both
 * products from the same shared-memory tiles (dC is the K-major operand of
 * one product and the MN-major operand of the other); other requests run as
 * two kami_gemm_batched products.
 */
int kami_gemm_backward_batched(kami_dtype_t in_type, kami_dtype_t out_type,
                               int M, int N, int K, int64_t batch,
                               const void *A, const void *B, const void *dC,
                               void *dA, void *dB, void *stream);

/*
 * 1D mma.sync block GEMM with the K dimension split between registers and
 * shared memory: each rank keeps reg_k_steps k-steps (16 elements each) of
 * its A and B slices in registers and the rest in a shared-memory cache read
 * at every stage -- the residency trade-off the reference explores with one
 * compile-time split (src/reg_smem/block_gemm_1d_half_mma.cu:30-46,
 * REG_K_SPLIT_BLOCK).  It lets 1D 128^3 run with P = 4, whose all-register
 * form does not fit the register file.  FP16 / BF16 in, FP32 / FP16 / BF16
 * out; A M x K row-major, B the reference's N x K row-major; M, N, K up to
 * 128 (the smallest compiled square tile covering them: 64 or 128).
 * P = 0 lets the library pick P; reg_k_steps = -1 measures every compiled
 * split (and all-register form) of the tile on the caller's A and B with a
 * scratch C, once per request shape, and keeps the fastest -- the split as
 * an autotuner dimension.  *reg_k_used (if not NULL) receives the split run.
 */
int kami_gemm_batched_ksplit(kami_dtype_t in_type, kami_dtype_t out_type,
                             int M, int N, int K, int P, int64_t batch,
                             const void *A, int64_t lda, int64_t strideA,
                             const void *B, int64_t ldb, int64_t strideB,
                             void *C, int64_t ldc, int64_t strideC,
                             double alpha, double beta, int num_iter,
                             int reg_k_steps, int *reg_k_used, void *stream);

/*
 * Communication / computation cycle trace of one FP16 block GEMM (the
 * reference's src/usage_cycle/block_gemm_{1d,2d,3d}_half_mma_usage_cycle.cu,
 * which print clock() sums per warp): C (M x N, FP32) = A (M x K) B^T (B
 * N x K), one problem, num_iter repeats, on a traced instance of the given
 * partition and P (reg_k_steps as in kami_gemm_batched_ksplit for 1D; -1
 * otherwise).  cycles (device, 2 x 32 entries) receives per warp w
 * cycles[2w] = clock64 cycles spent publishing fragments and waiting at the
 * stage barriers, cycles[2w+1] = cycles spent reading fragments and issuing
 * MMAs, summed over every stage and repeat; *nwarps the warp count.
 * Compiled for 64^3 and 128^3 tiles (1D P = 2, 4, 8; 2D P = 2, 4; 3D P = 2).
 */
int kami_gemm_trace(kami_partition_t partition, int M, int N, int K, int P, int reg_k_steps,
                    const void *A, const void *B, void *C, int num_iter,
                    unsigned long long *cycles, int *nwarps, void *stream);

/*
 * Describe the kernel kami_gemm_batched would launch (after AUTO resolution):
 * out[0] = variant, out[1] = partition, out[2] = P, out[3] = threads per
 * CTA, out[4] = dynamic shared memory bytes, out[5] = problems per CTA,
 * out[6] = CTAs in the grid.  Host-only; launches nothing.
 */
int kami_gemm_describe(kami_dtype_t in_type, kami_dtype_t out_type,
                       kami_partition_t partition, kami_variant_t variant,
                       int M, int N, int K, int P, int alloc_warps, int64_t batch,
                       kami_a_layout_t a_layout, kami_b_layout_t b_layout, int out[8]);

/* ------------------------------------------------------------------------ */
/* Uneven (grouped) batched GEMM: one persistent launch                    */
/* ------------------------------------------------------------------------ */
/*
 * `count` independent problems C_i = alpha * A_i * B_i^T + beta * C_i with
 * their own M_i, N_i, K_i (each 1..128; K a multiple of 8 for 16-bit
 * inputs, of 2 for FP64).  A_i is M_i x K_i row-major at A + a_offsets[i],
 * B_i is N_i x K_i row-major (the reference layout) at B + b_offsets[i],
 * C_i is M_i x N_i row-major at C + c_offsets[i] (offsets in elements).
 * The reference runs one launch per compile-time shape
 * (batched_gemm_{1d,2d,3d}_double_mma.cu, one problem per CTA); here one
 * persistent launch runs every problem, each with the warp partition (1D /
 * 2D / 3D warp grid) chosen for its shape.
 *
 * kami_gemm_grouped_plan_create builds (host, synchronous) the device
 * descriptors and a longest-first schedule over persistent CTAs.  Three
 * kernels run a plan: the mma.sync kernel, whose eight warps split each
 * problem by its warp partition; (FP16 / BF16 inputs) the tcgen05 kernel,
 * which issues each problem's MMAs from one thread into tensor memory while
 * loader and epilogue warps stream the operands and C; and (FP64 inputs) the
 * staged DMMA kernel, whose loader warps stream K chunks into shared memory
 * while fourteen compute warps share each problem's C.  The tcgen05 kernel
 * is the default for FP16 / BF16, the staged kernel for FP64 (the warp-grid
 * kernel when problems of at most 32 x 32 carry most of the bytes);
 * KAMI_PLAN_MMA_SYNC / KAMI_PLAN_TCGEN05 / KAMI_PLAN_STAGED force one.  With
 * flags & KAMI_PLAN_AUTOTUNE the plan first measures every valid partition
 * per 16-rounded shape bucket on this device (cached per process) instead of
 * using the static cost model, and, unless a kernel is forced, times both
 * kernels on the whole plan and keeps the faster.  kami_gemm_grouped_run is
 * a single kernel launch that allocates nothing and synchronises nothing, so
 * it can be captured in a CUDA graph; the plan must outlive the graph.
 */
#define KAMI_PLAN_AUTOTUNE 1
#define KAMI_PLAN_MMA_SYNC 2
#define KAMI_PLAN_TCGEN05 4
#define KAMI_PLAN_STAGED 8
/* With this flag a tcgen05 plan puts up to four problems of at most 64 rows
 * and 64 columns (rounded to 16) in one work item -- their A rows stacked in
 * one 128-row tile, their B rows in another, C on the accumulator's diagonal
 * -- so one chain of MMAs and one accumulator hand-off serve them all.  Off
 * by default: on the 20000-problem 8..128 mix it measured slower (0.104 ms
 * against 0.096 ms one problem per item). */
#define KAMI_PLAN_PACK 16
typedef struct kami_grouped_plan kami_grouped_plan;

int kami_gemm_grouped_plan_create(kami_dtype_t in_type, kami_dtype_t out_type, int count,
                                  const int *M, const int *N, const int *K,
                                  const int64_t *a_offsets, const int64_t *b_offsets,
                                  const int64_t *c_offsets, int flags, kami_grouped_plan **plan);
int kami_gemm_grouped_run(const kami_grouped_plan *plan, const void *A, const void *B, void *C,
                          double alpha, double beta, int num_iter, void *stream);
/* out[0] = problems, out[1] = persistent CTAs, out[2] = shared memory bytes,
 * out[3] = FLOPs, out[4] = bytes moved, out[5..12] = problems per partition
 * of the mma.sync kernel (0-2: 1D/2D warp grids, 3-6: 3D warp grids with K
 * depth, 7: one warp per problem), out[13] = kernel (0 mma.sync, 1 tcgen05,
 * 2 staged FP64 DMMA),
 * out[14] / out[15] = problems on M = 64 / M = 128 tcgen05 MMAs. */
int kami_gemm_grouped_plan_info(const kami_grouped_plan *plan, int64_t out[16]);
int kami_gemm_grouped_plan_destroy(kami_grouped_plan *plan);

/*
 * Allocation-free grouped GEMM (no counterpart in the reference).  The same
 * computation as kami_gemm_grouped_plan_create + kami_gemm_grouped_run, for
 * callers that cannot allocate device memory: hosts whose own allocator
 * carves up device memory once at start-up and treats any later cudaMalloc
 * as a fault (serving processes, real-time and embedded controllers), and
 * plug-ins running inside such hosts.  Instead of a plan in cudaMalloc'd
 * memory it uses one fixed device array owned by the library (room for
 * KAMI_NOALLOC_MAX_PROBLEMS problem descriptors plus the CTA schedule, about
 * 0.45 MB, resident on every GPU that loads the library until the process
 * exits).  Each call rebuilds the schedule on the host, copies it into that
 * array with cudaMemcpyAsync on `stream` and launches the mma.sync grouped
 * kernel; it calls no cudaMalloc or cudaFree.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress, with that
 * device current) and sets the kernel's attributes.  Requests with more than
 * KAMI_NOALLOC_MAX_PROBLEMS problems are rejected with KAMI_ERR_UNSUPPORTED.
 * All calls share the array, which keeps the last call's contents: calls on
 * one stream are ordered and safe, calls on different streams (or host
 * threads using different streams) whose work overlaps on the GPU race.
 * Partitions come from the static cost model (autotuning would allocate).
 * Argument meaning as in kami_gemm_grouped_plan_create / _run.
 */
#define KAMI_NOALLOC_MAX_PROBLEMS 8192
int kami_gemm_grouped_noalloc(kami_dtype_t in_type, kami_dtype_t out_type, int count,
                              const int *M, const int *N, const int *K,
                              const int64_t *a_offsets, const int64_t *b_offsets,
                              const int64_t *c_offsets, const void *A, const void *B, void *C,
                              double alpha, double beta, int num_iter, void *stream);

/* ------------------------------------------------------------------------ */
/* FP64-accurate batched GEMM on the FP16/BF16/INT8 tensor cores            */
/* ------------------------------------------------------------------------ */
/*
 * C[b] = alpha * A[b] * op(B[b]) + beta * C[b] in FP64, M, N, K <= 64, computed
 * by splitting each row of A and each column of op(B) into `nslices` exact
 * integer digits (power-of-two row/column scaling; 9-bit digits in binary16,
 * 7-bit digits in bfloat16 or 8-bit digits in int8), multiplying digit pairs
 * on the tensor cores with exact accumulation (FP32 for the 16-bit digits,
 * INT32 for int8), and recombining in FP64.  FP64 arithmetic is used only for
 * the recombination.  nslices: 2..7 (KAMI_F16), 2..8 (KAMI_BF16) or 2..8
 * (KAMI_S8; 8 int8 digits carry 62 bits).  A is M x K row-major; B is N x K
 * (KAMI_B_REF_NK) or K x N (KAMI_B_ROW_KN).  No counterpart in the
 * reference; its FP64 comparator is kami_gemm_batched with in_type KAMI_F64
 * (batched_gemm_{1d,2d,3d}_double_mma.cu).  num_iter repeats the tensor-core
 * products on the resident digits (C then holds num_iter times the product).
 */
int kami_split_f64_gemm_batched(int nslices, kami_dtype_t slice_type,
                                int M, int N, int K, int64_t batch,
                                const double *A, int64_t lda, int64_t strideA,
                                const double *B, int64_t ldb, int64_t strideB,
                                kami_b_layout_t b_layout,
                                double *C, int64_t ldc, int64_t strideC,
                                double alpha, double beta, int num_iter, void *stream);

/* ------------------------------------------------------------------------ */
/* Block SpGEMM on BSR matrices (16 x 16 tiles)                             */
/* ------------------------------------------------------------------------ */
/*
 * C = A * B with A (mb x kb blocks), B (kb x nb blocks) and C in BSR form:
 * row_ptr (int32, rows + 1), col_idx (int32, sorted ascending within each
 * block-row, as the reference generator emits them), values as nnz tiles of
 * bsr x bsr elements, each tile row-major (ValA[e*256 + r*16 + c],
 * block_spgemm_2d_half_mma.cu:242-245; B tiles are used as K x N).
 * bsr must be 16 (BSR_M = BSR_K = BSR_N = 16).  The three calls follow the
 * reference's host sequence (block_spgemm_2d_half_mma.cu:805-825):
 */

/* Symbolic pass: row_ptr_c[0..mb] (device) = exclusive scan of the number
 * of distinct block columns per block-row of C.  Replaces
 * spgemm_symbolic_kernel (:58-86) + thrust::exclusive_scan (:806).  When
 * nnz_c_host is not NULL the total is copied to it and the stream is
 * synchronised (the reference's D2H copy of nnzC, :808). */
int kami_spgemm_bsr_symbolic(int bsr, int mb, int kb, int nb,
                             const int *row_ptr_a, const int *col_idx_a,
                             const int *row_ptr_b, const int *col_idx_b,
                             int *row_ptr_c, int *nnz_c_host, void *stream);

/* Column fill: col_idx_c (nnz_c entries, device) in ascending order per
 * block-row.  Replaces spgemm_symbolic_col_kernel (:88-116). */
int kami_spgemm_bsr_fill_colidx(int bsr, int mb, int kb, int nb,
                                const int *row_ptr_a, const int *col_idx_a,
                                const int *row_ptr_b, const int *col_idx_b,
                                const int *row_ptr_c, int *col_idx_c, void *stream);

/* The symbolic pass and the column fill in one call with no copy to the
 * host and no synchronisation: one cooperative kernel on `stream` whose
 * count, scan and fill phases meet at bounded grid barriers (preceded by an
 * 8-byte memset of its barrier word; devices without cooperative launch get
 * the three separate kernels), so the whole SpGEMM can run inside one stream
 * or graph.  row_ptr_c[0..mb] as in
 * kami_spgemm_bsr_symbolic, nnzC = row_ptr_c[mb] left on the device, and
 * col_idx_c filled up to `capacity` entries (the caller's upper bound for
 * nnzC, e.g. mb * nb or the sum of B row lengths over A's entries; entries
 * beyond it are not written -- compare row_ptr_c[mb] with capacity when it
 * may be exceeded).  The reference's host sequence
 * (block_spgemm_2d_half_mma.cu:805-812) synchronises here to size ColIdxC. */
int kami_spgemm_bsr_symbolic_device(int bsr, int mb, int kb, int nb,
                                    const int *row_ptr_a, const int *col_idx_a,
                                    const int *row_ptr_b, const int *col_idx_b,
                                    int *row_ptr_c, int *col_idx_c, int64_t capacity, void *stream);

/* Numeric pass: val_c (nnz_c tiles in col_idx_c order) = alpha *
 * num_iter * (A * B) + beta * val_c, FP16 or BF16 tiles with FP32
 * accumulation; out_type KAMI_F32, KAMI_F16 or KAMI_BF16.  Replaces
 * block_spgemm_{1d,2d,3d}_half_mma (e.g. :171-174, argument order kept:
 * RowPtrA, ColIdxA, ValA, RowPtrB, ColIdxB, ValB, RowPtrC, ColIdxC, ValC,
 * alpha, beta); num_iter is the reference's NUM_ITER repeat.  nnz_c may be
 * an upper bound of row_ptr_c[mb] (tiles past row_ptr_c[mb] are untouched),
 * so a capacity from kami_spgemm_bsr_symbolic_device serves.  val_a / val_b
 * may be NULL only for an operand without entries. */
int kami_spgemm_bsr_numeric(kami_dtype_t in_type, kami_dtype_t out_type, int bsr,
                            int mb, int kb, int nb,
                            const int *row_ptr_a, const int *col_idx_a, const void *val_a,
                            const int *row_ptr_b, const int *col_idx_b, const void *val_b,
                            const int *row_ptr_c, const int *col_idx_c, void *val_c,
                            int64_t nnz_c, double alpha, double beta, int num_iter,
                            void *stream);

/* The reference's block SpGEMM method: one CTA multiplies one small BSR
 * pair (mb, kb, nb <= 16 blocks of 16 x 16, at most 384 A + B tiles) with its
 * warps owning C tiles by `partition` -- 1D: warp w a range of block-rows;
 * 2D: warp (r, c) a row range x column range; 3D: warp (r, c, d) the same
 * C tiles as (r, c) over the d-th range of k, the P partial tiles reduced on
 * the device -- and repeats the products num_iter times on register-resident
 * fragments (FP32 accumulation).  Replaces block_spgemm_{1d,2d,3d}_half_mma
 * (src/sparse/spgemm/1d/block_spgemm_1d_half_mma.cu:107, 2d/...:171,
 * 3d/...:175; argument order RowPtrA, ColIdxA, ValA, RowPtrB, ColIdxB, ValB,
 * RowPtrC, ColIdxC, ValC, alpha, beta kept), launched there as 16384 CTAs
 * on one matrix pair.  `batch` problems share the structure (row_ptr /
 * col_idx of A, B and C; C's from the symbolic pass) and take tile values at
 * the given per-problem strides in elements (0 = shared, the reference's
 * launch).  nnz_a / nnz_b / nnz_c = row_ptr_x[rows] (the caller knows them,
 * as the reference's host does).  P: 1D 1, 2, 4, 8; 2D 2, 4; 3D 2 (0 =
 * 4 for 1D, 2 otherwise); partition AUTO = 1D.  Larger matrices:
 * kami_spgemm_bsr_numeric. */
int kami_spgemm_bsr_block(kami_dtype_t in_type, kami_dtype_t out_type, kami_partition_t partition, int P, int bsr,
                          int mb, int kb, int nb, int64_t batch,
                          const int *row_ptr_a, const int *col_idx_a, const void *val_a, int64_t stride_val_a,
                          int nnz_a,
                          const int *row_ptr_b, const int *col_idx_b, const void *val_b, int64_t stride_val_b,
                          int nnz_b,
                          const int *row_ptr_c, const int *col_idx_c, void *val_c, int64_t stride_val_c, int nnz_c,
                          double alpha, double beta, int num_iter, void *stream);

/* kami_spgemm_bsr_numeric with the kernel chosen: KAMI_VARIANT_MMA_SYNC
 * (one CTA per block-row: A tiles staged, each C tile's products found by
 * searching its column in the B rows, two m16n8k16 MMAs per product),
 * KAMI_VARIANT_TCGEN05 (one CTA per SM: the row's products enumerated once
 * and streamed through a shared-memory ring, one tcgen05.mma of M = 64,
 * N = 16 per product into the tile's own tensor-memory accumulator; tile
 * arrays 16-byte aligned) or KAMI_VARIANT_AUTO (the measured faster one). */
int kami_spgemm_bsr_numeric_variant(kami_variant_t variant, kami_dtype_t in_type, kami_dtype_t out_type, int bsr,
                                    int mb, int kb, int nb,
                                    const int *row_ptr_a, const int *col_idx_a, const void *val_a,
                                    const int *row_ptr_b, const int *col_idx_b, const void *val_b,
                                    const int *row_ptr_c, const int *col_idx_c, void *val_c,
                                    int64_t nnz_c, double alpha, double beta, int num_iter, void *stream);

/* ------------------------------------------------------------------------ */
/* Block SpMM: BSR (16 x 16 tiles) times dense                              */
/* ------------------------------------------------------------------------ */
/*
 * C (M x N, M = 16 mb) = alpha * num_iter * (A * op(B)) + beta * C, with A an
 * mb x kb-block BSR matrix (row_ptr mb + 1 entries, col_idx, vals as
 * row-major 16 x 16 tiles in entry order: vals[e*256 + r*16 + c]) and B
 * dense: KAMI_B_REF_NK = N x K row-major (the reference's B, read as
 * B[n*K + k] in block_spmm_1d_half_mma.cu:121-127, so C = A * B^T) or
 * KAMI_B_ROW_KN = K x N row-major (C = A * B).  FP16 or BF16 tiles and B,
 * FP32 accumulation, C in KAMI_F32, KAMI_F16 or KAMI_BF16.  batch problems
 * at the given strides (a stride of 0 shares that operand, as the
 * reference's 16384-CTA launch shares A, B and C); row_ptr entries index
 * col_idx / vals of the same problem.  Replaces block_spmm_1d_half_mma
 * (src/sparse/spmm/1d/block_spmm_1d_half_mma.cu:78, arguments bsr_rowptr,
 * bsr_colidx, bsr_vals, B, C, alpha, beta; NUM_ITER -> num_iter).
 * Block columns outside [0, kb) are skipped. */
int kami_spmm_bsr(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int N,
                  int64_t batch, const int *row_ptr, const int *col_idx,
                  int64_t stride_row_ptr, int64_t stride_col_idx,
                  const void *vals, int64_t stride_vals,
                  const void *B, int64_t ldb, int64_t strideB, kami_b_layout_t b_layout,
                  void *C, int64_t ldc, int64_t strideC,
                  double alpha, double beta, int num_iter, void *stream);

/* The same product with A in the reference's tiled-BSR form (built by
 * bsr2tilebsr, src/sparse/spmm/2d/block_spmm_2d_half_mma.cu:264-293 and
 * 3d/...:268-294): row tiles of tile_rows block-rows (the reference's
 * NUMS_ROW) and column tiles of tile_cols block-columns (NUMS_COL);
 * blk_row_ptr has (mb / tile_rows) * (kb / tile_cols) * tile_rows + 1
 * entries, entry ((i * (kb / tile_cols) + j) * tile_rows + ii) starting
 * block-row i * tile_rows + ii of column tile j; blk_col_idx is relative to
 * the column tile; vals are tiles in blk entry order.  Replaces
 * block_spmm_2d_half_mma (2d/...:72) and block_spmm_3d_half_mma
 * (3d/...:73), whose argument order (blk_rowptr, blk_colidx, bsr_vals, B,
 * C, alpha, beta) is kept; the 3D form's P partial C slices are reduced
 * here (C is M x N). */
int kami_spmm_tilebsr(kami_dtype_t in_type, kami_dtype_t out_type, int bsr, int mb, int kb, int N,
                      int64_t batch, int tile_rows, int tile_cols,
                      const int *blk_row_ptr, const int *blk_col_idx,
                      int64_t stride_row_ptr, int64_t stride_col_idx,
                      const void *vals, int64_t stride_vals,
                      const void *B, int64_t ldb, int64_t strideB, kami_b_layout_t b_layout,
                      void *C, int64_t ldc, int64_t strideC,
                      double alpha, double beta, int num_iter, void *stream);

/* Host conversion BSR -> tiled-BSR, the reference's bsr2tilebsr
 * (2d/...:264-293) on host arrays: fills blk_row_ptr / blk_col_idx exactly
 * as the reference does and, when perm is not NULL, perm[e] = the BSR entry
 * that tiled entry e came from (the reference leaves the values in BSR
 * order; gather vals through perm to multiply the same matrix).  Returns
 * the number of entries (or a negative status). */
int kami_bsr_to_tilebsr(int mb, int kb, int tile_rows, int tile_cols,
                        const int *row_ptr, const int *col_idx,
                        int *blk_row_ptr, int *blk_col_idx, int *perm);

#ifdef __cplusplus
}
#endif

#endif /* KAMI_B200_H */
