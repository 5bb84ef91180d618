/*
 * kami_oracle.c -- CPU oracle for the KAMI block-GEMM / block-SpGEMM path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it restates, in plain
 * C with OpenMP, the host-side check code that every KAMI benchmark carries
 * in its main().  Only the test suite, the smoke check and the CPU-baseline
 * leg of the benchmark may load it.  The product library (libkami_b200.so)
 * never links, loads or calls anything in this directory.
 *
 * Pinning: the SpGEMM generator and SPA functions below are checked bit for
 * bit against the reference's own functions (compiled from its sources into
 * oracle/_ref by oracle/Makefile.ref); the dense GEMM restatement is checked
 * against golden vectors that the reference's own kernels produced on a B200
 * (tests/golden/).
 *
 * Reference files cited (paths inside the KAMI project):
 *   src/batched_gemm/KAMI/2d/batched_gemm_2d_double_mma.cu
 *   src/batched_gemm/KAMI/3d/batched_gemm_3d_double_mma.cu
 *   src/block_gemm/KAMI/1d/fp16/block_gemm_1d_half_mma.cu
 *   src/block_gemm/KAMI/3d/fp16/block_gemm_3d_half_mma.cu
 *   src/sparse/spgemm/2d/block_spgemm_2d_half_mma.cu
 *   src/sparse/spmm/{1d,2d,3d}/block_spmm_{1d,2d,3d}_half_mma.cu
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define KAMI_ORACLE_B_REF_NK 0 /* B stored N x K row-major (the reference layout) */
#define KAMI_ORACLE_B_ROW_KN 1 /* B stored K x N row-major */

/* ------------------------------------------------------------------------ */
/* scalar conversions                                                       */
/* ------------------------------------------------------------------------ */

static inline double h2d(uint16_t bits)
{
    _Float16 h;
    memcpy(&h, &bits, 2);
    return (double)h;
}

static inline uint16_t d2h(double x)
{
    /* IEEE round-to-nearest-even double -> binary16 */
    _Float16 h = (_Float16)x;
    uint16_t bits;
    memcpy(&bits, &h, 2);
    return bits;
}

static inline double bf2d(uint16_t bits)
{
    uint32_t u = ((uint32_t)bits) << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

double kami_oracle_half_to_double(uint16_t bits) { return h2d(bits); }
uint16_t kami_oracle_double_to_half(double x) { return d2h(x); }

/* ------------------------------------------------------------------------ */
/* input generators                                                         */
/* ------------------------------------------------------------------------ */

/* x[i] = rand_r(&seed_i) % mod with seed_i = i, exactly the fill of
 * batched_gemm_2d_double_mma.cu:271-285 (A and B both use it). */
void kami_oracle_fill_rand_r_mod(double *x, int64_t n, int mod)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++)
    {
        unsigned int seed = (unsigned int)i;
        x[i] = (double)(rand_r(&seed) % mod);
    }
}

/* Block-BSR generator shared by the reference's sparse programs: srand(0),
 * then one rand() per block position (kept when rand()/RAND_MAX > sparsity)
 * and BSR_M*BSR_K values rand() % mod + add per kept block, row by row:
 *   block_spgemm_2d_half_mma.cu:648-673   rand() % 3 + 1
 *   spmm/1d/block_spmm_1d_half_mma.cu:197-222   rand() % 3
 *   spmm/2d/...:236-262, spmm/3d/...:241-266   rand() % 2 + 1
 * Values are written as binary16 bits.  Returns the number of nonzero
 * blocks. */
int kami_oracle_bsr_generate_rule(int rows, int cols, float sparsity, int bsr_m, int bsr_k, int mod, int add,
                                  int *row_ptr, int *col_idx, uint16_t *values)
{
    int count = 0;
    srand(0);
    row_ptr[0] = 0;
    for (int i = 0; i < rows; i++)
    {
        for (int j = 0; j < cols; j++)
        {
            float r = (float)rand() / (float)RAND_MAX;
            if (r > sparsity)
            {
                col_idx[count] = j;
                for (int len = 0; len < bsr_m * bsr_k; len++)
                    values[(int64_t)count * bsr_m * bsr_k + len] = d2h((double)(rand() % mod) + (double)add);
                count++;
            }
        }
        row_ptr[i + 1] = count;
    }
    return count;
}

int kami_oracle_bsr_generate(int rows, int cols, float sparsity, int bsr_m,
                             int bsr_k, int *row_ptr, int *col_idx,
                             uint16_t *values)
{
    return kami_oracle_bsr_generate_rule(rows, cols, sparsity, bsr_m, bsr_k, 3, 1, row_ptr, col_idx, values);
}

/* ------------------------------------------------------------------------ */
/* dense GEMM checks                                                        */
/* ------------------------------------------------------------------------ */

static inline int64_t b_index(int b_layout, int N, int K, int64_t ldb, int n, int k)
{
    /* REF_NK: h_B[j * K_BLOCK + k]   (batched_gemm_2d_double_mma.cu:348)
     * ROW_KN: B[k * N + j]                                              */
    (void)N;
    (void)K;
    return b_layout == KAMI_ORACLE_B_REF_NK ? (int64_t)n * ldb + k : (int64_t)k * ldb + n;
}

/* C[b] = A[b] * op(B[b]) with a double accumulator in i, j, k order:
 * batched_gemm_2d_double_mma.cu:338-352 (OpenMP over the batch) and
 * block_gemm_1d_half_mma.cu:269-279 (single block).  lda/ldb/ldc are row
 * strides in elements; sA/sB/sC are per-problem strides. */
void kami_oracle_gemm_f64(int64_t batch, int M, int N, int K,
                          const double *A, int64_t lda, int64_t sA,
                          const double *B, int64_t ldb, int64_t sB, int b_layout,
                          double *C, int64_t ldc, int64_t sC)
{
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < batch; b++)
    {
        const double *a = A + b * sA;
        const double *bb = B + b * sB;
        double *c = C + b * sC;
        for (int i = 0; i < M; i++)
            for (int j = 0; j < N; j++)
            {
                double acc = 0;
                for (int k = 0; k < K; k++)
                    acc += a[(int64_t)i * lda + k] * bb[b_index(b_layout, N, K, ldb, j, k)];
                c[(int64_t)i * ldc + j] = acc;
            }
    }
}

/* Same loop for 16-bit inputs (binary16 when is_bf16 == 0, bfloat16
 * otherwise) widened to double, as the FP16 host check does
 * ((double)h_A[..] * (double)h_B[..], block_gemm_1d_half_mma.cu:276). */
void kami_oracle_gemm_h16(int64_t batch, int M, int N, int K,
                          const uint16_t *A, int64_t lda, int64_t sA,
                          const uint16_t *B, int64_t ldb, int64_t sB, int b_layout,
                          int is_bf16, double *C, int64_t ldc, int64_t sC)
{
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < batch; b++)
    {
        const uint16_t *a = A + b * sA;
        const uint16_t *bb = B + b * sB;
        double *c = C + b * sC;
        for (int i = 0; i < M; i++)
            for (int j = 0; j < N; j++)
            {
                double acc = 0;
                for (int k = 0; k < K; k++)
                {
                    uint16_t x = a[(int64_t)i * lda + k];
                    uint16_t y = bb[b_index(b_layout, N, K, ldb, j, k)];
                    acc += is_bf16 ? bf2d(x) * bf2d(y) : h2d(x) * h2d(y);
                }
                c[(int64_t)i * ldc + j] = acc;
            }
    }
}

/* Sum of the P partial C slices that a 3D-partitioned kernel writes into a
 * P-times larger C: slice 0 += slices 1..P-1, per problem
 * (batched_gemm_3d_double_mma.cu:361-373; block_gemm_3d_half_mma.cu:291-300).
 * Cp holds batch * P slices of M*N; out receives batch reduced slices. */
void kami_oracle_reduce_slices_f64(int64_t batch, int P, int M, int N,
                                   const double *Cp, double *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < batch; b++)
        for (int64_t e = 0; e < (int64_t)M * N; e++)
        {
            double acc = Cp[b * (int64_t)M * N * P + e];
            for (int s = 1; s < P; s++)
                acc += Cp[b * (int64_t)M * N * P + (int64_t)s * M * N + e];
            out[b * (int64_t)M * N + e] = acc;
        }
}

/* ------------------------------------------------------------------------ */
/* double-double GEMM (error reference for split-FP64)                      */
/* ------------------------------------------------------------------------ */

/* Error-free transformations: TwoSum (Knuth) and TwoProd via FMA, summed
 * with the compensated dot product Dot2 of Ogita, Rump and Oishi (2005).
 * Result: C = Chi + Clo with |error| ~ u^2 * sum |a||b|. */
static inline void two_sum(double a, double b, double *s, double *e)
{
    double x = a + b;
    double z = x - a;
    *e = (a - (x - z)) + (b - z);
    *s = x;
}

void kami_oracle_gemm_dd(int64_t batch, int M, int N, int K,
                         const double *A, int64_t lda, int64_t sA,
                         const double *B, int64_t ldb, int64_t sB, int b_layout,
                         double *Chi, double *Clo, int64_t ldc, int64_t sC)
{
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < batch; b++)
    {
        const double *a = A + b * sA;
        const double *bb = B + b * sB;
        for (int i = 0; i < M; i++)
            for (int j = 0; j < N; j++)
            {
                double s = 0, c = 0;
                for (int k = 0; k < K; k++)
                {
                    double x = a[(int64_t)i * lda + k];
                    double y = bb[b_index(b_layout, N, K, ldb, j, k)];
                    double p = x * y;
                    double pe = fma(x, y, -p);
                    double t, te;
                    two_sum(s, p, &t, &te);
                    s = t;
                    c += te + pe;
                }
                double hi, lo;
                two_sum(s, c, &hi, &lo);
                Chi[b * sC + (int64_t)i * ldc + j] = hi;
                Clo[b * sC + (int64_t)i * ldc + j] = lo;
            }
    }
}

/* Normwise relative error ||C - (Chi + Clo)||_F / ||Chi + Clo||_F, each
 * difference formed as (C - Chi) - Clo so the double-double tail counts. */
double kami_oracle_normwise_error_dd(int64_t n, const double *C,
                                     const double *Chi, const double *Clo)
{
    double num = 0, den = 0;
#pragma omp parallel for reduction(+ : num, den) schedule(static)
    for (int64_t i = 0; i < n; i++)
    {
        double d = (C[i] - Chi[i]) - Clo[i];
        num += d * d;
        den += Chi[i] * Chi[i];
    }
    return den > 0 ? sqrt(num / den) : sqrt(num);
}

/* ------------------------------------------------------------------------ */
/* block SpGEMM (BSR, dense bsr_m x bsr_k tiles)                           */
/* ------------------------------------------------------------------------ */

/* Symbolic pass of spgemm_spa (block_spgemm_2d_half_mma.cu:560-589): per
 * block-row a dense flag array over the nB block columns of B, then a count,
 * then an exclusive scan into RowPtrC[0..mA].  Returns nnzC in blocks. */
int kami_oracle_spgemm_symbolic(int mA, int nB, const int *RowPtrA,
                                const int *ColIdxA, const int *RowPtrB,
                                const int *ColIdxB, int *RowPtrC)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int iid = 0; iid < mA; iid++)
    {
        char *flag = (char *)calloc((size_t)nB, 1);
        for (int i = RowPtrA[iid]; i < RowPtrA[iid + 1]; i++)
        {
            int col = ColIdxA[i];
            for (int l = RowPtrB[col]; l < RowPtrB[col + 1]; l++)
                flag[ColIdxB[l]] = 1;
        }
        int nnzr = 0;
        for (int cid = 0; cid < nB; cid++)
            nnzr += flag[cid] == 1;
        RowPtrC[iid] = nnzr;
        free(flag);
    }
    /* exclusive scan over mA + 1 entries (the reference's exclusive_scan<int>) */
    int run = 0;
    for (int i = 0; i < mA; i++)
    {
        int v = RowPtrC[i];
        RowPtrC[i] = run;
        run += v;
    }
    RowPtrC[mA] = run;
    return run;
}

/* Numeric pass of spgemm_spa (block_spgemm_2d_half_mma.cu:590-645): per
 * block-row, accumulate every A-tile x B-tile product into a dense row of
 * tiles, then emit the flagged tiles in ascending column order.
 *   A tiles: bsr x bsr row-major (ValA[e*bsr*bsr + r*bsr + c]);
 *   B tiles: bsr x bsr row-major, used as K x N (ValB[.. + kk*bsr + jj]).
 * accum_mode 0 reproduces the reference exactly: the dense row is binary16
 * and each product (exact in double) is rounded to binary16, then added in
 * binary16 arithmetic (its "half += double" statement).
 * accum_mode 1 accumulates in double and writes double results (the FP32-
 * accumulating kernels are checked against this one).
 * ValC16 (mode 0) or ValC64 (mode 1) receives nnzC tiles. */
void kami_oracle_spgemm_numeric(int mA, int nB, int bsr, const int *RowPtrA,
                                const int *ColIdxA, const uint16_t *ValA,
                                const int *RowPtrB, const int *ColIdxB,
                                const uint16_t *ValB, const int *RowPtrC,
                                int *ColIdxC, int accum_mode, uint16_t *ValC16,
                                double *ValC64)
{
    const int tile = bsr * bsr;
#pragma omp parallel for schedule(dynamic, 4)
    for (int iid = 0; iid < mA; iid++)
    {
        /* touched columns of this row, kept as a flag array like the
         * reference; the dense value row is allocated for the touched span */
        char *flag = (char *)calloc((size_t)nB, 1);
        int lo = nB, hi = -1;
        for (int i = RowPtrA[iid]; i < RowPtrA[iid + 1]; i++)
        {
            int col = ColIdxA[i];
            for (int l = RowPtrB[col]; l < RowPtrB[col + 1]; l++)
            {
                int key = ColIdxB[l];
                flag[key] = 1;
                if (key < lo)
                    lo = key;
                if (key > hi)
                    hi = key;
            }
        }
        if (hi >= lo)
        {
            int64_t span = (int64_t)(hi - lo + 1) * tile;
            _Float16 *row16 = NULL;
            double *row64 = NULL;
            if (accum_mode == 0)
                row16 = (_Float16 *)calloc((size_t)span, sizeof(_Float16));
            else
                row64 = (double *)calloc((size_t)span, sizeof(double));
            for (int i = RowPtrA[iid]; i < RowPtrA[iid + 1]; i++)
            {
                int col = ColIdxA[i];
                const uint16_t *a = ValA + (int64_t)i * tile;
                for (int l = RowPtrB[col]; l < RowPtrB[col + 1]; l++)
                {
                    int key = ColIdxB[l];
                    const uint16_t *b = ValB + (int64_t)l * tile;
                    int64_t base = (int64_t)(key - lo) * tile;
                    for (int ii = 0; ii < bsr; ii++)
                        for (int jj = 0; jj < bsr; jj++)
                            for (int kk = 0; kk < bsr; kk++)
                            {
                                double p = h2d(a[ii * bsr + kk]) * h2d(b[kk * bsr + jj]);
                                if (accum_mode == 0)
                                {
                                    _Float16 ph = (_Float16)p;
                                    row16[base + ii * bsr + jj] =
                                        (_Float16)((float)row16[base + ii * bsr + jj] + (float)ph);
                                }
                                else
                                    row64[base + ii * bsr + jj] += p;
                            }
                }
            }
            int nnzr = RowPtrC[iid];
            for (int cid = lo; cid <= hi; cid++)
            {
                if (flag[cid] != 1)
                    continue;
                int64_t src = (int64_t)(cid - lo) * tile;
                for (int t = 0; t < tile; t++)
                {
                    if (accum_mode == 0)
                    {
                        uint16_t bits;
                        memcpy(&bits, &row16[src + t], 2);
                        ValC16[(int64_t)nnzr * tile + t] = bits;
                    }
                    else
                        ValC64[(int64_t)nnzr * tile + t] = row64[src + t];
                }
                ColIdxC[nnzr] = cid;
                nnzr++;
            }
            free(row16);
            free(row64);
        }
        free(flag);
    }
}

/* nnzCub: sum over nonzero A blocks (i,k) of the length of B's block-row k
 * (block_spgemm_2d_half_mma.cu:763-768).  The SpGEMM FLOP count is
 * 2 * nnzCub * bsr^3. */
int64_t kami_oracle_spgemm_nnzcub(int nnzA_blocks, const int *ColIdxA,
                                  const int *RowPtrB)
{
    int64_t s = 0;
    for (int i = 0; i < nnzA_blocks; i++)
    {
        int r = ColIdxA[i];
        s += RowPtrB[r + 1] - RowPtrB[r];
    }
    return s;
}

/* A random block pattern with independent Bernoulli(density) positions from
 * a 64-bit LCG seeded by `seed` (the large SpGEMM workload; the reference's
 * own generator above always reseeds with srand(0)).  Values are left to the
 * caller.  Returns the number of blocks, or -1 when capacity is exceeded. */
int kami_oracle_bsr_pattern(int rows, int cols, double density, uint64_t seed,
                            int *row_ptr, int *col_idx, int capacity)
{
    uint64_t s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    int count = 0;
    row_ptr[0] = 0;
    for (int i = 0; i < rows; i++)
    {
        for (int j = 0; j < cols; j++)
        {
            s = s * 6364136223846793005ULL + 1442695040888963407ULL;
            double u = (double)(s >> 11) * (1.0 / 9007199254740992.0);
            if (u < density)
            {
                if (count >= capacity)
                    return -1;
                col_idx[count++] = j;
            }
        }
        row_ptr[i + 1] = count;
    }
    return count;
}

/* ------------------------------------------------------------------------ */
/* block SpMM (BSR or tiled-BSR A, dense B)                                 */
/* ------------------------------------------------------------------------ */

/* bsr2tilebsr of spmm/2d/block_spmm_2d_half_mma.cu:264-293 (the same code
 * in spmm/3d/...:268-294): for each row tile i (row_tiles of them, tile_rows
 * block-rows each), each column tile j (tile_cols block-columns), each
 * block-row ii of the tile: the entries of BSR row i*tile_rows + ii whose
 * column falls in tile j, column kept relative to the tile.  Returns the
 * number of entries. */
int kami_oracle_bsr2tilebsr(int row_tiles, int tile_rows, int cols, int tile_cols, const int *bsr_rowptr,
                            const int *bsr_colidx, int *blk_rowptr, int *blk_colidx)
{
    int count = 0;
    blk_rowptr[0] = 0;
    for (int i = 0; i < row_tiles; i++)
        for (int j = 0; j < cols / tile_cols; j++)
        {
            int start = j * tile_cols, end = (j + 1) * tile_cols;
            for (int ii = 0; ii < tile_rows; ii++)
            {
                for (int jj = bsr_rowptr[i * tile_rows + ii]; jj < bsr_rowptr[i * tile_rows + ii + 1]; jj++)
                {
                    int col = bsr_colidx[jj];
                    if (col >= start && col < end)
                        blk_colidx[count++] = col % tile_cols;
                }
                blk_rowptr[i * tile_rows * (cols / tile_cols) + j * tile_rows + ii + 1] = count;
            }
        }
    return count;
}

/* Host check of the block SpMM programs, in their loop order and with a
 * double accumulator: for each row tile i, column tile j, block-row ii of
 * the tile and entry jj, C[(row) * ldc + n] += a[r*16 + c] * B(n, k)
 * (spmm/1d/...:305-326 for plain BSR, which is tile_rows = 1 and one column
 * tile; spmm/2d/...:385-408 and 3d/...:398-419 for the tiled form).  vals
 * are the tiles as doubles; B(n, k) = B[n*ldb + k] (b_layout 0, the
 * reference's N x K) or B[k*ldb + n] (b_layout 1, K x N).  C is zeroed
 * first (mb*16 x N, row stride ldc). */
void kami_oracle_spmm(int mb, int kb, int N, int tile_rows, int tile_cols, const int *rowptr, const int *colidx,
                      const double *vals, const double *B, int64_t ldb, int b_layout, double *C, int64_t ldc)
{
    const int ntiles = tile_cols > 0 ? kb / tile_cols : 1;
    const int tc = tile_cols > 0 ? tile_cols : 0;
    for (int r = 0; r < mb * 16; r++)
        for (int n = 0; n < N; n++)
            C[(int64_t)r * ldc + n] = 0.0;
    for (int i = 0; i < mb / tile_rows; i++)
        for (int j = 0; j < ntiles; j++)
            for (int ii = 0; ii < tile_rows; ii++)
            {
                int q = i * tile_rows * ntiles + j * tile_rows + ii;
                for (int jj = rowptr[q]; jj < rowptr[q + 1]; jj++)
                {
                    int col = colidx[jj] + j * tc;
                    const double *a = vals + (int64_t)jj * 256;
                    for (int iii = 0; iii < 16; iii++)
                        for (int jjj = 0; jjj < 16; jjj++)
                        {
                            int k = col * 16 + jjj;
                            double av = a[iii * 16 + jjj];
                            double *crow = C + (int64_t)((i * tile_rows + ii) * 16 + iii) * ldc;
                            for (int n = 0; n < N; n++)
                                crow[n] += av * (b_layout == 0 ? B[(int64_t)n * ldb + k] : B[(int64_t)k * ldb + n]);
                        }
                }
            }
}
