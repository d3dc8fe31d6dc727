/*
 * ORACLE (test infrastructure only).  CPU restatement of the reference's hot path:
 * block-cyclic / 2D-block / Cannon pack and unpack, the 2.5D Cannon step schedule,
 * and an extended-precision (double-double) GEMM checker.  Only tests/, the smoke
 * check and bench.py's CPU legs use it, as the checker; the product never links it.
 * Each function cites the reference lines (paths relative to the reference root)
 * it restates.  All matrices are column-major unless stated otherwise.
 */
#ifndef ORC_H
#define ORC_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/Decompositions/pblasDecomposition.cpp:3-23 */
int orc_numroc(int n, int nb, int iproc, int isrproc, int nprocs);

/* pblasDecomposer ctor, pblasDecomposition.cpp:25-71: local rows/cols and owned blocks
 * of rank `rank` on a row-major dRow x dCol grid. */
void orc_pblas_local_shape(int M, int N, int Mb, int Nb, int dRow, int dCol, int rank, int* rows, int* cols,
                           int* blocks);

/* scatterMatrix (pblasDecomposition.cpp:73-148) seen from all ranks at once:
 * global (ld = ldg) -> locals[rank] (ld = lld[rank]).  Returns 0, or -1 when a rank
 * owns no rows/columns (the reference divides by zero there). */
int orc_pblas_scatter(int M, int N, int Mb, int Nb, int dRow, int dCol, const double* global, int64_t ldg,
                      double* const* locals, const int64_t* lld);

/* gatherMatrix (pblasDecomposition.cpp:150-221): locals -> global. */
int orc_pblas_gather(int M, int N, int Mb, int Nb, int dRow, int dCol, double* global, int64_t ldg,
                     const double* const* locals, const int64_t* lld);

/* calculateVirtualDeviceGrid (2DBlockSequentialDecomposition.cpp:27-54). */
void orc_block2d_grid(int P, int* dRow, int* dCol);

/* deliverMatrix (2DBlockSequentialDecomposition.cpp:56-162): tiles of A (row panel,
 * full K), B (column panel), C per rank; remainder rows/cols go to the last grid
 * row/column.  colMajor selects the reference's column- or row-major convention. */
void orc_block2d_deliver(int64_t M, int64_t N, int64_t K, int dRow, int dCol, int colMajor, const double* gA,
                         const double* gB, const double* gC, double* const* lA, double* const* lB, double* const* lC);

/* gatherResult (2DBlockSequentialDecomposition.cpp:164-253): C tiles -> global C. */
void orc_block2d_gather(int64_t M, int64_t N, int dRow, int dCol, int colMajor, double* C, const double* const* lC);

/* decompose2D (src/25DCannon.cpp:87-149): equal p x p blocks of square A, B, C to the
 * stack-0 ranks i*p+j (tile ld = M/p). */
void orc_cannon_decompose(int64_t M, int p, const double* A, const double* B, const double* C, double* const* lA,
                          double* const* lB, double* const* lC);

/* reorderMatrix (src/25DCannon.cpp:231-284): stack-0 C tiles -> global C. */
void orc_cannon_reorder(int64_t M, int p, double* C, const double* const* lC);

/* The k-block indices virtual rank (i,j,k) multiplies, in step order, under the
 * reference's skew (25DCannon.cpp:303-310) and rotation targets (:333-334, :364-365):
 * t_0 = (i + j - k*pc3) mod p, t_r = t_{r-1} - r mod p.  out has pc3 = p/c entries.
 * Returns 1 if every stack's steps together cover all p k-blocks exactly once. */
int orc_cannon_schedule(int p, int c, int i, int j, int k, int* out);

/* copyBlock (src/Transfers/sharedTransfers.cpp:29-63): rows x cols strided copy; when
 * colMajor is 0 the dims are swapped first, as the reference does. */
void orc_copy_block(int64_t rows, int64_t cols, const double* src, double* dst, int64_t ldS, int64_t ldD,
                    int colMajor);

/* Extended-precision checker: C_ref(i,j) = alpha*sum_k op(A)(i,k)*op(B)(k,j) + beta*C0(i,j)
 * evaluated in double-double (TwoSum / TwoProduct via fma, Ogita-Rump-Oishi 2005) at
 * n sampled (row, col) positions, rounded once to double. */
void orc_dgemm_dd_sample(char ta, char tb, int64_t K, double alpha, const double* A, int64_t lda, const double* B,
                         int64_t ldb, double beta, const double* C0, int64_t ldc, int64_t n, const int64_t* rows,
                         const int64_t* cols, double* out);

/* Sampled rows of alpha*op(A)*B in double-double over every column of B (the exact-product
 * yardstick of the FP64 emulation's error): At holds the rows K-contiguously (row s at
 * At + s*ldat), out[s + j*ldo]; work split over nthreads threads (<= 0: all online cores). */
void orc_dd_rows(int64_t K, int64_t nrows, const double* At, int64_t ldat, int64_t ncols, const double* B,
                 int64_t ldb, double alpha, double* out, int64_t ldo, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
