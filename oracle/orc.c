/*
 * ORACLE (test infrastructure only) -- see orc.h.  Plain C restatement of the
 * reference's hot-path index arithmetic and data movement, written to follow the
 * cited loops so that tests can check the CUDA product against it bit for bit, and
 * the restatement itself against the reference's own code (oracle/_ref).
 */
#define _DEFAULT_SOURCE /* sysconf(_SC_NPROCESSORS_ONLN) under -std=c11 */
#include "orc.h"

#include <pthread.h>
#include <unistd.h>

#include <math.h>
#include <string.h>

/* numroc, src/Decompositions/pblasDecomposition.cpp:3-23 */
int orc_numroc(int n, int nb, int iproc, int isrproc, int nprocs) {
    int myDistance = (nprocs + iproc - isrproc) % nprocs;
    int numBlocks = n / nb;
    int r = (numBlocks / nprocs) * nb;
    int extraBlocks = numBlocks % nprocs;
    if (myDistance < extraBlocks)
        r += nb;
    else if (myDistance == extraBlocks)
        r += n % nb;
    return r;
}

/* pblasDecomposer ctor, pblasDecomposition.cpp:35-65 (row-major grid, root (0,0)) */
void orc_pblas_local_shape(int M, int N, int Mb, int Nb, int dRow, int dCol, int rank, int* rows, int* cols,
                           int* blocks) {
    int procRow = rank / dCol, procCol = rank % dCol;
    int gridRows = M / Mb + (M % Mb ? 1 : 0);
    int gridCols = N / Nb + (N % Nb ? 1 : 0);
    *rows = orc_numroc(M, Mb, procRow, 0, dRow);
    *cols = orc_numroc(N, Nb, procCol, 0, dCol);
    int b = 0;
    for (int i = 0; i < gridRows; ++i)
        if (i % dRow == procRow)
            for (int j = 0; j < gridCols; ++j)
                if (j % dCol == procCol) ++b;
    *blocks = b;
}

static void copy_cols(int64_t rows, int64_t cols, const double* src, int64_t ldS, double* dst, int64_t ldD) {
    for (int64_t c = 0; c < cols; ++c) memcpy(dst + c * ldD, src + c * ldS, (size_t)rows * sizeof(double));
}

static int pblas_grid_ok(int M, int N, int Mb, int Nb, int dRow, int dCol) {
    if (M <= 0 || N <= 0 || Mb <= 0 || Nb <= 0 || dRow <= 0 || dCol <= 0) return 0;
    for (int r = 0; r < dRow; ++r)
        if (orc_numroc(M, Mb, r, 0, dRow) <= 0) return 0;
    for (int c = 0; c < dCol; ++c)
        if (orc_numroc(N, Nb, c, 0, dCol) <= 0) return 0;
    return 1;
}

/*
 * One pass of the reference's block walk (pblasDecomposition.cpp:95-131 for scatter,
 * :172-206 for gather) for a single rank: every block (row, col) it owns is moved
 * between global[col*ldg + row] and local[columnOffset*lld + rowOffset], with the
 * offsets advanced exactly as the reference advances them (modulo the local extent).
 */
static void pblas_walk(int M, int N, int Mb, int Nb, int dRow, int dCol, int rank, double* global, int64_t ldg,
                       double* local, int64_t lld, int to_local) {
    int procRow = rank / dCol;
    int localRows = orc_numroc(M, Mb, procRow, 0, dRow);
    int localCols = orc_numroc(N, Nb, rank % dCol, 0, dCol);
    int rowOffset = 0, columnOffset = 0;
    int pr = 0;
    for (int row = 0; row < M; row += Mb, pr = (pr + 1) % dRow) {
        int pc = 0;
        int rowsToSend = (M - row < Mb) ? M - row : Mb;
        for (int col = 0; col < N; col += Nb, pc = (pc + 1) % dCol) {
            int receiver = pr * dCol + pc;
            int colsToSend = (N - col < Nb) ? N - col : Nb;
            if (receiver == rank) {
                double* g = global + (int64_t)col * ldg + row;
                double* l = local + (int64_t)columnOffset * lld + rowOffset;
                if (to_local)
                    copy_cols(rowsToSend, colsToSend, g, ldg, l, lld);
                else
                    copy_cols(rowsToSend, colsToSend, l, lld, g, ldg);
                columnOffset = (columnOffset + colsToSend) % localCols;
            }
        }
        if (procRow == pr) rowOffset = (rowOffset + rowsToSend) % localRows;
    }
}

int orc_pblas_scatter(int M, int N, int Mb, int Nb, int dRow, int dCol, const double* global, int64_t ldg,
                      double* const* locals, const int64_t* lld) {
    if (!pblas_grid_ok(M, N, Mb, Nb, dRow, dCol)) return -1;
    for (int r = 0; r < dRow * dCol; ++r)
        pblas_walk(M, N, Mb, Nb, dRow, dCol, r, (double*)global, ldg, locals[r], lld[r], 1);
    return 0;
}

int orc_pblas_gather(int M, int N, int Mb, int Nb, int dRow, int dCol, double* global, int64_t ldg,
                     const double* const* locals, const int64_t* lld) {
    if (!pblas_grid_ok(M, N, Mb, Nb, dRow, dCol)) return -1;
    for (int r = 0; r < dRow * dCol; ++r)
        pblas_walk(M, N, Mb, Nb, dRow, dCol, r, global, ldg, (double*)locals[r], lld[r], 0);
    return 0;
}

/* calculateVirtualDeviceGrid, 2DBlockSequentialDecomposition.cpp:27-54 */
void orc_block2d_grid(int P, int* dRow, int* dCol) {
    int Px = (int)sqrt((double)P);
    int Py = Px;
    if (Px == 0) {
        Py = P;
        Px = 1;
    }
    int counter;
    for (counter = Px; counter > 0; --counter)
        if (P % counter == 0) break;
    if (counter == 0) {
        Px = P;
        Py = 1;
    } else {
        Px = counter;
        Py = P / counter;
    }
    *dRow = Py;
    *dCol = Px;
}

/* copyBlock, src/Transfers/sharedTransfers.cpp:29-63, including its shortcut at :51:
 * when rows == ldS and cols == ldD (after the swap) the block is copied as ONE
 * contiguous run of rows*cols elements, whatever ldD is. */
void orc_copy_block(int64_t rows, int64_t cols, const double* src, double* dst, int64_t ldS, int64_t ldD,
                    int colMajor) {
    if (!src || !dst) return;
    if (rows * cols <= 0) return;
    if (!colMajor) {
        int64_t t = rows;
        rows = cols;
        cols = t;
    }
    if (rows == ldS && cols == ldD)
        memcpy(dst, src, (size_t)(rows * cols) * sizeof(double));
    else
        copy_cols(rows, cols, src, ldS, dst, ldD);
}

/* MPI_Type_vector transfer pair (src/Transfers/mpiTransfers.cpp:16-57): a strided
 * block send matched with a strided receive is a plain strided copy. */
static void vector_transfer(int64_t rows, int64_t cols, const double* src, int64_t ldS, double* dst, int64_t ldD,
                            int colMajor) {
    if (!colMajor) {
        int64_t t = rows;
        rows = cols;
        cols = t;
    }
    copy_cols(rows, cols, src, ldS, dst, ldD);
}

/* deliverMatrix, 2DBlockSequentialDecomposition.cpp:76-144 */
void orc_block2d_deliver(int64_t M, int64_t N, int64_t K, int dRow, int dCol, int colMajor, const double* gA,
                         const double* gB, const double* gC, double* const* lA, double* const* lB, double* const* lC) {
    int64_t tileK = K;
    for (int i = 0; i < dRow; ++i) {
        int64_t tileM = M / dRow + ((i + 1 == dRow) ? M % dRow : 0);
        for (int j = 0; j < dCol; ++j) {
            int r = i * dCol + j;
            int64_t tileN = N / dCol + ((j + 1 == dCol) ? N % dCol : 0);
            int64_t aOff = (M / dRow) * K * i, bOff = (N / dCol) * j, cOff = (M / dRow) * N * i + (N / dCol) * j;
            int64_t lda = K, ldb = N, ldc = N, llda = tileK, lldb = tileN, lldc = tileN;
            if (colMajor) {
                aOff = (M / dRow) * i;
                bOff = (N / dCol) * K * j;
                cOff = (N / dCol) * M * j + (M / dRow) * i;
                lda = M;
                ldb = K;
                ldc = M;
                llda = tileM;
                lldb = tileK;
                lldc = tileM;
            }
            if (r == 0) { /* sender copies its own tiles with copyBlock (:129-135) */
                orc_copy_block(tileM, tileK, gA, lA[r], lda, llda, colMajor);
                orc_copy_block(tileK, tileN, gB, lB[r], ldb, lldb, colMajor);
                orc_copy_block(tileM, tileN, gC, lC[r], ldc, lldc, colMajor);
            } else { /* MPI vector send/recv (:122-126, :136-141) */
                vector_transfer(tileM, tileK, gA + aOff, lda, lA[r], llda, colMajor);
                vector_transfer(tileK, tileN, gB + bOff, ldb, lB[r], lldb, colMajor);
                vector_transfer(tileM, tileN, gC + cOff, ldc, lC[r], lldc, colMajor);
            }
        }
    }
}

/* gatherResult with gatherRank 0, 2DBlockSequentialDecomposition.cpp:185-236 */
void orc_block2d_gather(int64_t M, int64_t N, int dRow, int dCol, int colMajor, double* C, const double* const* lC) {
    for (int i = 0; i < dRow; ++i) {
        int64_t tileM = M / dRow + ((i + 1 == dRow) ? M % dRow : 0);
        for (int j = 0; j < dCol; ++j) {
            int r = i * dCol + j;
            int64_t tileN = N / dCol + ((j + 1 == dCol) ? N % dCol : 0);
            int64_t cOff = (M / dRow) * N * i + (N / dCol) * j;
            int64_t ldc = N, lldc = tileN;
            if (colMajor) {
                cOff = (N / dCol) * M * j + (M / dRow) * i;
                ldc = M;
                lldc = tileM;
            }
            if (r == 0) /* the gather rank's own tile goes through copyBlock (:226-228) */
                orc_copy_block(tileM, tileN, lC[r], C + cOff, lldc, ldc, colMajor);
            else
                vector_transfer(tileM, tileN, lC[r], lldc, C + cOff, ldc, colMajor);
        }
    }
}

/* decompose2D, src/25DCannon.cpp:113-136 (tiles of M/p; sender is rank 0) */
void orc_cannon_decompose(int64_t M, int p, const double* A, const double* B, const double* C, double* const* lA,
                          double* const* lB, double* const* lC) {
    int64_t lm = M / p;
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) {
            int r = i * p + j;
            int64_t off = lm * (j * M + i);
            if (r == 0) {
                orc_copy_block(lm, lm, A + off, lA[r], M, lm, 1);
                orc_copy_block(lm, lm, B + off, lB[r], M, lm, 1);
                orc_copy_block(lm, lm, C + off, lC[r], M, lm, 1);
            } else {
                vector_transfer(lm, lm, A + off, M, lA[r], lm, 1);
                vector_transfer(lm, lm, B + off, M, lB[r], lm, 1);
                vector_transfer(lm, lm, C + off, M, lC[r], lm, 1);
            }
        }
}

/* reorderMatrix, src/25DCannon.cpp:254-271 (gather rank 0) */
void orc_cannon_reorder(int64_t M, int p, double* C, const double* const* lC) {
    int64_t lm = M / p;
    for (int i = 0; i < p; ++i)
        for (int j = 0; j < p; ++j) {
            int r = i * p + j;
            int64_t off = lm * (j * M + i);
            if (r == 0)
                orc_copy_block(lm, lm, lC[r], C + off, lm, M, 1);
            else
                vector_transfer(lm, lm, lC[r], lm, C + off, M, 1);
        }
}

/*
 * Cannon schedule.  After the skew (25DCannon.cpp:303-310) rank (i,j,k) holds A's and
 * B's k-block t_0 = (i + j - k*pc3) mod pc (A_ij went to column j - i + k*pc3, so the
 * receiver at column s holds A_{i, s+i-k*pc3}; the same for B by rows).  Rotation r
 * (:333-334, :364-365) sends every tile to column (j + r) mod pc, i.e. a shift by r,
 * so t_r = t_{r-1} - r.  truncatedDivisionRemainer (25DCannonNCCL.cpp:6-9) is the
 * non-negative modulo used here.
 */
static int nmod(int a, int b) { return ((a % b) + b) % b; }

int orc_cannon_schedule(int p, int c, int i, int j, int k, int* out) {
    int pc3 = (int)sqrt((double)(p * p * c) / (double)(c * c * c));
    int pc = (int)sqrt((double)(p * p * c) / (double)c);
    int t = nmod(i + j - k * pc3, pc);
    for (int r = 0; r < pc3; ++r) {
        if (r > 0) t = nmod(t - r, pc);
        out[r] = t;
    }
    /* coverage: the union over stacks of the steps of rank (i,j,*) */
    int seen[1024];
    if (pc > 1024) return 0;
    memset(seen, 0, sizeof(seen));
    for (int kk = 0; kk < c; ++kk) {
        int tt = nmod(i + j - kk * pc3, pc);
        for (int r = 0; r < pc3; ++r) {
            if (r > 0) tt = nmod(tt - r, pc);
            seen[tt]++;
        }
    }
    for (int q = 0; q < pc; ++q)
        if (seen[q] != 1) return 0;
    return 1;
}

/* ---- double-double checker ---------------------------------------------------- */
typedef struct {
    double hi, lo;
} dd;

static dd two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    dd r = {s, e};
    return r;
}

static dd dd_add_prod(dd acc, double a, double b) {
    double p = a * b;
    double pe = fma(a, b, -p); /* exact product error (TwoProduct) */
    dd s = two_sum(acc.hi, p);
    double lo = s.lo + acc.lo + pe;
    return two_sum(s.hi, lo);
}

void orc_dgemm_dd_sample(char ta, char tb, int64_t K, double alpha, const double* A, int64_t lda, const double* B,
                         int64_t ldb, double beta, const double* C0, int64_t ldc, int64_t n, const int64_t* rows,
                         const int64_t* cols, double* out) {
    int tA = (ta == 'T' || ta == 't' || ta == 'C' || ta == 'c');
    int tB = (tb == 'T' || tb == 't' || tb == 'C' || tb == 'c');
    for (int64_t s = 0; s < n; ++s) {
        int64_t i = rows[s], j = cols[s];
        dd acc = {0.0, 0.0};
        for (int64_t p = 0; p < K; ++p) {
            double a = tA ? A[p + i * lda] : A[i + p * lda];
            double b = tB ? B[j + p * ldb] : B[p + j * ldb];
            acc = dd_add_prod(acc, a, b);
        }
        /* alpha * acc in double-double, then + beta*C0 */
        double h = alpha * acc.hi;
        double he = fma(alpha, acc.hi, -h);
        dd r = two_sum(h, he + alpha * acc.lo);
        if (beta != 0.0 && C0) r = dd_add_prod(r, beta, C0[i + j * ldc]);
        out[s] = r.hi + r.lo;
    }
}

/* Sampled rows of alpha*op(A)*B in double-double, for the whole width of B: row s of op(A)
 * is At[0..K) + s*ldat (K-contiguous), column j of B is B + j*ldb, and the result (rounded
 * once to double) goes to out[s + j*ldo].  Columns are split across nthreads POSIX threads
 * (<= 0: one per online core); each thread carries four rows' accumulators at once so the
 * dependent TwoSum chains overlap. */
typedef struct {
    int64_t K, nrows, ldat, ldb, ldo, j0, j1;
    const double *At, *B;
    double alpha, *out;
} dd_rows_job;

static void* dd_rows_worker(void* arg) {
    const dd_rows_job* J = (const dd_rows_job*)arg;
    for (int64_t j = J->j0; j < J->j1; ++j) {
        const double* b = J->B + j * J->ldb;
        for (int64_t s = 0; s < J->nrows; s += 4) {
            const int64_t nr = J->nrows - s < 4 ? J->nrows - s : 4;
            dd acc[4] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
            const double* a[4];
            for (int r = 0; r < 4; ++r) a[r] = J->At + (s + (r < nr ? r : 0)) * J->ldat;
            for (int64_t p = 0; p < J->K; ++p) {
                const double bp = b[p];
                for (int r = 0; r < 4; ++r) acc[r] = dd_add_prod(acc[r], a[r][p], bp);
            }
            for (int r = 0; r < nr; ++r) {
                double h = J->alpha * acc[r].hi;
                double he = fma(J->alpha, acc[r].hi, -h);
                dd v = two_sum(h, he + J->alpha * acc[r].lo);
                J->out[(s + r) + j * J->ldo] = v.hi + v.lo;
            }
        }
    }
    return NULL;
}

void orc_dd_rows(int64_t K, int64_t nrows, const double* At, int64_t ldat, int64_t ncols, const double* B,
                 int64_t ldb, double alpha, double* out, int64_t ldo, int nthreads) {
    if (nthreads <= 0) {
        long c = sysconf(_SC_NPROCESSORS_ONLN);
        nthreads = c > 0 ? (int)c : 1;
    }
    if (nthreads > 256) nthreads = 256;
    if (nthreads > ncols) nthreads = ncols > 0 ? (int)ncols : 1;
    pthread_t tid[256];
    dd_rows_job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        dd_rows_job J = {K, nrows, ldat, ldb, ldo, ncols * t / nthreads, ncols * (t + 1) / nthreads, At, B, alpha, out};
        jobs[t] = J;
    }
    int started = 0;
    for (int t = 1; t < nthreads; ++t)
        if (pthread_create(&tid[t], NULL, dd_rows_worker, &jobs[t]) == 0)
            started = t;
        else
            break;
    /* threads that could not start run here, after this thread's own share */
    dd_rows_worker(&jobs[0]);
    for (int t = started + 1; t < nthreads; ++t) dd_rows_worker(&jobs[t]);
    for (int t = 1; t <= started; ++t) pthread_join(tid[t], NULL);
}
