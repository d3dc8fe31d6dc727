// C entry points that run the reference's OWN hot-path classes (compiled from the
// reference tree by oracle/Makefile) as an in-process MPI job, one host thread per
// virtual rank.  Used only by tests/ (golden fixtures, pinning the restatement) and by
// bench.py's CPU reference arm.  Every entry returns 0 on success, -1 on failure
// (message via ref_last_error()).
#include <unistd.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "2DBlockSequentialDecomposition.hpp"
#include "25DCannon.hpp"
#include "pblasDecomposition.hpp"
#include "transfers.hpp"

int fake_mpi_run(int size, const std::function<void(int)>& fn, std::string* err);
extern "C" void ref_set_process_grid(int dRow, int dCol);
extern "C" void ref_set_dgemm(void* fn);
extern "C" void* ref_get_dgemm(void);

static std::mutex g_run_mutex;  // one job at a time (the test doubles hold global state)
static std::string g_err;

extern "C" const char* ref_last_error(void) { return g_err.c_str(); }

static int run_job(int size, const std::function<void(int)>& fn) {
    g_err.clear();
    std::string err;
    int rc = fake_mpi_run(size, fn, &err);
    if (rc != 0) g_err = err;
    return rc;
}

extern "C" int ref_numroc(int n, int nb, int iproc, int isrproc, int nprocs) {
    return numroc(n, nb, iproc, isrproc, nprocs);
}

// ---- block-cyclic (src/Decompositions/pblasDecomposition.cpp) ------------------------

static bool pblas_guard(int M, int N, int Mb, int Nb, int dRow, int dCol) {
    // The reference divides by localRows / localColumns (pblasDecomposition.cpp:125,130);
    // a rank that owns no rows or no columns would divide by zero, so refuse such grids.
    for (int r = 0; r < dRow; ++r)
        if (numroc(M, Mb, r, 0, dRow) <= 0) return false;
    for (int c = 0; c < dCol; ++c)
        if (numroc(N, Nb, c, 0, dCol) <= 0) return false;
    return M > 0 && N > 0 && Mb > 0 && Nb > 0;
}

extern "C" int ref_pblas_shapes(int M, int N, int Mb, int Nb, int dRow, int dCol, int* rows, int* cols, int* blocks) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    ref_set_process_grid(dRow, dCol);
    return run_job(dRow * dCol, [&](int rank) {
        pblasDecomposer d(M, N, Mb, Nb, MPI_COMM_WORLD);
        rows[rank] = d.localRows;
        cols[rank] = d.localColumns;
        blocks[rank] = d.myBlocks;
    });
}

extern "C" int ref_pblas_scatter(int M, int N, int Mb, int Nb, int dRow, int dCol, double* global, double** locals) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!pblas_guard(M, N, Mb, Nb, dRow, dCol)) {
        g_err = "grid leaves a rank without rows or columns (reference divides by zero)";
        return -1;
    }
    ref_set_process_grid(dRow, dCol);
    return run_job(dRow * dCol, [&](int rank) {
        pblasDecomposer d(M, N, Mb, Nb, MPI_COMM_WORLD);
        d.scatterMatrix(0, global, locals[rank]);
    });
}

extern "C" int ref_pblas_gather(int M, int N, int Mb, int Nb, int dRow, int dCol, double* global, double** locals) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!pblas_guard(M, N, Mb, Nb, dRow, dCol)) {
        g_err = "grid leaves a rank without rows or columns (reference divides by zero)";
        return -1;
    }
    ref_set_process_grid(dRow, dCol);
    return run_job(dRow * dCol, [&](int rank) {
        pblasDecomposer d(M, N, Mb, Nb, MPI_COMM_WORLD);
        d.gatherMatrix(0, global, locals[rank]);
    });
}

// ---- 2D block (src/Decompositions/2DBlockSequentialDecomposition.cpp) ---------------

extern "C" int ref_block2d_shapes(int M, int N, int K, int P, int* dRow, int* dCol, int* localM, int* localN) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    return run_job(P, [&](int rank) {
        BlockSequentialDecomposer d(M, N, K, MPI_COMM_WORLD, true);
        if (rank == 0) {
            *dRow = d.dRow;
            *dCol = d.dCol;
        }
        localM[rank] = d.localM;
        localN[rank] = d.localN;
    });
}

extern "C" int ref_block2d_deliver(int M, int N, int K, int P, int colMajor, double* gA, double* gB, double* gC,
                                   double** lA, double** lB, double** lC) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    return run_job(P, [&](int rank) {
        BlockSequentialDecomposer d(M, N, K, MPI_COMM_WORLD, colMajor != 0);
        double* a = lA[rank];
        double* b = lB[rank];
        double* c = lC[rank];
        d.deliverMatrix(gA, gB, gC, &a, &b, &c);
    });
}

extern "C" int ref_block2d_gather(int M, int N, int K, int P, int colMajor, int gatherRank, double* C, double** lC) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    return run_job(P, [&](int rank) {
        BlockSequentialDecomposer d(M, N, K, MPI_COMM_WORLD, colMajor != 0);
        d.gatherResult(gatherRank, C, lC[rank]);
    });
}

// ---- 2.5D Cannon (src/25DCannon.cpp) -------------------------------------------------

static bool cannon_guard(long long M, int p, int c) {
    if (M <= 0 || p <= 0 || c <= 0 || M % p != 0 || p % c != 0) return false;
    return true;
}

// decompose2D only: the stack-0 tiles that rank i*p+j receives.
extern "C" int ref_cannon_decompose(long long M, int p, int c, double* A, double* B, double* C, double** lA,
                                    double** lB, double** lC) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!cannon_guard(M, p, c)) {
        g_err = "Cannon needs M % p == 0 and p % c == 0";
        return -1;
    }
    return run_job(p * p * c, [&](int rank) {
        Summa25Decomposer d(M, M, M, p, p, c, false);
        d.decompose2D(0, A, B, C, d.localA, d.localB, d.localC);
        if (d.processStack == 0) {
            size_t t = (size_t)d.localM * d.localK;
            std::memcpy(lA[rank], d.localA, t * sizeof(double));
            std::memcpy(lB[rank], d.localB, t * sizeof(double));
            std::memcpy(lC[rank], d.localC, t * sizeof(double));
        }
    });
}

// reorderMatrix only: gather stack-0 tiles lC[rank] into C on rank 0.
extern "C" int ref_cannon_reorder(long long M, int p, int c, double* C, double** lC) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!cannon_guard(M, p, c)) {
        g_err = "Cannon needs M % p == 0 and p % c == 0";
        return -1;
    }
    return run_job(p * p * c, [&](int rank) {
        Summa25Decomposer d(M, M, M, p, p, c, false);
        if (d.processStack == 0) std::memcpy(d.localC, lC[rank], (size_t)d.localM * d.localN * sizeof(double));
        d.reorderMatrix(0, C, d.localC);
    });
}

// The reference's full-offload 2.5D Cannon (fullOffloadSumma25Dgemm, src/25DCannon.cpp:392-459,
// without logging): decompose2D -> multiply -> reorderMatrix.  C is overwritten with
// alpha*A*B + beta*C on return.  The host GEMM behind cublasDgemm is ref_set_dgemm's.
extern "C" int ref_cannon_fulloffload(long long M, int p, int c, double alpha, double beta, double* A, double* B,
                                      double* C) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!cannon_guard(M, p, c)) {
        g_err = "Cannon needs M % p == 0 and p % c == 0";
        return -1;
    }
    return run_job(p * p * c, [&](int rank) {
        Summa25Decomposer d(M, M, M, p, p, c, false);
        d.decompose2D(0, A, B, C, d.localA, d.localB, d.localC);
        d.multiply('N', 'N', A, B, C, alpha, beta);
        d.reorderMatrix(0, C, d.localC);
    });
}

// The reference's full-offload driver itself, logging on (fullOffloadSumma25Dgemm,
// src/25DCannon.cpp:392-459): run in `dir`, where its own createLogCsv / writeLineToFile
// (src/Utilities/Logging.cpp) create or extend its CSV log, one row per run.  Its node count
// comes from SLURM_JOB_NUM_NODES, set to 1 here when absent (the reference reads it
// unchecked).  The working directory is the process's, so it is restored before returning.
extern "C" int ref_cannon_fulloffload_logged(const char* dir, long long M, int p, int c, double alpha, double beta,
                                             double* A, double* B, double* C, int runs) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    if (!cannon_guard(M, p, c) || runs < 1 || !dir) {
        g_err = "Cannon needs M % p == 0, p % c == 0, runs >= 1 and a directory";
        return -1;
    }
    setenv("SLURM_JOB_NUM_NODES", "1", 0);
    char old[4096];
    if (!getcwd(old, sizeof(old)) || chdir(dir) != 0) {
        g_err = "cannot enter the log directory";
        return -1;
    }
    int rc = run_job(p * p * c, [&](int) {
        fullOffloadSumma25Dgemm('N', 'N', M, M, M, alpha, A, M, B, M, beta, C, M, p, p, c, runs, true, true);
    });
    if (chdir(old) != 0 && rc == 0) {
        g_err = "cannot return to the working directory";
        rc = -1;
    }
    return rc;
}

// The reference's copyBlock in its two instantiations (src/Transfers/sharedTransfers.cpp:29-63,
// :87-88), on host memory through the CUDA test double: its contiguous shortcut included.
extern "C" int ref_copy_block_f64(long long rows, long long cols, double* src, double* dst, long long ldS,
                                  long long ldD, int colMajor) {
    copyBlock<double>(rows, cols, src, dst, ldS, ldD, colMajor != 0);
    return 0;
}
extern "C" int ref_copy_block_f32(long long rows, long long cols, float* src, float* dst, long long ldS,
                                  long long ldD, int colMajor) {
    copyBlock<float>(rows, cols, src, dst, ldS, ldD, colMajor != 0);
    return 0;
}

// Step trace of the Cannon schedule: for every world rank and every local GEMM it
// issues, the k-block index of the A and B tiles it multiplies.  A's global block
// (bi,bk) and B's block (bk,bj) are filled with the value bk, so the first element
// of each operand the GEMM sees names the block.  trace has p*p*c*(p/c)*2 ints.
static thread_local int tl_step = 0;
static int* g_trace = nullptr;
static int g_trace_steps = 0;
int fake_mpi_world_rank(void);

static void trace_dgemm(int, int, int, int, int, int, double, const double* A, int, const double* B, int, double,
                        double*, int) {
    int r = fake_mpi_world_rank();
    int s = tl_step++;
    if (s < g_trace_steps) {
        g_trace[(r * g_trace_steps + s) * 2 + 0] = (int)A[0];
        g_trace[(r * g_trace_steps + s) * 2 + 1] = (int)B[0];
    }
}

extern "C" int ref_cannon_trace(int p, int c, int* trace) {
    std::lock_guard<std::mutex> g(g_run_mutex);
    long long M = 2LL * p;
    if (!cannon_guard(M, p, c)) {
        g_err = "Cannon needs p % c == 0";
        return -1;
    }
    int pc3 = (int)std::sqrt((double)(p * p * c) / (double)(c * c * c));
    std::vector<double> A(M * M), B(M * M), C(M * M, 0.0);
    long long bs = M / p;
    for (long long col = 0; col < M; ++col)
        for (long long row = 0; row < M; ++row) {
            A[row + col * M] = (double)(col / bs);  // k-block of A is its column block
            B[row + col * M] = (double)(row / bs);  // k-block of B is its row block
        }
    g_trace = trace;
    g_trace_steps = pc3;
    void* saved = ref_get_dgemm();
    ref_set_dgemm((void*)&trace_dgemm);
    int rc = run_job(p * p * c, [&](int rank) {
        tl_step = 0;
        Summa25Decomposer d(M, M, M, p, p, c, false);
        d.decompose2D(0, A.data(), B.data(), C.data(), d.localA, d.localB, d.localC);
        d.multiply('N', 'N', A.data(), B.data(), C.data(), 1.0, 0.0);
    });
    ref_set_dgemm(saved);
    g_trace = nullptr;
    return rc;
}
