// Runs the reference-shaped 2.5D Cannon drivers of include/dgt_drivers.hpp the way the
// reference's benchmarks call theirs (src/25DCannon.cpp:392-530), logging into argv[1]:
//  * fullOffloadSumma25Dgemm from pageable host matrices (lda > M for A) with gather: after
//    R runs, C = alpha A B (1 + beta + ... + beta^(R-1)) + beta^R C0 (every run applies the
//    GEMM to the same tiles), checked against a host triple loop to 12 digits;
//  * the same from page-locked A, B, C (ld = M): packed and gathered straight from host memory;
//  * preDistributedSumma25Dgemm with gather: the operands are the documented seeded
//    stream (global A, B, C from std::mt19937_64(seed)), so the host recomputes the result;
//  * the CSV rows each run appends (read back with pandas by the Python tests that run this);
//  * a non-square problem is rejected with DGT_ERROR_INVALID_VALUE, as the reference's
//    constructor rejects it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "dgt_drivers.hpp"

static double rel_fro(const std::vector<double>& ref, const std::vector<double>& got, long long M, long long ld) {
    double num = 0, den = 0;
    for (long long j = 0; j < M; ++j)
        for (long long i = 0; i < M; ++i) {
            double r = ref[i + j * M], d = got[i + j * ld] - r;
            num += d * d;
            den += r * r;
        }
    return std::sqrt(num / den);
}

static void host_gemm(const std::vector<double>& A, long long lda, const std::vector<double>& B,
                      std::vector<double>& AB, long long M) {
    for (long long j = 0; j < M; ++j)
        for (long long i = 0; i < M; ++i) {
            double s = 0;
            for (long long k = 0; k < M; ++k) s += A[i + k * lda] * B[k + j * M];
            AB[i + j * M] = s;
        }
}

static int test_full_offload(const char* dir, long long M, int p, int c, int runs) {
    const long long lda = M + 3, ldc = M + 1;
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> A(lda * M), B(M * M), C(ldc * M), C0(M * M), AB(M * M), ref(M * M);
    for (auto& x : A) x = U(rng);
    for (auto& x : B) x = U(rng);
    for (auto& x : C) x = U(rng);
    for (long long j = 0; j < M; ++j)
        for (long long i = 0; i < M; ++i) C0[i + j * M] = C[i + j * ldc];
    const double alpha = 1.5, beta = -0.5;
    host_gemm(A, lda, B, AB, M);
    double geo = 0, bR = 1;
    for (int r = 0; r < runs; ++r) {
        geo += bR;
        bR *= beta;
    }
    for (long long i = 0; i < M * M; ++i) ref[i] = alpha * AB[i] * geo + bR * C0[i];
    dgt::DriverOptions opt;
    opt.logDir = dir;
    opt.machine = "b200test";
    dgt::fullOffloadSumma25Dgemm('N', 'N', M, M, M, alpha, A.data(), lda, B.data(), M, beta, C.data(), ldc, p, p, c,
                                 runs, true, true, opt);
    const double e = rel_fro(ref, C, M, ldc);
    std::printf("full offload M=%lld grid %dx%dx%d runs=%d: rel Frobenius %.3e\n", M, p, p, c, runs, e);
    return e <= 1e-12 ? 0 : 1;
}

// A, B, C in page-locked host memory with ld = M, as the reference's test allocates them
// (src/Tests/summa25Dtest.cpp:40-42): the driver packs and gathers straight from host memory.
static int test_full_offload_pinned(const char* dir, long long M, int p, int c) {
    double *A = nullptr, *B = nullptr, *C = nullptr;
    const size_t n = size_t(M) * size_t(M);
    if (cudaMallocHost((void**)&A, n * 8) != cudaSuccess || cudaMallocHost((void**)&B, n * 8) != cudaSuccess ||
        cudaMallocHost((void**)&C, n * 8) != cudaSuccess)
        return 1;
    std::mt19937_64 rng(13);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (size_t i = 0; i < n; ++i) A[i] = U(rng);
    for (size_t i = 0; i < n; ++i) B[i] = U(rng);
    for (size_t i = 0; i < n; ++i) C[i] = U(rng);
    std::vector<double> Av(A, A + n), Bv(B, B + n), AB(n), ref(n);
    host_gemm(Av, M, Bv, AB, M);
    for (size_t i = 0; i < n; ++i) ref[i] = 1.5 * AB[i] - 0.5 * C[i];
    dgt::DriverOptions opt;
    opt.logDir = dir;
    opt.machine = "b200test";
    dgt::fullOffloadSumma25Dgemm('N', 'N', M, M, M, 1.5, A, M, B, M, -0.5, C, M, p, p, c, 1, true, true, opt);
    std::vector<double> got(C, C + n);
    const double e = rel_fro(ref, got, M, M);
    std::printf("full offload from page-locked memory M=%lld grid %dx%dx%d: rel Frobenius %.3e\n", M, p, p, c, e);
    cudaFreeHost(A);
    cudaFreeHost(B);
    cudaFreeHost(C);
    return e <= 1e-12 ? 0 : 1;
}

static int test_pre_distributed(const char* dir, long long M, int p, int c) {
    const uint64_t seed = 11;
    const double alpha = 1.0, beta = 0.25;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> A(M * M), B(M * M), C0(M * M), AB(M * M), ref(M * M), C(M * M, 0.0);
    for (auto& x : A) x = U(rng);
    for (auto& x : B) x = U(rng);
    for (auto& x : C0) x = U(rng);
    host_gemm(A, M, B, AB, M);
    for (long long i = 0; i < M * M; ++i) ref[i] = alpha * AB[i] + beta * C0[i];
    dgt::DriverOptions opt;
    opt.logDir = dir;
    opt.machine = "b200test";
    opt.seed = seed;
    dgt::preDistributedSumma25Dgemm('N', 'N', M, M, M, alpha, nullptr, M, nullptr, M, beta, C.data(), M, p, p, c, 1,
                                    true, true, opt);
    const double e = rel_fro(ref, C, M, M);
    std::printf("pre-distributed M=%lld grid %dx%dx%d: rel Frobenius %.3e\n", M, p, p, c, e);
    return e <= 1e-12 ? 0 : 1;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    try {
        int fails = 0;
        fails += test_full_offload(argv[1], 64, 2, 1, 2);
        fails += test_full_offload(argv[1], 96, 4, 2, 1);
        fails += test_full_offload_pinned(argv[1], 64, 2, 1);
        fails += test_pre_distributed(argv[1], 96, 4, 2);
        bool threw = false;
        std::vector<double> X(64 * 64, 0.0);
        try {
            dgt::fullOffloadSumma25Dgemm('N', 'N', 64, 64, 32, 1.0, X.data(), 64, X.data(), 64, 0.0, X.data(), 64, 2,
                                         2, 1, 1, false, false);
        } catch (const dgt::Error& e) {
            threw = e.status == DGT_ERROR_INVALID_VALUE;
        }
        fails += threw ? 0 : 1;
        std::printf("%s\n", fails ? "FAILED" : "ALL OK");
        return fails ? 1 : 0;
    } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
        return 2;
    }
}
