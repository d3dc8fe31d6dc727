// Drives the C++ mirror classes (include/dgt_mirror.hpp) the way the reference's own
// test drivers drive its classes: src/Tests/summa25Dtest.cpp (decompose2D -> multiply ->
// reorderMatrix -> compare), src/Tests/sequentialDecomposerTest.cpp (deliverMatrix /
// gatherResult) and the block-cyclic scatter / gather of the cuBLASMp validator
// (src/Wrappers/cuBLASMp/cuBLASMpValidator.cpp:31-50).  The host check is a plain
// column-major triple loop; the pass rule is the reference's Dtest_equality digit count
// (src/Utilities/Validation.cpp:57-83) with |a| in the denominator.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "dgt_mirror.hpp"

static int digits(const std::vector<double>& ref, const std::vector<double>& got) {
    auto failed = [&](double eps) {
        for (size_t i = 0; i < ref.size(); ++i) {
            double a = ref[i], d = std::fabs(a - got[i]);
            double e = (a == 0.0) ? d : d / std::fabs(a);
            if (e > eps) return true;
        }
        return false;
    };
    int acc = 8;
    double eps = 1e-8;
    bool f = failed(eps);
    while (eps > 2.2250738585072014e-308 && !f && acc < 30) {
        eps *= 0.1;
        ++acc;
        f = failed(eps);
    }
    return acc == 8 ? 0 : acc;
}

static double* dmalloc(size_t n) {
    double* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(double) + 8) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    return p;
}

static int test_cannon(dgt::Context& ctx, long long M, int p, int c) {
    std::mt19937_64 rng(42);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<double> A(M * M), B(M * M), C(M * M), ref(M * M);
    for (auto& x : A) x = U(rng);
    for (auto& x : B) x = U(rng);
    for (auto& x : C) x = U(rng);
    const double alpha = 1.5, beta = -0.5;
    for (long long j = 0; j < M; ++j)
        for (long long i = 0; i < M; ++i) {
            double s = 0;
            for (long long k = 0; k < M; ++k) s += A[i + k * M] * B[k + j * M];
            ref[i + j * M] = alpha * s + beta * C[i + j * M];
        }
    dgt::Summa25Decomposer dec(ctx.get(), M, M, M, p, p, c);
    double *dA = dmalloc(M * M), *dB = dmalloc(M * M), *dC = dmalloc(M * M);
    cudaMemcpy(dA, A.data(), M * M * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B.data(), M * M * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dC, C.data(), M * M * 8, cudaMemcpyHostToDevice);
    std::vector<double*> tA, tB, tC;
    for (int r = 0; r < p * p; ++r) {
        tA.push_back(dmalloc(dec.localM * dec.localK));
        tB.push_back(dmalloc(dec.localK * dec.localN));
        tC.push_back(dmalloc(dec.localM * dec.localN));
    }
    dec.decompose2D(dA, dB, dC, tA.data(), tB.data(), tC.data());
    dec.multiply('N', 'N', tA.data(), tB.data(), tC.data(), alpha, beta);
    dec.reorderMatrix(dC, tC.data());
    std::vector<double> got(M * M);
    cudaMemcpy(got.data(), dC, M * M * 8, cudaMemcpyDeviceToHost);
    dgt::check(ctx.get(), dgt_check_device(ctx.get()));
    int acc = digits(ref, got);
    std::printf("cannon M=%lld p=%d c=%d: %d digits\n", M, p, c, acc);
    for (int r = 0; r < p * p; ++r) {
        cudaFree(tA[r]);
        cudaFree(tB[r]);
        cudaFree(tC[r]);
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return acc >= 12 ? 0 : 1;
}

static int test_pblas(dgt::Context& ctx, int M, int N, int Mb, int Nb, int p, int q) {
    std::vector<double> G(size_t(M) * N), back(size_t(M) * N);
    for (size_t i = 0; i < G.size(); ++i) G[i] = double(i);
    dgt::pblasDecomposer dec(ctx.get(), M, N, Mb, Nb, p, q);
    double* dG = dmalloc(G.size());
    cudaMemcpy(dG, G.data(), G.size() * 8, cudaMemcpyHostToDevice);
    std::vector<double*> locs;
    for (int r = 0; r < p * q; ++r) locs.push_back(dmalloc(size_t(std::max(dec.localRows[r], 1)) * dec.localColumns[r]));
    dec.scatterMatrix(dG, locs.data());
    // rank 0's first block must be the global top-left block (pblasDecomposition.cpp:113)
    std::vector<double> l0(size_t(dec.localRows[0]) * dec.localColumns[0]);
    cudaMemcpy(l0.data(), locs[0], l0.size() * 8, cudaMemcpyDeviceToHost);
    int bad = 0;
    for (int j = 0; j < std::min(Nb, N); ++j)
        for (int i = 0; i < std::min(Mb, M); ++i) bad += l0[i + size_t(j) * dec.localRows[0]] != G[i + size_t(j) * M];
    cudaMemset(dG, 0, G.size() * 8);
    dec.gatherMatrix(dG, locs.data());
    cudaMemcpy(back.data(), dG, G.size() * 8, cudaMemcpyDeviceToHost);
    bad += std::memcmp(back.data(), G.data(), G.size() * 8) != 0;
    std::printf("pblas %dx%d (%d,%d) on %dx%d: %s\n", M, N, Mb, Nb, p, q, bad ? "FAIL" : "ok");
    for (auto* l : locs) cudaFree(l);
    cudaFree(dG);
    return bad ? 1 : 0;
}

static int test_block2d(dgt::Context& ctx, int M, int N, int K, int P) {
    dgt::BlockSequentialDecomposer dec(ctx.get(), M, N, K, P, true);
    std::vector<double> A(size_t(M) * K), B(size_t(K) * N), C(size_t(M) * N), back(size_t(M) * N);
    for (size_t i = 0; i < A.size(); ++i) A[i] = double(i);
    for (size_t i = 0; i < B.size(); ++i) B[i] = -double(i);
    for (size_t i = 0; i < C.size(); ++i) C[i] = 0.5 * double(i);
    double *dA = dmalloc(A.size()), *dB = dmalloc(B.size()), *dC = dmalloc(C.size());
    cudaMemcpy(dA, A.data(), A.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B.data(), B.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(dC, C.data(), C.size() * 8, cudaMemcpyHostToDevice);
    std::vector<double*> lA, lB, lC;
    for (int r = 0; r < P; ++r) {
        lA.push_back(dmalloc(size_t(dec.localM[r]) * K));
        lB.push_back(dmalloc(size_t(K) * dec.localN[r]));
        lC.push_back(dmalloc(size_t(dec.localM[r]) * dec.localN[r]));
    }
    dec.deliverMatrix(dA, dB, dC, lA.data(), lB.data(), lC.data());
    cudaMemset(dC, 0, C.size() * 8);
    dec.gatherResult(dC, lC.data());
    cudaMemcpy(back.data(), dC, C.size() * 8, cudaMemcpyDeviceToHost);
    int bad = std::memcmp(back.data(), C.data(), C.size() * 8) != 0;
    std::printf("block2d %dx%dx%d P=%d (grid %dx%d): %s\n", M, N, K, P, dec.dRow, dec.dCol, bad ? "FAIL" : "ok");
    for (int r = 0; r < P; ++r) {
        cudaFree(lA[r]);
        cudaFree(lB[r]);
        cudaFree(lC[r]);
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return bad;
}

int main() {
    try {
        dgt::Context ctx;
        int fails = 0;
        fails += test_cannon(ctx, 64, 2, 1);
        fails += test_cannon(ctx, 96, 4, 2);
        fails += test_cannon(ctx, 90, 3, 1);  // the reference's schedule misses k-blocks here
        fails += test_pblas(ctx, 150, 170, 16, 16, 4, 4);
        fails += test_pblas(ctx, 37, 29, 5, 4, 2, 3);
        fails += test_block2d(ctx, 20, 20, 20, 2);
        fails += test_block2d(ctx, 33, 17, 8, 5);
        bool threw = false;
        try {
            dgt::Summa25Decomposer bad(ctx.get(), 64, 64, 32, 2, 2, 1);
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
