// Command-line 2.5D Cannon benchmark with the reference's arguments and CSV logs
// (src/Benchmarks/cuBLAS25Benchmark.cpp:3-82), on this library's drivers
// (include/dgt_drivers.hpp): the whole dRow x dCol x C grid runs on the current GPU.
//
//   dgt_cublas25d_benchmark '{TransA}{TransB}' M N K alpha beta dRow dCol C numberOfRuns
//                           dataLocation={host,devices} [fullOffload]
//                           [--mode native|ozaki|ozaki2|bf16] [--slices S] [--machine NAME]
//                           [--logdir DIR] [--seed SEED]
//
// As in the reference: a 12th positional argument selects the full-offload driver (global
// A, B, C generated on the host, decomposed, multiplied, gathered every run), otherwise the
// pre-distributed driver (operands generated on the tiles, no gather); dataLocation is
// validated but does not change the run; logging is always on.  Operands are U[-1, 1) from
// std::mt19937_64(seed) instead of the reference's wall-clock-seeded generator.  Errors
// print a message and return a non-zero status instead of aborting.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dgt_drivers.hpp"

static const char* kUsage =
    "Usage: dgt_cublas25d_benchmark '{TransA}{TransB}' M N K alpha beta dRow dCol C numberOfRuns "
    "dataLocation={host,devices} fullOffload{default=false} [--mode native|ozaki|ozaki2|bf16] [--slices S] "
    "[--machine NAME] [--logdir DIR] [--seed SEED]\n";

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    dgt::DriverOptions opt;
    bool slices_set = false;
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        if (s.rfind("--", 0) == 0) {
            if (a + 1 >= argc) {
                std::fprintf(stderr, "%s needs a value\n%s", s.c_str(), kUsage);
                return 1;
            }
            std::string v = argv[++a];
            if (s == "--mode") {
                if (v == "native") opt.mode = DGT_FP64_NATIVE;
                else if (v == "ozaki") opt.mode = DGT_FP64_OZAKI_INT8;
                else if (v == "ozaki2") opt.mode = DGT_FP64_OZAKI2_INT8;
                else if (v == "bf16") opt.mode = DGT_FP64_OZAKI_BF16;
                else {
                    std::fprintf(stderr, "unknown mode %s\n%s", v.c_str(), kUsage);
                    return 1;
                }
            } else if (s == "--slices") {
                opt.slices = std::atoi(v.c_str());
                slices_set = true;
            } else if (s == "--machine") {
                opt.machine = v;
            } else if (s == "--logdir") {
                opt.logDir = v;
            } else if (s == "--seed") {
                opt.seed = std::strtoull(v.c_str(), nullptr, 10);
            } else {
                std::fprintf(stderr, "unknown option %s\n%s", s.c_str(), kUsage);
                return 1;
            }
        } else {
            pos.push_back(s);
        }
    }
    if (pos.size() < 11 || pos[0].size() < 2) {
        std::fprintf(stderr, "%s", kUsage);
        return 1;
    }
    if (!slices_set && opt.mode == DGT_FP64_OZAKI2_INT8) opt.slices = 15;
    if (!slices_set && opt.mode != DGT_FP64_OZAKI2_INT8 && opt.mode != DGT_FP64_NATIVE) opt.slices = 8;
    const char ta = pos[0][0], tb = pos[0][1];
    const long long M = std::atoll(pos[1].c_str()), N = std::atoll(pos[2].c_str()), K = std::atoll(pos[3].c_str());
    const double alpha = std::atof(pos[4].c_str()), beta = std::atof(pos[5].c_str());
    const int dRow = std::atoi(pos[6].c_str()), dCol = std::atoi(pos[7].c_str()), c = std::atoi(pos[8].c_str());
    const int runs = std::atoi(pos[9].c_str());
    const std::string dataLocation = pos[10];
    const bool fullOffload = pos.size() >= 12;
    if (dataLocation != "host" && dataLocation != "devices") {
        std::printf("Initial Data location not recognized, check usage\n%s", kUsage);
        return 2;
    }
    if (M <= 0 || N <= 0 || K <= 0 || runs < 1) {
        std::fprintf(stderr, "sizes and numberOfRuns must be positive\n%s", kUsage);
        return 1;
    }
    try {
        if (fullOffload) {
            std::printf("Running Full Offload 2.5D SUMMA dgt Run (%d runs) with M=%lld, N=%lld, K=%lld on a %dx%dx%d grid\n",
                        runs, M, N, K, dRow, dCol, c);
            std::mt19937_64 rng(opt.seed);
            std::uniform_real_distribution<double> U(-1.0, 1.0);
            std::vector<double> A(size_t(M) * size_t(K)), B(size_t(K) * size_t(N)), C(size_t(M) * size_t(N));
            for (auto* v : {&A, &B, &C})
                for (auto& x : *v) x = U(rng);
            dgt::fullOffloadSumma25Dgemm(ta, tb, M, N, K, alpha, A.data(), M, B.data(), K, beta, C.data(), M, dRow,
                                         dCol, c, runs, true, true, opt);
        } else {
            std::printf("Running Pre Distributed 2.5D SUMMA dgt Run (%d runs) with M=%lld, N=%lld, K=%lld on a %dx%dx%d grid\n",
                        runs, M, N, K, dRow, dCol, c);
            dgt::preDistributedSumma25Dgemm(ta, tb, M, N, K, alpha, nullptr, M, nullptr, K, beta, nullptr, M, dRow,
                                            dCol, c, runs, true, false, opt);
        }
    } catch (const dgt::Error& e) {
        std::fprintf(stderr, "dgt error (status %d): %s\n", int(e.status), e.what());
        return 3;
    }
    return 0;
}
