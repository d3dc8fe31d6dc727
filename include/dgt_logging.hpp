// Execution logs in the reference's CSV schema, so that the thesis's plotting notebooks
// (plotters/executionAnalysis.ipynb, plotters/thesisPlotters.ipynb: pandas.read_csv with
// header=0, rows grouped by Algo, M, N, K, TotalGPUs, DataLocation) read runs of this
// library without change.  Host-only C++17; no CUDA.
//
//   createLogCsv / writeLineToFile   src/Utilities/Logging.cpp:3-36
//   calculateGflops                  src/Utilities/GeneralUtilities.cpp:8-11
//   getSlurmNumNodes                 src/Utilities/GeneralUtilities.cpp:3-6
//   2.5D Cannon file names, header   src/25DCannon.cpp:405-408 (full offload), :475-478 (pre-distributed)
//   2.5D Cannon row                  src/25DCannon.cpp:443-446, :522-525
//
// Differences, all on error paths: createLogCsv returns nullptr where the reference exits,
// getSlurmNumNodes returns 1 when SLURM_JOB_NUM_NODES is unset (the reference passes the
// null getenv result to atoi), and nothing is printed.
#ifndef DGT_LOGGING_HPP
#define DGT_LOGGING_HPP

#include <unistd.h>

#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace dgt {

// Column header of the 2.5D Cannon logs (src/25DCannon.cpp:407, :477).
inline const char* cannonLogHeader() {
    return "Algo,M,N,K,TotalNodes,TotalGPUs,dRow,dCol,StackSize,DecompositionTime,ExecutionTime,GatherTime,"
           "GFlops,DataLocation,CommunicationTime,GemmCallTime";
}

// "DGEMM_execution_logs-<PreDistributed|FullOffload>_GEMM-<machine>-2.5DCANNON-<impl>.csv";
// the reference's impl is "cuBLAS".
inline std::string cannonLogFileName(bool preDistributed, const std::string& machine, const std::string& impl) {
    return std::string("DGEMM_execution_logs-") + (preDistributed ? "PreDistributed_GEMM-" : "FullOffload_GEMM-") +
           machine + "-2.5DCANNON-" + impl + ".csv";
}

// Opens `filename` for appending.  The header is written unless the file's first line is
// exactly `header` followed by a newline; a file that starts with any other line gets the
// header appended after its last line, as the reference does.  nullptr if the file cannot
// be opened.
inline FILE* createLogCsv(const std::string& filename, const std::string& header) {
    FILE* f = std::fopen(filename.c_str(), "a+");
    if (!f) return nullptr;
    char* line = nullptr;
    size_t cap = 0;
    const bool placed = getline(&line, &cap, f) != -1 && header + "\n" == line;
    std::free(line);
    if (!placed) {
        std::fputs(header.c_str(), f);
        std::fputs("\n", f);
    }
    return f;
}

inline void writeLineToFile(FILE* logfile, const char* dataLine) { std::fputs(dataLine, logfile); }

// 2 M N K / t in GFLOP/s, with the product formed in 64-bit integers as the reference does.
inline double calculateGflops(long long M, long long N, long long K, double executionTime) {
    return (2 * M * N * K * 1e-9) / executionTime;
}

inline int getSlurmNumNodes() {
    const char* v = std::getenv("SLURM_JOB_NUM_NODES");
    return v ? std::atoi(v) : 1;
}

// Machine name used in log file names: the compile-time DGT_MACHINE_NAME (the reference's
// MACHINE_NAME definition, CMakeLists.txt:92), else the environment variable of that name,
// else the host name, else "unknown".
inline std::string machineName() {
#ifdef DGT_MACHINE_NAME
    return DGT_MACHINE_NAME;
#else
    if (const char* v = std::getenv("DGT_MACHINE_NAME")) return v;
    char buf[HOST_NAME_MAX + 1] = {};
    if (gethostname(buf, sizeof(buf) - 1) == 0 && buf[0]) return buf;
    return "unknown";
#endif
}

// printf into a string of exactly the needed length.
__attribute__((format(printf, 1, 2))) inline std::string formatString(const char* fmt, ...) {
    va_list ap, ap2;
    va_start(ap, fmt);
    va_copy(ap2, ap);
    const int n = std::vsnprintf(nullptr, 0, fmt, ap);
    va_end(ap);
    std::string out;
    if (n > 0) {
        out.resize(size_t(n) + 1);
        std::vsnprintf(&out[0], out.size(), fmt, ap2);
        out.resize(size_t(n));
    }
    va_end(ap2);
    return out;
}

// One row of the 2.5D Cannon log, times in seconds, with the reference's printf format.
inline std::string cannonCsvLine(const char* algo, long long M, long long N, long long K, int totalNodes,
                                 int totalGPUs, int dRow, int dCol, int stackSize, double decompositionTime,
                                 double executionTime, double gatherTime, double gflops, const char* dataLocation,
                                 double communicationTime, double gemmCallTime) {
    return formatString("%s,%lld,%lld,%lld,%d,%d,%d,%d,%d,%lf,%lf,%lf,%lf,%s,%lf,%lf\n", algo, M, N, K, totalNodes,
                        totalGPUs, dRow, dCol, stackSize, decompositionTime, executionTime, gatherTime, gflops,
                        dataLocation, communicationTime, gemmCallTime);
}

}  // namespace dgt

#endif
