// Host-only checks of include/dgt_logging.hpp against the reference's logging behaviour
// (src/Utilities/Logging.cpp:3-36, src/25DCannon.cpp:405-408, :443-446, :475-478):
// file names, header placement on new, matching and foreign files, the row format and
// calculateGflops.  argv[1] is an empty scratch directory; the files written there are
// read back by tests/test_csv_log.py with pandas, as the thesis notebooks read them.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "dgt_logging.hpp"

static int fails = 0;

static void expect(bool ok, const char* what) {
    if (!ok) {
        std::printf("FAIL: %s\n", what);
        ++fails;
    }
}

static std::string slurp(const std::string& path) {
    std::ifstream in(path);
    std::stringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    const std::string header = dgt::cannonLogHeader();

    expect(dgt::cannonLogFileName(true, "b200", "dgt") ==
               "DGEMM_execution_logs-PreDistributed_GEMM-b200-2.5DCANNON-dgt.csv",
           "pre-distributed file name");
    expect(dgt::cannonLogFileName(false, "meluxina", "cuBLAS") ==
               "DGEMM_execution_logs-FullOffload_GEMM-meluxina-2.5DCANNON-cuBLAS.csv",
           "full-offload file name (the reference's own)");

    // row format: "%s,%lld,%lld,%lld,%d,%d,%d,%d,%d,%lf,%lf,%lf,%lf,%s,%lf,%lf\n"
    const double g = dgt::calculateGflops(8192, 8192, 8192, 0.03125);
    expect(g == (2LL * 8192 * 8192 * 8192 * 1e-9) / 0.03125, "calculateGflops");
    const std::string row = dgt::cannonCsvLine("2.5D CANNON dgt", 8192, 8192, 8192, 1, 1, 4, 4, 2, 0.5, 0.03125,
                                               0.125, g, "devices", 0.0, 0.03125);
    expect(row == "2.5D CANNON dgt,8192,8192,8192,1,1,4,4,2,0.500000,0.031250,0.125000,35184.372089,devices,"
                  "0.000000,0.031250\n",
           "row format");

    // new file: header once; reopened: header skipped; rows appended after it
    const std::string a = dir + "/" + dgt::cannonLogFileName(true, "b200", "dgt");
    FILE* f = dgt::createLogCsv(a, header);
    expect(f != nullptr, "open new log");
    if (f) {
        dgt::writeLineToFile(f, row.c_str());
        std::fclose(f);
    }
    f = dgt::createLogCsv(a, header);
    expect(f != nullptr, "reopen log");
    if (f) {
        const std::string r2 = dgt::cannonCsvLine("2.5D CANNON dgt OzakiII-14moduli", 4096, 4096, 4096, 1, 1, 2, 2,
                                                  1, 0.25, 0.002, 0.01, dgt::calculateGflops(4096, 4096, 4096, 0.002),
                                                  "devices", 0.0, 0.002);
        dgt::writeLineToFile(f, r2.c_str());
        std::fclose(f);
    }
    const std::string body = slurp(a);
    expect(body.rfind(header + "\n", 0) == 0, "header first");
    expect(body.find(header, header.size()) == std::string::npos, "header written once");
    size_t lines = 0;
    for (char ch : body) lines += ch == '\n';
    expect(lines == 3, "header + 2 rows");

    // a file whose first line is some other header gets this header appended (the
    // reference compares only the first line)
    const std::string b = dir + "/foreign.csv";
    {
        std::ofstream out(b);
        out << "Algo,M,N,K\nx,1,2,3\n";
    }
    f = dgt::createLogCsv(b, header);
    expect(f != nullptr, "open foreign log");
    if (f) std::fclose(f);
    expect(slurp(b) == "Algo,M,N,K\nx,1,2,3\n" + header + "\n", "header appended after a foreign first line");

    // an unopenable path is reported, not fatal
    expect(dgt::createLogCsv(dir + "/no/such/dir/x.csv", header) == nullptr, "unopenable path -> nullptr");

    std::printf("%s\n", fails ? "FAILED" : "ALL OK");
    return fails ? 1 : 0;
}
