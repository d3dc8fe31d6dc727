// Command-line view of include/dgt_logging.hpp for tests/test_csv_log.py, which compares
// its output with the CSV logs the reference's own driver writes:
//   csv_format name <pre|full> <machine> <impl>   log file name
//   csv_format header                             2.5D Cannon header
//   csv_format rows                               stdin: rows of that schema; stdout: each
//                                                 parsed and printed again by cannonCsvLine
//   csv_format open <path>                        createLogCsv(path, header), then close
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "dgt_logging.hpp"

static int rows() {
    std::string line;
    while (std::getline(std::cin, line)) {
        std::vector<std::string> f;
        std::stringstream ss(line);
        std::string x;
        while (std::getline(ss, x, ',')) f.push_back(x);
        if (f.size() != 16) return 1;
        auto ll = [&](int i) { return std::strtoll(f[i].c_str(), nullptr, 10); };
        auto in = [&](int i) { return int(std::strtol(f[i].c_str(), nullptr, 10)); };
        auto db = [&](int i) { return std::strtod(f[i].c_str(), nullptr); };
        std::fputs(dgt::cannonCsvLine(f[0].c_str(), ll(1), ll(2), ll(3), in(4), in(5), in(6), in(7), in(8), db(9),
                                      db(10), db(11), db(12), f[13].c_str(), db(14), db(15))
                       .c_str(),
                   stdout);
    }
    return 0;
}

int main(int argc, char** argv) {
    const std::string cmd = argc > 1 ? argv[1] : "";
    if (cmd == "name" && argc == 5) {
        std::printf("%s\n", dgt::cannonLogFileName(std::string(argv[2]) == "pre", argv[3], argv[4]).c_str());
        return 0;
    }
    if (cmd == "header") {
        std::printf("%s\n", dgt::cannonLogHeader());
        return 0;
    }
    if (cmd == "rows") return rows();
    if (cmd == "open" && argc == 3) {
        FILE* f = dgt::createLogCsv(argv[2], dgt::cannonLogHeader());
        if (!f) return 1;
        std::fclose(f);
        return 0;
    }
    return 2;
}
