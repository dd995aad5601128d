// ORACLE — test infrastructure only. Command-line front end of the CPU
// restatement with racon's flags (src/main.cpp:23-44, defaults :51-67):
//   racon_oracle [-u] [-f] [-w N] [-q F] [-e F] [--no-trimming] [-m N] [-x N]
//                [-g N] [-t N] <sequences> <overlaps> <targets>
// Prints the polished FASTA on stdout like src/main.cpp:164-166, and stage
// times on stderr.
#include <getopt.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "racon_cpu.hpp"

int main(int argc, char** argv) {
    static struct option options[] = {
        {"include-unpolished", no_argument, 0, 'u'},
        {"fragment-correction", no_argument, 0, 'f'},
        {"window-length", required_argument, 0, 'w'},
        {"quality-threshold", required_argument, 0, 'q'},
        {"error-threshold", required_argument, 0, 'e'},
        {"no-trimming", no_argument, 0, 'T'},
        {"match", required_argument, 0, 'm'},
        {"mismatch", required_argument, 0, 'x'},
        {"gap", required_argument, 0, 'g'},
        {"threads", required_argument, 0, 't'},
        {0, 0, 0, 0}};
    oracle::PolishOptions opt;
    int a;
    while ((a = getopt_long(argc, argv, "ufw:q:e:m:x:g:t:", options, nullptr)) != -1) {
        switch (a) {
            case 'u': opt.drop_unpolished = false; break;
            case 'f': opt.fragment = true; break;
            case 'w': opt.window_length = uint32_t(atoi(optarg)); break;
            case 'q': opt.quality_threshold = atof(optarg); break;
            case 'e': opt.error_threshold = atof(optarg); break;
            case 'T': opt.trim = false; break;
            case 'm': opt.match = int8_t(atoi(optarg)); break;
            case 'x': opt.mismatch = int8_t(atoi(optarg)); break;
            case 'g': opt.gap = int8_t(atoi(optarg)); break;
            case 't': opt.threads = uint32_t(atoi(optarg)); break;
            default: return 1;
        }
    }
    if (argc - optind < 3) {
        fprintf(stderr, "[racon::] error: missing input file(s)!\n");
        return 1;
    }
    std::vector<std::pair<std::string, std::string>> out;
    oracle::PolishTimes tm;
    const auto t0 = std::chrono::steady_clock::now();
    if (oracle::polish_files(argv[optind], argv[optind + 1], argv[optind + 2], opt, out, &tm))
        return 1;
    const double wall =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (const auto& s : out) fprintf(stdout, ">%s\n%s\n", s.first.c_str(), s.second.c_str());
    fprintf(stderr,
            "[oracle] load %.3f s, align %.3f s (%lu overlaps), layers %.3f s, consensus %.3f s "
            "(%lu windows, %lu cells), wall %.3f s, threads %u\n",
            tm.load_s, tm.align_s, (unsigned long)tm.overlaps, tm.layers_s, tm.consensus_s,
            (unsigned long)tm.windows, (unsigned long)tm.poa_cells, wall, opt.threads);
    return 0;
}
