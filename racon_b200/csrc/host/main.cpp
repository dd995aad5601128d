// racon_b200 command line: racon's options (src/main.cpp:23-44, defaults
// :51-67) with the polishing hot path on the B200. The reference's CUDA
// options (-c/--cudapoa-batches, -b/--cuda-banded-alignment,
// --cudaaligner-batches, --cudaaligner-band-width) are accepted and ignored:
// this build always runs the device path.
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "racon.hpp"

namespace {

const char* kVersion = "v1.4.17-b200";
const int kAlignerBatches = 10000;
const int kAlignerBand = 10001;

void help() {
    printf(
        "usage: racon_b200 [options ...] <sequences> <overlaps> <target sequences>\n"
        "\n"
        "    #default output is stdout\n"
        "    <sequences>\n"
        "        input file in FASTA/FASTQ format (can be compressed with gzip)\n"
        "        containing sequences used for correction\n"
        "    <overlaps>\n"
        "        input file in MHAP/PAF/SAM format (can be compressed with gzip)\n"
        "        containing overlaps between sequences and target sequences\n"
        "    <target sequences>\n"
        "        input file in FASTA/FASTQ format (can be compressed with gzip)\n"
        "        containing sequences which will be corrected\n"
        "\n"
        "    options:\n"
        "        -u, --include-unpolished\n"
        "            output unpolished target sequences\n"
        "        -f, --fragment-correction\n"
        "            perform fragment correction instead of contig polishing\n"
        "            (overlaps file should contain dual/self overlaps!)\n"
        "        -w, --window-length <int>\n"
        "            default: 500\n"
        "            size of window on which POA is performed\n"
        "        -q, --quality-threshold <float>\n"
        "            default: 10.0\n"
        "            threshold for average base quality of windows used in POA\n"
        "        -e, --error-threshold <float>\n"
        "            default: 0.3\n"
        "            maximum allowed error rate used for filtering overlaps\n"
        "        --no-trimming\n"
        "            disables consensus trimming at window ends\n"
        "        -m, --match <int>\n"
        "            default: 3\n"
        "            score for matching bases\n"
        "        -x, --mismatch <int>\n"
        "            default: -5\n"
        "            score for mismatching bases\n"
        "        -g, --gap <int>\n"
        "            default: -4\n"
        "            gap penalty (must be negative)\n"
        "        -t, --threads <int>\n"
        "            default: 1\n"
        "            number of threads\n"
        "        --version\n"
        "            prints the version number\n"
        "        -h, --help\n"
        "            prints the usage\n"
        "        -c, --cudapoa-batches, -b, --cuda-banded-alignment,\n"
        "        --cudaaligner-batches <int>, --cudaaligner-band-width <int>\n"
        "            accepted for compatibility; the B200 path is always used\n"
        "            (device: RACON_B200_DEVICE, default 0)\n");
}

}  // namespace

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
        {"version", no_argument, 0, 'v'},
        {"help", no_argument, 0, 'h'},
        {"cudapoa-batches", optional_argument, 0, 'c'},
        {"cuda-banded-alignment", no_argument, 0, 'b'},
        {"cudaaligner-batches", required_argument, 0, kAlignerBatches},
        {"cudaaligner-band-width", required_argument, 0, kAlignerBand},
        {0, 0, 0, 0}};
    std::vector<std::string> paths;
    uint32_t window_length = 500;
    double quality_threshold = 10.0, error_threshold = 0.3;
    bool trim = true, drop = true;
    int8_t match = 3, mismatch = -5, gap = -4;
    uint32_t type = 0, threads = 1;
    int a;
    while ((a = getopt_long(argc, argv, "ufw:q:e:m:x:g:t:hbc::", options, nullptr)) != -1) {
        switch (a) {
            case 'u': drop = false; break;
            case 'f': type = 1; break;
            case 'w': window_length = uint32_t(atoi(optarg)); break;
            case 'q': quality_threshold = atof(optarg); break;
            case 'e': error_threshold = atof(optarg); break;
            case 'T': trim = false; break;
            case 'm': match = int8_t(atoi(optarg)); break;
            case 'x': mismatch = int8_t(atoi(optarg)); break;
            case 'g': gap = int8_t(atoi(optarg)); break;
            case 't': threads = uint32_t(atoi(optarg)); break;
            case 'v': printf("%s\n", kVersion); return 0;
            case 'h': help(); return 0;
            case 'c':
                if (optarg == nullptr && optind < argc && argv[optind] != nullptr && argv[optind][0] != '-') ++optind;
                break;
            case 'b':
            case kAlignerBatches:
            case kAlignerBand: break;
            default: return 1;
        }
    }
    for (int i = optind; i < argc; ++i) paths.emplace_back(argv[i]);
    if (paths.size() < 3) {
        fprintf(stderr, "[racon::] error: missing input file(s)!\n");
        help();
        return 1;
    }
    auto polisher = racon::createPolisher(paths[0], paths[1], paths[2],
                                          type == 0 ? racon::PolisherType::kC : racon::PolisherType::kF,
                                          window_length, quality_threshold, error_threshold, trim, match,
                                          mismatch, gap, threads);
    polisher->initialize();
    std::vector<std::unique_ptr<racon::Sequence>> out;
    polisher->polish(out, drop);
    for (const auto& s : out) fprintf(stdout, ">%s\n%s\n", s->name().c_str(), s->data().c_str());
    const double* st = polisher->stage_seconds();
    fprintf(stderr, "[racon_b200] load %.3f s, align %.3f s, layers %.3f s, consensus %.3f s\n", st[0], st[1],
            st[2], st[3]);
    return 0;
}
