// ORACLE — test infrastructure only. Never linked into, or called by, the
// racon_b200 product path.
//
// CPU restatement of racon's polishing pipeline, following the reference
// sources line by line in semantics:
//   src/sequence.cpp:19-100  uppercase data, quality kept only when not all
//                            '!', reverse complement / reversed quality
//   src/overlap.cpp:15-108   MHAP / PAF / SAM overlap construction
//   src/overlap.cpp:129-177  transmute (name/id resolution, length checks)
//   src/overlap.cpp:179-292  alignment + breaking points
//   src/window.cpp:15-142    window layers and consensus
//   src/polisher.cpp:55-548  createPolisher checks, initialize, polish
// The third-party pieces are restated in edlib_nw.* and spoa_poa.*; the
// absent bioparser readers are restated here (FASTA/FASTQ multi-line,
// PAF/MHAP/SAM text, gzip or plain, names cut at the first whitespace).
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "spoa_poa.hpp"

namespace oracle {

struct CpuSequence {
    std::string name, data, rc, quality, rquality;
    void build_reverse();
};

struct CpuOverlap {
    std::string q_name, t_name;
    uint64_t q_id = 0, t_id = 0;
    uint32_t q_begin = 0, q_end = 0, q_length = 0;
    uint32_t t_begin = 0, t_end = 0, t_length = 0;
    uint32_t strand = 0, length = 0;
    double error = 0;
    std::string cigar;
    bool valid = true, transmuted = false;
    std::vector<std::pair<uint32_t, uint32_t>> breaking_points;
};

// Breaking points of one overlap from its CIGAR (src/overlap.cpp:226-292).
void breakpoints_from_cigar(const CpuOverlap& o, uint32_t window_length,
                            std::vector<std::pair<uint32_t, uint32_t>>& out);

struct CpuWindowInput {
    const char* backbone;
    uint32_t backbone_len;
    const char* backbone_qual;  // never null: dummy '!' when the target has none
    std::vector<const char*> seqs;
    std::vector<const char*> quals;  // entries may be null
    std::vector<uint32_t> lens;
    std::vector<std::pair<uint32_t, uint32_t>> positions;
};

struct WindowStats {
    uint64_t cells = 0, edge_cells = 0;
    uint32_t nodes = 0, edges = 0, layers = 0;
};

// Window::generate_consensus (src/window.cpp:65-142). Returns true when the
// window had at least two layers (polished).
bool window_consensus(const CpuWindowInput& w, bool tgs, bool trim, int match,
                      int mismatch, int gap, std::string& consensus,
                      WindowStats* stats, uint64_t window_id = 0, uint32_t rank = 0);

struct PolishOptions {
    bool fragment = false;  // -f
    uint32_t window_length = 500;
    double quality_threshold = 10.0;
    double error_threshold = 0.3;
    bool trim = true;
    int match = 3, mismatch = -5, gap = -4;
    uint32_t threads = 1;
    bool drop_unpolished = true;  // false with -u
};

struct PolishTimes {
    double load_s = 0, align_s = 0, layers_s = 0, consensus_s = 0;
    uint64_t overlaps = 0, windows = 0, poa_cells = 0;
};

// Runs initialize + polish; returns 0 on success, prints racon's message and
// returns 1 where racon would exit(1).
int polish_files(const std::string& sequences, const std::string& overlaps,
                 const std::string& targets, const PolishOptions& opt,
                 std::vector<std::pair<std::string, std::string>>& out,
                 PolishTimes* times);

// Window-level dump: every window's backbone, layers and consensus, after the
// same initialize() steps (used to build per-window test fixtures).
struct DumpedWindow {
    uint64_t target_id;
    uint32_t rank;
    bool tgs;
    std::string backbone, backbone_qual;
    std::vector<std::string> seqs, quals;  // empty qual = none
    std::vector<std::pair<uint32_t, uint32_t>> positions;
};
int collect_windows(const std::string& sequences, const std::string& overlaps,
                    const std::string& targets, const PolishOptions& opt,
                    std::vector<DumpedWindow>& windows);

// initialize() up to and including the breaking points: the sequence table
// (targets first), the target count, racon's window type and the kept
// overlaps with their breaking points, in racon's order.
int collect_layer_input(const std::string& sequences, const std::string& overlaps,
                        const std::string& targets, const PolishOptions& opt,
                        std::vector<CpuSequence>& seqs, uint64_t& n_targets, bool& tgs,
                        std::vector<CpuOverlap>& overlaps_out);

// Reads every record of a FASTA/FASTQ file (gzip or plain).
bool read_sequences(const std::string& path, std::vector<CpuSequence>& out);

}  // namespace oracle
