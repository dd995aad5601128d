// ORACLE — test infrastructure only. Never linked into, or called by, the
// racon_b200 product path.
//
// CPU restatement of the partial-order-alignment library racon calls per
// window (src/window.cpp:65-142, engine built at src/polisher.cpp:181-185):
//   spoa::createAlignmentEngine(kNW, match, mismatch, gap)  (linear gaps)
//   spoa::createGraph(); Graph::add_alignment(aln, seq, len[, qual, qlen]);
//   Graph::subgraph(begin, end, mapping); Graph::update_alignment(aln, mapping);
//   Graph::generate_consensus(coverages)
// spoa (github.com/rvaser/spoa, 3.x API; pin unrecoverable) is absent from the
// reference tree. This restates the published algorithm (Lee, Grasso &
// Sharlow 2002, partial order alignment with heaviest-bundle consensus) with
// spoa 3.x's observable conventions: node/edge insertion order, DFS
// topological order with aligned-node groups kept adjacent, NW end cell = first
// sink in rank order with the best last-column score, traceback preferring the
// diagonal (predecessors in in-edge order), then vertical, then horizontal,
// edge weight = sum of both endpoint base weights, coverage = distinct
// sequence labels on a node's edges.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace oracle {

// (node id or -1, sequence position or -1) pairs, in path order.
using PoaAlignment = std::vector<std::pair<int32_t, int32_t>>;

class PoaGraph {
public:
    struct Edge {
        uint32_t begin, end;
        std::vector<uint32_t> labels;
        int64_t weight;
    };
    struct Node {
        uint32_t code;
        std::vector<uint32_t> in_edges;   // indices into edges_
        std::vector<uint32_t> out_edges;  // indices into edges_
        std::vector<uint32_t> aligned;    // aligned node ids
    };

    PoaGraph();

    void add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                       const std::vector<uint32_t>& weights);
    void add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                       uint32_t weight = 1);
    void add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                       const char* qual, uint32_t qual_len);

    std::unique_ptr<PoaGraph> subgraph(uint32_t begin_node, uint32_t end_node,
                                       std::vector<int32_t>& sub_to_graph) const;
    static void update_alignment(PoaAlignment& aln,
                                 const std::vector<int32_t>& sub_to_graph);

    std::string generate_consensus(std::vector<uint32_t>& coverages);

    const std::vector<Node>& nodes() const { return nodes_; }
    const std::vector<Edge>& edges() const { return edges_; }
    const std::vector<uint32_t>& rank_to_node() const { return rank_to_node_; }
    int32_t decoder(uint32_t code) const { return decoder_[code]; }

private:
    uint32_t add_node(uint32_t code);
    void add_edge(uint32_t begin, uint32_t end, int64_t weight);
    int32_t add_sequence(const char* seq, const std::vector<uint32_t>& w,
                         uint32_t begin, uint32_t end);
    void topological_sort();
    void traverse_heaviest_bundle();
    uint32_t branch_completion(std::vector<int64_t>& scores,
                               std::vector<int32_t>& pred, uint32_t rank);
    uint32_t coverage(uint32_t node) const;

    uint32_t num_sequences_ = 0;
    uint32_t num_codes_ = 0;
    std::vector<int32_t> coder_, decoder_;
    std::vector<Node> nodes_;
    std::vector<Edge> edges_;
    std::vector<uint32_t> rank_to_node_;
    std::vector<uint32_t> consensus_;
};

// Per-alignment DP statistics, used to count algorithmic work (cells).
struct PoaStats {
    uint64_t cells = 0;       // sum of |sequence| x |nodes aligned against|
    uint64_t edge_cells = 0;  // sum of |sequence| x sum_v (1 + indeg v)
};

// Linear-gap global alignment of seq to the graph.
PoaAlignment poa_align_nw(const char* seq, uint32_t len, const PoaGraph& g,
                          int match, int mismatch, int gap, PoaStats* stats);

}  // namespace oracle
