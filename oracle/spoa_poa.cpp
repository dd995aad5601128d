// ORACLE — test infrastructure only (see spoa_poa.hpp).
#include "spoa_poa.hpp"

#include <algorithm>
#include <limits>
#include <stack>
#include <stdexcept>
#include <unordered_set>

namespace oracle {

PoaGraph::PoaGraph() : coder_(256, -1), decoder_(256, -1) {}

uint32_t PoaGraph::add_node(uint32_t code) {
    nodes_.push_back(Node{code, {}, {}, {}});
    return uint32_t(nodes_.size() - 1);
}

void PoaGraph::add_edge(uint32_t begin, uint32_t end, int64_t weight) {
    for (uint32_t e : nodes_[begin].out_edges) {
        if (edges_[e].end == end) {
            edges_[e].labels.push_back(num_sequences_);
            edges_[e].weight += weight;
            return;
        }
    }
    edges_.push_back(Edge{begin, end, {num_sequences_}, weight});
    const uint32_t e = uint32_t(edges_.size() - 1);
    nodes_[begin].out_edges.push_back(e);
    nodes_[end].in_edges.push_back(e);
}

int32_t PoaGraph::add_sequence(const char* seq, const std::vector<uint32_t>& w,
                               uint32_t begin, uint32_t end) {
    if (begin == end) return -1;
    const int32_t first = int32_t(add_node(uint32_t(coder_[uint8_t(seq[begin])])));
    for (uint32_t i = begin + 1; i < end; ++i) {
        const uint32_t id = add_node(uint32_t(coder_[uint8_t(seq[i])]));
        add_edge(id - 1, id, int64_t(w[i - 1]) + int64_t(w[i]));
    }
    return first;
}

void PoaGraph::add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                             uint32_t weight) {
    add_alignment(aln, seq, len, std::vector<uint32_t>(len, weight));
}

void PoaGraph::add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                             const char* qual, uint32_t qual_len) {
    if (len != qual_len) throw std::invalid_argument("quality length mismatch");
    std::vector<uint32_t> w(qual_len);
    for (uint32_t i = 0; i < qual_len; ++i) w[i] = uint32_t(qual[i] - 33);
    add_alignment(aln, seq, len, w);
}

void PoaGraph::add_alignment(const PoaAlignment& aln, const char* seq, uint32_t len,
                             const std::vector<uint32_t>& w) {
    if (len == 0) return;
    if (len != w.size()) throw std::invalid_argument("weights length mismatch");
    for (uint32_t i = 0; i < len; ++i) {
        const uint8_t c = uint8_t(seq[i]);
        if (coder_[c] == -1) {
            coder_[c] = int32_t(num_codes_);
            decoder_[num_codes_] = c;
            ++num_codes_;
        }
    }
    if (aln.empty()) {
        add_sequence(seq, w, 0, len);
        ++num_sequences_;
        topological_sort();
        return;
    }
    std::vector<uint32_t> valid;
    for (const auto& a : aln)
        if (a.second != -1) valid.push_back(uint32_t(a.second));

    const size_t before = nodes_.size();
    int32_t begin_id = add_sequence(seq, w, 0, valid.front());
    int32_t head = before == nodes_.size() ? -1 : int32_t(nodes_.size() - 1);
    const int32_t tail = add_sequence(seq, w, valid.back() + 1, len);

    int64_t prev_w = head == -1 ? 0 : w[valid.front() - 1];
    for (const auto& a : aln) {
        if (a.second == -1) continue;
        const uint8_t letter = uint8_t(seq[a.second]);
        int32_t nid;
        if (a.first == -1) {
            nid = int32_t(add_node(uint32_t(coder_[letter])));
        } else {
            const uint32_t at = uint32_t(a.first);
            if (decoder_[nodes_[at].code] == letter) {
                nid = int32_t(at);
            } else {
                int32_t hit = -1;
                for (uint32_t x : nodes_[at].aligned) {
                    if (decoder_[nodes_[x].code] == letter) {
                        hit = int32_t(x);
                        break;
                    }
                }
                if (hit == -1) {
                    nid = int32_t(add_node(uint32_t(coder_[letter])));
                    const std::vector<uint32_t> group = nodes_[at].aligned;
                    for (uint32_t x : group) {
                        nodes_[uint32_t(nid)].aligned.push_back(x);
                        nodes_[x].aligned.push_back(uint32_t(nid));
                    }
                    nodes_[uint32_t(nid)].aligned.push_back(at);
                    nodes_[at].aligned.push_back(uint32_t(nid));
                } else {
                    nid = hit;
                }
            }
        }
        if (begin_id == -1) begin_id = nid;
        if (head != -1) add_edge(uint32_t(head), uint32_t(nid), prev_w + w[a.second]);
        head = nid;
        prev_w = w[a.second];
    }
    if (tail != -1) add_edge(uint32_t(head), uint32_t(tail), prev_w + w[valid.back() + 1]);
    ++num_sequences_;
    topological_sort();
}

void PoaGraph::topological_sort() {
    rank_to_node_.clear();
    const size_t n = nodes_.size();
    std::vector<uint8_t> mark(n, 0);  // 0 new, 1 on stack, 2 done
    std::vector<bool> primary(n, true);
    std::stack<uint32_t> st;
    for (uint32_t i = 0; i < n; ++i) {
        if (mark[i] != 0) continue;
        st.push(i);
        while (!st.empty()) {
            const uint32_t v = st.top();
            bool ready = true;
            if (mark[v] != 2) {
                for (uint32_t e : nodes_[v].in_edges) {
                    const uint32_t u = edges_[e].begin;
                    if (mark[u] != 2) {
                        st.push(u);
                        ready = false;
                    }
                }
                if (primary[v]) {
                    for (uint32_t x : nodes_[v].aligned) {
                        if (mark[x] != 2) {
                            st.push(x);
                            primary[x] = false;
                            ready = false;
                        }
                    }
                }
                if (ready) {
                    mark[v] = 2;
                    if (primary[v]) {
                        rank_to_node_.push_back(v);
                        for (uint32_t x : nodes_[v].aligned) rank_to_node_.push_back(x);
                    }
                } else {
                    mark[v] = 1;
                }
            }
            if (ready) st.pop();
        }
    }
}

std::unique_ptr<PoaGraph> PoaGraph::subgraph(uint32_t begin_node, uint32_t end_node,
                                             std::vector<int32_t>& sub_to_graph) const {
    // nodes reachable backwards (in-edges and aligned groups) from end_node
    // whose id is not below begin_node
    std::vector<bool> keep(nodes_.size(), false);
    std::stack<uint32_t> st;
    st.push(end_node);
    while (!st.empty()) {
        const uint32_t v = st.top();
        st.pop();
        if (!keep[v] && v >= begin_node) {
            for (uint32_t e : nodes_[v].in_edges) st.push(edges_[e].begin);
            for (uint32_t x : nodes_[v].aligned) st.push(x);
            keep[v] = true;
        }
    }
    auto sub = std::unique_ptr<PoaGraph>(new PoaGraph());
    sub->num_sequences_ = num_sequences_;
    sub->num_codes_ = num_codes_;
    sub->coder_ = coder_;
    sub->decoder_ = decoder_;
    sub_to_graph.resize(nodes_.size(), -1);
    std::vector<int32_t> graph_to_sub(nodes_.size(), -1);
    for (uint32_t i = 0; i < keep.size(); ++i) {
        if (!keep[i]) continue;
        const uint32_t s = sub->add_node(nodes_[i].code);
        graph_to_sub[i] = int32_t(s);
        sub_to_graph[s] = int32_t(i);
    }
    for (uint32_t i = 0; i < keep.size(); ++i) {
        if (!keep[i]) continue;
        const uint32_t s = uint32_t(graph_to_sub[i]);
        for (uint32_t e : nodes_[i].in_edges) {
            const int32_t b = graph_to_sub[edges_[e].begin];
            if (b == -1) continue;
            sub->add_edge(uint32_t(b), s, edges_[e].weight);
        }
        for (uint32_t x : nodes_[i].aligned) {
            if (graph_to_sub[x] == -1) continue;
            sub->nodes_[s].aligned.push_back(uint32_t(graph_to_sub[x]));
        }
    }
    sub->topological_sort();
    return sub;
}

void PoaGraph::update_alignment(PoaAlignment& aln, const std::vector<int32_t>& map) {
    for (auto& a : aln)
        if (a.first != -1) a.first = map[uint32_t(a.first)];
}

uint32_t PoaGraph::coverage(uint32_t v) const {
    std::unordered_set<uint32_t> labels;
    for (uint32_t e : nodes_[v].in_edges)
        for (uint32_t l : edges_[e].labels) labels.insert(l);
    for (uint32_t e : nodes_[v].out_edges)
        for (uint32_t l : edges_[e].labels) labels.insert(l);
    return uint32_t(labels.size());
}

uint32_t PoaGraph::branch_completion(std::vector<int64_t>& scores,
                                     std::vector<int32_t>& pred, uint32_t rank) {
    const uint32_t v0 = rank_to_node_[rank];
    for (uint32_t e : nodes_[v0].out_edges) {
        for (uint32_t oe : nodes_[edges_[e].end].in_edges) {
            if (edges_[oe].begin != v0) scores[edges_[oe].begin] = -1;
        }
    }
    int64_t best = 0;
    uint32_t best_id = 0;
    for (uint32_t r = rank + 1; r < rank_to_node_.size(); ++r) {
        const uint32_t v = rank_to_node_[r];
        scores[v] = -1;
        pred[v] = -1;
        for (uint32_t e : nodes_[v].in_edges) {
            const uint32_t u = edges_[e].begin;
            if (scores[u] == -1) continue;
            const int64_t w = edges_[e].weight;
            if (scores[v] < w || (scores[v] == w && scores[uint32_t(pred[v])] <= scores[u])) {
                scores[v] = w;
                pred[v] = int32_t(u);
            }
        }
        if (pred[v] != -1) scores[v] += scores[uint32_t(pred[v])];
        if (best < scores[v]) {
            best = scores[v];
            best_id = v;
        }
    }
    return best_id;
}

void PoaGraph::traverse_heaviest_bundle() {
    const size_t n = nodes_.size();
    std::vector<int32_t> pred(n, -1);
    std::vector<int64_t> scores(n, -1);
    uint32_t best_id = 0;
    for (uint32_t v : rank_to_node_) {
        for (uint32_t e : nodes_[v].in_edges) {
            const uint32_t u = edges_[e].begin;
            const int64_t w = edges_[e].weight;
            if (scores[v] < w || (scores[v] == w && scores[uint32_t(pred[v])] <= scores[u])) {
                scores[v] = w;
                pred[v] = int32_t(u);
            }
        }
        if (pred[v] != -1) scores[v] += scores[uint32_t(pred[v])];
        if (scores[best_id] < scores[v]) best_id = v;
    }
    if (!nodes_[best_id].out_edges.empty()) {
        std::vector<uint32_t> node_to_rank(n, 0);
        for (uint32_t r = 0; r < n; ++r) node_to_rank[rank_to_node_[r]] = r;
        while (!nodes_[best_id].out_edges.empty())
            best_id = branch_completion(scores, pred, node_to_rank[best_id]);
    }
    consensus_.clear();
    while (pred[best_id] != -1) {
        consensus_.push_back(best_id);
        best_id = uint32_t(pred[best_id]);
    }
    consensus_.push_back(best_id);
    std::reverse(consensus_.begin(), consensus_.end());
}

std::string PoaGraph::generate_consensus(std::vector<uint32_t>& coverages) {
    traverse_heaviest_bundle();
    std::string out;
    coverages.clear();
    for (uint32_t v : consensus_) {
        out += char(decoder_[nodes_[v].code]);
        uint32_t cov = coverage(v);
        for (uint32_t x : nodes_[v].aligned) cov += coverage(x);
        coverages.push_back(cov);
    }
    return out;
}

__attribute__((target_clones("avx2", "default")))
PoaAlignment poa_align_nw(const char* seq, uint32_t len, const PoaGraph& g,
                          int match, int mismatch, int gap, PoaStats* stats) {
    const auto& nodes = g.nodes();
    const auto& edges = g.edges();
    if (nodes.empty() || len == 0) return PoaAlignment();
    const auto& r2n = g.rank_to_node();
    const uint32_t V = uint32_t(nodes.size());
    const uint32_t W = len + 1;  // column 0 = empty sequence prefix
    std::vector<uint32_t> n2r(V);
    for (uint32_t r = 0; r < V; ++r) n2r[r2n[r]] = r;
    if (stats) {
        stats->cells += uint64_t(len) * V;
        uint64_t deg = 0;
        for (const auto& nd : nodes) deg += 1 + nd.in_edges.size();
        stats->edge_cells += uint64_t(len) * deg;
    }
    auto pred_row = [&](uint32_t v, size_t p) -> uint32_t {
        return n2r[edges[nodes[v].in_edges[p]].begin] + 1;
    };
    std::vector<int32_t> H(size_t(V + 1) * W);
    H[0] = 0;
    for (uint32_t j = 1; j < W; ++j) H[j] = H[j - 1] + gap;
    for (uint32_t i = 1; i <= V; ++i) {
        const uint32_t v = r2n[i - 1];
        int32_t best = 0;
        if (!nodes[v].in_edges.empty()) {
            best = std::numeric_limits<int32_t>::min();
            for (size_t p = 0; p < nodes[v].in_edges.size(); ++p)
                best = std::max(best, H[size_t(pred_row(v, p)) * W]);
        }
        H[size_t(i) * W] = best + gap;
    }
    std::vector<int32_t> prof(W);
    int32_t max_score = std::numeric_limits<int32_t>::min();
    uint32_t max_i = 0;
    for (uint32_t i = 1; i <= V; ++i) {
        const uint32_t v = r2n[i - 1];
        const int32_t c = g.decoder(nodes[v].code);
        for (uint32_t j = 1; j < W; ++j) prof[j] = (uint8_t(seq[j - 1]) == c) ? match : mismatch;
        int32_t* row = &H[size_t(i) * W];
        const size_t np = nodes[v].in_edges.size();
        const int32_t* pr = &H[size_t(np ? pred_row(v, 0) : 0) * W];
        for (uint32_t j = 1; j < W; ++j) row[j] = std::max(pr[j - 1] + prof[j], pr[j] + gap);
        for (size_t p = 1; p < np; ++p) {
            pr = &H[size_t(pred_row(v, p)) * W];
            for (uint32_t j = 1; j < W; ++j)
                row[j] = std::max(pr[j - 1] + prof[j], std::max(row[j], pr[j] + gap));
        }
        for (uint32_t j = 1; j < W; ++j) row[j] = std::max(row[j - 1] + gap, row[j]);
        if (nodes[v].out_edges.empty() && max_score < row[W - 1]) {
            max_score = row[W - 1];
            max_i = i;
        }
    }
    // traceback from the best sink
    PoaAlignment aln;
    uint32_t i = max_i, j = W - 1;
    while (!(i == 0 && j == 0)) {
        const int32_t h = H[size_t(i) * W + j];
        bool found = false;
        uint32_t pi = 0, pj = 0;
        if (i != 0 && j != 0) {
            const uint32_t v = r2n[i - 1];
            const int32_t s = (uint8_t(seq[j - 1]) == g.decoder(nodes[v].code)) ? match : mismatch;
            const size_t np = nodes[v].in_edges.size();
            for (size_t p = 0; p < std::max<size_t>(np, 1); ++p) {
                const uint32_t r = np ? pred_row(v, p) : 0;
                if (h == H[size_t(r) * W + j - 1] + s) {
                    pi = r;
                    pj = j - 1;
                    found = true;
                    break;
                }
            }
        }
        if (!found && i != 0) {
            const uint32_t v = r2n[i - 1];
            const size_t np = nodes[v].in_edges.size();
            for (size_t p = 0; p < std::max<size_t>(np, 1); ++p) {
                const uint32_t r = np ? pred_row(v, p) : 0;
                if (h == H[size_t(r) * W + j] + gap) {
                    pi = r;
                    pj = j;
                    found = true;
                    break;
                }
            }
        }
        if (!found && j != 0 && h == H[size_t(i) * W + j - 1] + gap) {
            pi = i;
            pj = j - 1;
            found = true;
        }
        if (!found) throw std::runtime_error("poa traceback: no predecessor");
        aln.emplace_back(i == pi ? -1 : int32_t(r2n[i - 1]), j == pj ? -1 : int32_t(j - 1));
        i = pi;
        j = pj;
    }
    std::reverse(aln.begin(), aln.end());
    return aln;
}

}  // namespace oracle
