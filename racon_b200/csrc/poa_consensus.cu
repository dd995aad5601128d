// Window consensus on the device with the semantics of racon's
//   src/window.cpp:65-142  Window::generate_consensus
// over spoa's partial-order graph (linear-gap NW, match/mismatch/gap from
// racon's -m/-x/-g, engine built at src/polisher.cpp:181-185).
//
// Design (B200, sm_100a). One CTA owns one window at a time; CTAs are
// persistent and pull windows from a size-sorted queue. Each CTA has a slot of
// global scratch holding the window's graph (node/edge arrays with ordered
// in/out/aligned lists), the DP matrix and the traceback decisions.
// * Graph maintenance (insertion of an aligned layer, the DFS topological order
//   with aligned groups kept adjacent, subgraph extraction, heaviest-bundle
//   consensus) is inherently sequential pointer work and runs on thread 0.
// * The DP of one layer against the (sub)graph runs on all threads, one row
//   (graph node in topological order) at a time: the diagonal and vertical
//   terms over the predecessors are independent per column, the in-row gap
//   term H[i][j] = max(T[j], H[i][j-1] + g) is a max-plus prefix scan done as
//   a per-thread segment scan followed by a block-wide scan of segment
//   carries. The traceback decision of every cell (first predecessor giving
//   the diagonal value, else first giving the vertical value, else
//   horizontal) is computed in the same pass, so the walk back reads one byte
//   per step.
// * The NW end cell is the first sink, in topological order, with the best
//   last-column score (block reduction with rank tie-break).
// Exact int32 arithmetic throughout; results are byte-identical to the CPU
// algorithm by construction.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <numeric>

#include "rb_internal.hpp"

namespace rb {
namespace {

constexpr int kPoaThreads = 128;
constexpr int kNegInf = -1000000000;
constexpr uint64_t kNoQual = ~0ull;

enum PoaFlag : uint8_t {
    kPolished = 1,
    kChimeric = 2,
    kOverflow = 4,
    kFailed = 8,
};

struct PoaWinDev {
    uint64_t bb_off;
    uint64_t bq_off;       // kNoQual: weight 0 ('!' dummy quality)
    uint64_t layer_base;   // first entry in the layer table (already in racon's sorted order)
    uint64_t out_off;
    uint32_t bb_len;
    uint32_t n_layers;
    uint32_t out_cap;
    uint32_t offset;       // uint32(0.01 * backbone length)
    uint32_t tgs;
    uint32_t pad;
};

struct PoaLayerDev {
    uint64_t seq_off;
    uint64_t qual_off;     // kNoQual: weight 1 per base
    uint32_t len, begin, end, pad;
};

struct PoaArgs {
    const uint8_t* in;
    const PoaWinDev* wins;
    const PoaLayerDev* layers;
    const uint32_t* order;
    uint32_t nwin;
    char* out;
    uint32_t* out_len;
    uint8_t* flags;
    uint8_t* scratch;
    size_t slot_bytes;
    int ncap, ecap, acap, lcap;  // node / edge / aligned-entry / DP-column capacities
    int match, mismatch, gap;
    int trim;
    unsigned int* counters;      // [0] window cursor, [1] status
    unsigned long long* cells;   // DP cells computed
};

// Per-slot scratch view.
struct Graph {
    uint8_t* code;
    uint32_t* cov;
    int *in_head, *in_tail, *out_head, *out_tail, *al_head, *al_tail;
    uint8_t *mark, *prim, *member, *sink;
    int *dprank, *rank_to_node, *dporder, *node_rank;
    int *e_src, *e_dst, *e_w, *e_next_in, *e_next_out;
    int *a_node, *a_next;
    int* stack;
    int *pred_off, *pred_idx;
    int *aln_node, *aln_pos;
    long long* bscore;
    int* bpred;
    int* cons;
    int* H;
    uint8_t* dec;
    int ncap, ecap, acap, scap, lcap, alncap;
};

__host__ __device__ size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct SlotLayout {
    size_t bytes;
};

template <class F>
__host__ __device__ size_t walk_layout(int ncap, int ecap, int acap, int lcap, F&& f) {
    size_t off = 0;
    auto take = [&](size_t bytes, int id) {
        f(id, off);
        off += align256(bytes);
    };
    const size_t N = size_t(ncap), E = size_t(ecap), A = size_t(acap), L = size_t(lcap);
    const size_t S = N + E + A + 16;
    take(N, 0);            // code
    take(N * 4, 1);        // cov
    take(N * 4, 2);        // in_head
    take(N * 4, 3);        // in_tail
    take(N * 4, 4);        // out_head
    take(N * 4, 5);        // out_tail
    take(N * 4, 6);        // al_head
    take(N * 4, 7);        // al_tail
    take(N, 8);            // mark
    take(N, 9);            // prim
    take(N, 10);           // member
    take(N, 11);           // sink
    take(N * 4, 12);       // dprank
    take(N * 4, 13);       // rank_to_node
    take(N * 4, 14);       // dporder
    take(N * 4, 15);       // node_rank
    take(E * 4, 16);       // e_src
    take(E * 4, 17);       // e_dst
    take(E * 4, 18);       // e_w
    take(E * 4, 19);       // e_next_in
    take(E * 4, 20);       // e_next_out
    take(A * 4, 21);       // a_node
    take(A * 4, 22);       // a_next
    take(S * 4, 23);       // stack
    take((N + 2) * 4, 24); // pred_off
    take((E + N + 2) * 4, 25);  // pred_idx
    take((N + L + 2) * 4, 26);  // aln_node
    take((N + L + 2) * 4, 27);  // aln_pos
    take(N * 8, 28);       // bscore
    take(N * 4, 29);       // bpred
    take(N * 4, 30);       // cons
    take((N + 1) * L * 4, 31);  // H
    take((N + 1) * L, 32);      // dec
    return off;
}

__device__ Graph make_graph(const PoaArgs& a, uint32_t slot) {
    uint8_t* base = a.scratch + size_t(slot) * a.slot_bytes;
    Graph g;
    void* p[33];
    walk_layout(a.ncap, a.ecap, a.acap, a.lcap, [&](int id, size_t off) { p[id] = base + off; });
    g.code = (uint8_t*)p[0];
    g.cov = (uint32_t*)p[1];
    g.in_head = (int*)p[2];
    g.in_tail = (int*)p[3];
    g.out_head = (int*)p[4];
    g.out_tail = (int*)p[5];
    g.al_head = (int*)p[6];
    g.al_tail = (int*)p[7];
    g.mark = (uint8_t*)p[8];
    g.prim = (uint8_t*)p[9];
    g.member = (uint8_t*)p[10];
    g.sink = (uint8_t*)p[11];
    g.dprank = (int*)p[12];
    g.rank_to_node = (int*)p[13];
    g.dporder = (int*)p[14];
    g.node_rank = (int*)p[15];
    g.e_src = (int*)p[16];
    g.e_dst = (int*)p[17];
    g.e_w = (int*)p[18];
    g.e_next_in = (int*)p[19];
    g.e_next_out = (int*)p[20];
    g.a_node = (int*)p[21];
    g.a_next = (int*)p[22];
    g.stack = (int*)p[23];
    g.pred_off = (int*)p[24];
    g.pred_idx = (int*)p[25];
    g.aln_node = (int*)p[26];
    g.aln_pos = (int*)p[27];
    g.bscore = (long long*)p[28];
    g.bpred = (int*)p[29];
    g.cons = (int*)p[30];
    g.H = (int*)p[31];
    g.dec = (uint8_t*)p[32];
    g.ncap = a.ncap;
    g.ecap = a.ecap;
    g.acap = a.acap;
    g.scap = a.ncap + a.ecap + a.acap + 16;
    g.lcap = a.lcap;
    g.alncap = a.ncap + a.lcap + 2;
    return g;
}

// Shared per-CTA state.
struct PoaShared {
    int nnodes, nedges, naligned, nseq;
    int nranks;   // entries of rank_to_node (full graph order)
    int ndp;      // rows of the current DP
    int fail;     // 0 ok, else PoaFlag
    int iend;     // DP rank of the NW end cell
    int naln;
    int best_val, best_rank;
    int scan_v[kPoaThreads / 32];
    int scan_l[kPoaThreads / 32];
    int red_v[kPoaThreads / 32];
    int red_r[kPoaThreads / 32];
};

// ---------------- graph primitives (thread 0) ----------------

__device__ int g_add_node(const Graph& g, PoaShared& sh, uint8_t c) {
    if (sh.nnodes >= g.ncap) {
        sh.fail = kOverflow;
        return -1;
    }
    const int id = sh.nnodes++;
    g.code[id] = c;
    g.cov[id] = 0;
    g.in_head[id] = g.in_tail[id] = -1;
    g.out_head[id] = g.out_tail[id] = -1;
    g.al_head[id] = g.al_tail[id] = -1;
    return id;
}

__device__ void g_add_edge(const Graph& g, PoaShared& sh, int b, int e, int w) {
    for (int x = g.out_head[b]; x != -1; x = g.e_next_out[x]) {
        if (g.e_dst[x] == e) {
            g.e_w[x] += w;
            return;
        }
    }
    if (sh.nedges >= g.ecap) {
        sh.fail = kOverflow;
        return;
    }
    const int id = sh.nedges++;
    g.e_src[id] = b;
    g.e_dst[id] = e;
    g.e_w[id] = w;
    g.e_next_in[id] = -1;
    g.e_next_out[id] = -1;
    if (g.out_tail[b] == -1) g.out_head[b] = id;
    else g.e_next_out[g.out_tail[b]] = id;
    g.out_tail[b] = id;
    if (g.in_tail[e] == -1) g.in_head[e] = id;
    else g.e_next_in[g.in_tail[e]] = id;
    g.in_tail[e] = id;
}

__device__ void g_add_aligned(const Graph& g, PoaShared& sh, int v, int x) {
    if (sh.naligned >= g.acap) {
        sh.fail = kOverflow;
        return;
    }
    const int id = sh.naligned++;
    g.a_node[id] = x;
    g.a_next[id] = -1;
    if (g.al_tail[v] == -1) g.al_head[v] = id;
    else g.a_next[g.al_tail[v]] = id;
    g.al_tail[v] = id;
}

// spoa's DFS topological order over the nodes with member flag set (all nodes
// when all_nodes). Writes the order to out; returns its length, -1 on overflow.
__device__ int g_topo_sort(const Graph& g, PoaShared& sh, bool all_nodes, int* out) {
    const int N = sh.nnodes;
    int nr = 0;
    int sp = 0;
    for (int i = 0; i < N; ++i) {
        if (!all_nodes && !g.member[i]) continue;
        if (g.mark[i] != 0) continue;
        g.stack[sp++] = i;
        while (sp > 0) {
            const int v = g.stack[sp - 1];
            bool valid = true;
            if (g.mark[v] != 2) {
                for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
                    const int u = g.e_src[e];
                    if (!all_nodes && !g.member[u]) continue;
                    if (g.mark[u] != 2) {
                        if (sp >= g.scap) return -1;
                        g.stack[sp++] = u;
                        valid = false;
                    }
                }
                if (g.prim[v]) {
                    for (int x = g.al_head[v]; x != -1; x = g.a_next[x]) {
                        const int y = g.a_node[x];
                        if (!all_nodes && !g.member[y]) continue;
                        if (g.mark[y] != 2) {
                            if (sp >= g.scap) return -1;
                            g.stack[sp++] = y;
                            g.prim[y] = 0;
                            valid = false;
                        }
                    }
                }
                if (valid) {
                    g.mark[v] = 2;
                    if (g.prim[v]) {
                        out[nr++] = v;
                        for (int x = g.al_head[v]; x != -1; x = g.a_next[x]) {
                            const int y = g.a_node[x];
                            if (!all_nodes && !g.member[y]) continue;
                            out[nr++] = y;
                        }
                    }
                } else {
                    g.mark[v] = 1;
                }
            }
            if (valid) --sp;
        }
    }
    return nr;
}

// Nodes reachable backwards (in-edges and aligned groups) from end_node whose
// id is not below begin_node (spoa's subgraph node set).
__device__ bool g_mark_subgraph(const Graph& g, PoaShared& sh, int begin_node, int end_node) {
    if (end_node < 0 || end_node >= sh.nnodes) {
        sh.fail = kFailed;
        return true;
    }
    int sp = 0;
    g.stack[sp++] = end_node;
    while (sp > 0) {
        const int v = g.stack[--sp];
        if (!g.member[v] && v >= begin_node) {
            for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
                if (sp >= g.scap) return false;
                g.stack[sp++] = g.e_src[e];
            }
            for (int x = g.al_head[v]; x != -1; x = g.a_next[x]) {
                if (sp >= g.scap) return false;
                g.stack[sp++] = g.a_node[x];
            }
            g.member[v] = 1;
        }
    }
    return true;
}

__device__ int layer_weight(const uint8_t* qual, int k) { return qual ? int(qual[k]) - 33 : 1; }

// Graph::add_alignment for one layer (alignment in g.aln_* reversed order,
// entries [0, naln) from the end of the path back to its start).
__device__ void g_add_alignment(const Graph& g, PoaShared& sh, const uint8_t* seq, const uint8_t* qual,
                                int len) {
    if (len == 0) return;
    const int naln = sh.naln;
    const bool count_cov = len >= 2;
    int first_pos = -1, last_pos = -1;
    for (int k = naln - 1; k >= 0; --k) {
        if (g.aln_pos[k] != -1) {
            if (first_pos == -1) first_pos = g.aln_pos[k];
            last_pos = g.aln_pos[k];
        }
    }
    if (first_pos == -1) {  // no sequence position aligned: cannot happen for NW
        sh.fail = kFailed;
        return;
    }
    // head part [0, first_pos), then tail part (last_pos, len)
    int head = -1, begin_id = -1;
    for (int k = 0; k < first_pos; ++k) {
        const int id = g_add_node(g, sh, seq[k]);
        if (id < 0) return;
        if (count_cov) g.cov[id] += 1;
        if (k > 0) g_add_edge(g, sh, id - 1, id, layer_weight(qual, k - 1) + layer_weight(qual, k));
        if (begin_id == -1) begin_id = id;
        head = id;
    }
    int tail = -1;
    for (int k = last_pos + 1; k < len; ++k) {
        const int id = g_add_node(g, sh, seq[k]);
        if (id < 0) return;
        if (count_cov) g.cov[id] += 1;
        if (k > last_pos + 1) g_add_edge(g, sh, id - 1, id, layer_weight(qual, k - 1) + layer_weight(qual, k));
        if (tail == -1) tail = id;
    }
    int prev_w = head == -1 ? 0 : layer_weight(qual, first_pos - 1);
    for (int k = naln - 1; k >= 0; --k) {
        const int pos = g.aln_pos[k];
        if (pos == -1) continue;
        const uint8_t letter = seq[pos];
        const int at = g.aln_node[k];
        int nid;
        if (at == -1) {
            nid = g_add_node(g, sh, letter);
        } else if (g.code[at] == letter) {
            nid = at;
        } else {
            int hit = -1;
            for (int x = g.al_head[at]; x != -1; x = g.a_next[x]) {
                if (g.code[g.a_node[x]] == letter) {
                    hit = g.a_node[x];
                    break;
                }
            }
            if (hit == -1) {
                nid = g_add_node(g, sh, letter);
                if (nid < 0) return;
                for (int x = g.al_head[at]; x != -1; x = g.a_next[x]) {
                    const int y = g.a_node[x];
                    g_add_aligned(g, sh, nid, y);
                    g_add_aligned(g, sh, y, nid);
                }
                g_add_aligned(g, sh, nid, at);
                g_add_aligned(g, sh, at, nid);
            } else {
                nid = hit;
            }
        }
        if (nid < 0 || sh.fail) return;
        if (count_cov) g.cov[nid] += 1;
        if (begin_id == -1) begin_id = nid;
        if (head != -1) g_add_edge(g, sh, head, nid, prev_w + layer_weight(qual, pos));
        head = nid;
        prev_w = layer_weight(qual, pos);
    }
    if (tail != -1) g_add_edge(g, sh, head, tail, prev_w + layer_weight(qual, last_pos + 1));
    sh.nseq += 1;
}

__device__ int g_branch_completion(const Graph& g, PoaShared& sh, int rank) {
    const int v0 = g.rank_to_node[rank];
    for (int e = g.out_head[v0]; e != -1; e = g.e_next_out[e]) {
        const int d = g.e_dst[e];
        for (int oe = g.in_head[d]; oe != -1; oe = g.e_next_in[oe]) {
            if (g.e_src[oe] != v0) g.bscore[g.e_src[oe]] = -1;
        }
    }
    long long best = 0;
    int best_id = 0;
    for (int r = rank + 1; r < sh.nranks; ++r) {
        const int v = g.rank_to_node[r];
        g.bscore[v] = -1;
        g.bpred[v] = -1;
        for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
            const int u = g.e_src[e];
            if (g.bscore[u] == -1) continue;
            const long long w = g.e_w[e];
            if (g.bscore[v] < w ||
                (g.bscore[v] == w && g.bpred[v] != -1 && g.bscore[g.bpred[v]] <= g.bscore[u])) {
                g.bscore[v] = w;
                g.bpred[v] = u;
            }
        }
        if (g.bpred[v] != -1) g.bscore[v] += g.bscore[g.bpred[v]];
        if (best < g.bscore[v]) {
            best = g.bscore[v];
            best_id = v;
        }
    }
    return best_id;
}

// Heaviest bundle over the full graph in rank order; writes the path to
// g.cons and returns its length (-1 on failure).
__device__ int g_heaviest_bundle(const Graph& g, PoaShared& sh) {
    const int N = sh.nnodes;
    int best_id = 0;
    for (int r = 0; r < sh.nranks; ++r) {
        const int v = g.rank_to_node[r];
        for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
            const int u = g.e_src[e];
            const long long w = g.e_w[e];
            if (g.bscore[v] < w ||
                (g.bscore[v] == w && g.bpred[v] != -1 && g.bscore[g.bpred[v]] <= g.bscore[u])) {
                g.bscore[v] = w;
                g.bpred[v] = u;
            }
        }
        if (g.bpred[v] != -1) g.bscore[v] += g.bscore[g.bpred[v]];
        if (g.bscore[best_id] < g.bscore[v]) best_id = v;
    }
    if (g.out_head[best_id] != -1) {
        for (int r = 0; r < sh.nranks; ++r) g.node_rank[g.rank_to_node[r]] = r;
        int guard = 0;
        while (g.out_head[best_id] != -1) {
            best_id = g_branch_completion(g, sh, g.node_rank[best_id]);
            if (++guard > N + 1) return -1;
        }
    }
    int len = 0;
    while (g.bpred[best_id] != -1) {
        g.cons[len++] = best_id;
        best_id = g.bpred[best_id];
        if (len > N) return -1;
    }
    g.cons[len++] = best_id;
    // reverse in place
    for (int i = 0, j = len - 1; i < j; ++i, --j) {
        const int t = g.cons[i];
        g.cons[i] = g.cons[j];
        g.cons[j] = t;
    }
    return len;
}

// ---------------- block helpers ----------------

// Inclusive block scan of max-plus segments: element = (value at segment
// end, segment length). Returns the exclusive carry (value at the position
// before this thread's segment, kNegInf for the first).
__device__ int block_carry_scan(PoaShared& sh, int v, int len, int gap) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // inclusive warp scan
    int sv = v, sl = len;
    for (int o = 1; o < 32; o <<= 1) {
        const int pv = __shfl_up_sync(0xffffffffu, sv, o);
        const int pl = __shfl_up_sync(0xffffffffu, sl, o);
        if (lane >= o) {
            const int cand = pv <= kNegInf / 2 ? kNegInf : pv + sl * gap;
            sv = max(sv, cand);
            sl = pl + sl;
        }
    }
    if (lane == 31) {
        sh.scan_v[wid] = sv;
        sh.scan_l[wid] = sl;
    }
    __syncthreads();
    // carry from previous warps
    int cv = kNegInf;
    for (int w = 0; w < wid; ++w) {
        const int wv = sh.scan_v[w], wl = sh.scan_l[w];
        cv = max(wv, cv <= kNegInf / 2 ? kNegInf : cv + wl * gap);
    }
    // inclusive value of this thread with warp-carry applied
    int incl = max(sv, cv <= kNegInf / 2 ? kNegInf : cv + sl * gap);
    // exclusive: shift by one lane
    int excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = cv;
    __syncthreads();
    return excl;
}

// ---------------- one window ----------------

__device__ void poa_window(const PoaArgs& a, const Graph& g, PoaShared& sh, uint32_t wi, int* s_seq_row) {
    const int tid = threadIdx.x;
    const PoaWinDev W = a.wins[wi];
    const uint8_t* bb = a.in + W.bb_off;
    const uint8_t* bq = W.bq_off == kNoQual ? nullptr : a.in + W.bq_off;
    uint8_t* outp = reinterpret_cast<uint8_t*>(a.out) + W.out_off;
    const int B = int(W.bb_len);
    if (W.n_layers < 2) {
        for (int i = tid; i < B; i += blockDim.x) outp[i] = bb[i];
        if (tid == 0) {
            a.out_len[wi] = uint32_t(B);
            a.flags[wi] = 0;
        }
        return;
    }
    if (B > g.ncap) {
        if (tid == 0) {
            a.flags[wi] = kOverflow;
            a.out_len[wi] = 0;
        }
        return;
    }
    // backbone: chain of B nodes, edge weights from quality (0 with the dummy)
    for (int i = tid; i < B; i += blockDim.x) {
        g.code[i] = bb[i];
        g.cov[i] = B >= 2 ? 1u : 0u;
        g.al_head[i] = g.al_tail[i] = -1;
        if (i == 0) {
            g.in_head[i] = g.in_tail[i] = -1;
        } else {
            const int e = i - 1;
            g.in_head[i] = g.in_tail[i] = e;
            const int w = (bq ? int(bq[i - 1]) - 33 : 0) + (bq ? int(bq[i]) - 33 : 0);
            g.e_src[e] = i - 1;
            g.e_dst[e] = i;
            g.e_w[e] = w;
            g.e_next_in[e] = -1;
            g.e_next_out[e] = -1;
        }
        if (i == B - 1) {
            g.out_head[i] = g.out_tail[i] = -1;
        } else {
            g.out_head[i] = g.out_tail[i] = i;
        }
        g.rank_to_node[i] = i;
    }
    if (tid == 0) {
        sh.nnodes = B;
        sh.nedges = B - 1;
        sh.naligned = 0;
        sh.nseq = 1;
        sh.nranks = B;
        sh.fail = 0;
    }
    __syncthreads();
    unsigned long long cells = 0;

    for (uint32_t li = 0; li < W.n_layers; ++li) {
        const PoaLayerDev Lr = a.layers[W.layer_base + li];
        const uint8_t* seq = a.in + Lr.seq_off;
        const uint8_t* qual = Lr.qual_off == kNoQual ? nullptr : a.in + Lr.qual_off;
        const int L = int(Lr.len);
        const int Wc = L + 1;
        const bool full = Lr.begin < W.offset && Lr.end > uint32_t(B) - W.offset;
        // ---- choose the node set and its topological order ----
        const int N = sh.nnodes;
        for (int i = tid; i < N; i += blockDim.x) {
            g.member[i] = full ? 1 : 0;
            g.mark[i] = 0;
            g.prim[i] = 1;
            g.dprank[i] = 0;
        }
        __syncthreads();
        if (!full) {
            if (tid == 0) {
                if (!g_mark_subgraph(g, sh, int(Lr.begin), int(Lr.end))) sh.fail = kOverflow;
                if (!sh.fail) {
                    const int nr = g_topo_sort(g, sh, false, g.dporder);
                    if (nr < 0) sh.fail = kOverflow;
                    sh.ndp = nr;
                }
            }
        } else if (tid == 0) {
            sh.ndp = sh.nranks;
        }
        __syncthreads();
        if (sh.fail) break;
        const int ndp = sh.ndp;
        const int* order = full ? g.rank_to_node : g.dporder;
        if (ndp + 1 > g.ncap + 1 || Wc > g.lcap) {
            if (tid == 0) sh.fail = kOverflow;
            __syncthreads();
            break;
        }
        for (int i = tid; i < ndp; i += blockDim.x) g.dprank[order[i]] = i + 1;
        // layer sequence into shared memory
        for (int j = tid; j < L; j += blockDim.x) s_seq_row[j] = seq[j];
        __syncthreads();
        // ---- predecessor lists (DP ranks, in in-edge order) and sinks ----
        for (int i = tid; i < ndp; i += blockDim.x) {
            const int v = order[i];
            int cnt = 0;
            for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e])
                if (g.dprank[g.e_src[e]] > 0) ++cnt;
            g.pred_off[i + 1] = cnt;
            bool sink = true;
            for (int e = g.out_head[v]; e != -1; e = g.e_next_out[e])
                if (g.dprank[g.e_dst[e]] > 0) {
                    sink = false;
                    break;
                }
            g.sink[i] = sink ? 1 : 0;
        }
        __syncthreads();
        if (tid == 0) {
            g.pred_off[0] = 0;
            for (int i = 1; i <= ndp; ++i) g.pred_off[i] += g.pred_off[i - 1];
        }
        __syncthreads();
        for (int i = tid; i < ndp; i += blockDim.x) {
            const int v = order[i];
            int k = g.pred_off[i];
            for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
                const int r = g.dprank[g.e_src[e]];
                if (r > 0) g.pred_idx[k++] = r;
            }
        }
        // ---- DP ----
        const int lc = g.lcap;
        for (int j = tid; j < Wc; j += blockDim.x) g.H[j] = j * a.gap;
        __syncthreads();
        const int seg = (Wc + blockDim.x - 1) / blockDim.x;
        const int j0 = min(Wc, tid * seg), j1 = min(Wc, j0 + seg);
        int* sT = s_seq_row + L + 1;  // per-row temporaries, Wc entries
        for (int i = 1; i <= ndp; ++i) {
            const int v = order[i - 1];
            const uint8_t cv = g.code[v];
            const int pb = g.pred_off[i - 1], pe = g.pred_off[i];
            const int np = pe - pb;
            int* Hi = g.H + size_t(i) * lc;
            // diagonal / vertical terms
            for (int j = j0; j < j1; ++j) {
                int t = kNegInf;
                if (np == 0) {
                    const int* Hp = g.H;
                    t = Hp[j] + a.gap;
                    if (j > 0) t = max(t, Hp[j - 1] + (s_seq_row[j - 1] == cv ? a.match : a.mismatch));
                } else {
                    for (int p = pb; p < pe; ++p) {
                        const int* Hp = g.H + size_t(g.pred_idx[p]) * lc;
                        t = max(t, Hp[j] + a.gap);
                        if (j > 0) t = max(t, Hp[j - 1] + (s_seq_row[j - 1] == cv ? a.match : a.mismatch));
                    }
                }
                sT[j] = t;
            }
            // segment prefix, then block carry
            int run = kNegInf;
            for (int j = j0; j < j1; ++j) {
                run = max(sT[j], run <= kNegInf / 2 ? kNegInf : run + a.gap);
                sT[j] = run;
            }
            const int carry = block_carry_scan(sh, run, j1 - j0, a.gap);
            uint8_t* Di = g.dec + size_t(i) * lc;
            for (int j = j0; j < j1; ++j) {
                const int cin = carry <= kNegInf / 2 ? kNegInf : carry + (j - j0 + 1) * a.gap;
                const int h = max(sT[j], cin);
                Hi[j] = h;
                // traceback decision in spoa's order
                uint8_t code = 128;
                const int s = j > 0 ? (s_seq_row[j - 1] == cv ? a.match : a.mismatch) : 0;
                bool found = false;
                const int cnt = np == 0 ? 1 : np;
                if (j > 0) {
                    for (int p = 0; p < cnt; ++p) {
                        const int r = np == 0 ? 0 : g.pred_idx[pb + p];
                        if (g.H[size_t(r) * lc + j - 1] + s == h) {
                            code = p < 64 ? uint8_t(p) : uint8_t(255);
                            found = true;
                            break;
                        }
                    }
                }
                if (!found) {
                    for (int p = 0; p < cnt; ++p) {
                        const int r = np == 0 ? 0 : g.pred_idx[pb + p];
                        if (g.H[size_t(r) * lc + j] + a.gap == h) {
                            code = p < 64 ? uint8_t(64 + p) : uint8_t(255);
                            found = true;
                            break;
                        }
                    }
                }
                Di[j] = code;
            }
            __syncthreads();
        }
        cells += (unsigned long long)ndp * (unsigned long long)L;
        // ---- NW end: first sink in order with the best last-column score ----
        int bv = kNegInf, br = INT_MAX;
        for (int i = tid; i < ndp; i += blockDim.x) {
            if (g.sink[i]) {
                const int val = g.H[size_t(i + 1) * lc + L];
                if (val > bv || (val == bv && i + 1 < br)) {
                    bv = val;
                    br = i + 1;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const int ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > bv || (ov == bv && orr < br)) {
                bv = ov;
                br = orr;
            }
        }
        if ((tid & 31) == 0) {
            sh.red_v[tid >> 5] = bv;
            sh.red_r[tid >> 5] = br;
        }
        __syncthreads();
        if (tid == 0) {
            int vv = kNegInf, rr = INT_MAX;
            for (int w = 0; w < int(blockDim.x >> 5); ++w) {
                if (sh.red_v[w] > vv || (sh.red_v[w] == vv && sh.red_r[w] < rr)) {
                    vv = sh.red_v[w];
                    rr = sh.red_r[w];
                }
            }
            sh.iend = rr;
            // ---- traceback ----
            int i = rr, j = L, n = 0;
            bool bad = rr == INT_MAX;
            while (!bad && !(i == 0 && j == 0)) {
                if (n >= g.alncap) {
                    bad = true;
                    break;
                }
                if (i == 0) {
                    g.aln_node[n] = -1;
                    g.aln_pos[n] = j - 1;
                    ++n;
                    --j;
                    continue;
                }
                uint8_t code = g.dec[size_t(i) * lc + j];
                const int pb = g.pred_off[i - 1], np = g.pred_off[i] - pb;
                const int v = order[i - 1];
                if (code == 255) {  // predecessor index >= 64: decide again from H
                    const int h = g.H[size_t(i) * lc + j];
                    const int s = j > 0 ? (seq[j - 1] == g.code[v] ? a.match : a.mismatch) : 0;
                    const int cnt = np == 0 ? 1 : np;
                    code = 128;
                    int pick = -1;
                    if (j > 0)
                        for (int p = 0; p < cnt && pick < 0; ++p) {
                            const int r = np == 0 ? 0 : g.pred_idx[pb + p];
                            if (g.H[size_t(r) * lc + j - 1] + s == h) pick = p;
                        }
                    if (pick >= 0) {
                        const int r = np == 0 ? 0 : g.pred_idx[pb + pick];
                        g.aln_node[n] = v;
                        g.aln_pos[n] = j - 1;
                        ++n;
                        i = r;
                        --j;
                        continue;
                    }
                    for (int p = 0; p < cnt && pick < 0; ++p) {
                        const int r = np == 0 ? 0 : g.pred_idx[pb + p];
                        if (g.H[size_t(r) * lc + j] + a.gap == h) pick = p;
                    }
                    if (pick >= 0) {
                        g.aln_node[n] = v;
                        g.aln_pos[n] = -1;
                        ++n;
                        i = np == 0 ? 0 : g.pred_idx[pb + pick];
                        continue;
                    }
                }
                if (code < 64) {
                    g.aln_node[n] = v;
                    g.aln_pos[n] = j - 1;
                    ++n;
                    i = np == 0 ? 0 : g.pred_idx[pb + code];
                    --j;
                } else if (code < 128) {
                    g.aln_node[n] = v;
                    g.aln_pos[n] = -1;
                    ++n;
                    i = np == 0 ? 0 : g.pred_idx[pb + (code - 64)];
                } else {
                    if (j == 0) {
                        bad = true;
                        break;
                    }
                    g.aln_node[n] = -1;
                    g.aln_pos[n] = j - 1;
                    ++n;
                    --j;
                }
            }
            sh.naln = n;
            if (bad) sh.fail = kFailed;
            // ---- insert the layer and re-sort ----
            if (!sh.fail) g_add_alignment(g, sh, seq, qual, L);
        }
        __syncthreads();
        if (sh.fail) break;
        const int N2 = sh.nnodes;
        for (int i = tid; i < N2; i += blockDim.x) {
            g.mark[i] = 0;
            g.prim[i] = 1;
        }
        __syncthreads();
        if (tid == 0) {
            const int nr = g_topo_sort(g, sh, true, g.rank_to_node);
            if (nr < 0) sh.fail = kOverflow;
            sh.nranks = nr;
        }
        __syncthreads();
        if (sh.fail) break;
    }
    if (tid == 0 && cells) atomicAdd(a.cells, cells);
    if (sh.fail) {
        if (tid == 0) {
            a.flags[wi] = uint8_t(sh.fail);
            a.out_len[wi] = 0;
        }
        return;
    }
    // ---- consensus ----
    const int N = sh.nnodes;
    for (int i = tid; i < N; i += blockDim.x) {
        g.bscore[i] = -1;
        g.bpred[i] = -1;
    }
    __syncthreads();
    if (tid == 0) {
        const int len = g_heaviest_bundle(g, sh);
        uint8_t flags = kPolished;
        if (len < 0) {
            flags = kFailed;
            a.out_len[wi] = 0;
        } else {
            // per-node coverage = own + aligned nodes' coverage
            int b = 0, e = len - 1;
            if (W.tgs && a.trim) {
                const uint32_t avg = W.n_layers / 2;
                auto cov_at = [&](int k) {
                    const int v = g.cons[k];
                    uint32_t c = g.cov[v];
                    for (int x = g.al_head[v]; x != -1; x = g.a_next[x]) c += g.cov[g.a_node[x]];
                    return c;
                };
                for (b = 0; b < len; ++b)
                    if (cov_at(b) >= avg) break;
                for (e = len - 1; e >= 0; --e)
                    if (cov_at(e) >= avg) break;
                if (b >= e) {
                    flags |= kChimeric;
                    b = 0;
                    e = len - 1;
                }
            }
            const int outl = e - b + 1;
            if (uint32_t(outl) > W.out_cap) {
                flags = kOverflow;
                a.out_len[wi] = 0;
            } else {
                for (int k = 0; k < outl; ++k) outp[k] = g.code[g.cons[b + k]];
                a.out_len[wi] = uint32_t(outl);
            }
        }
        a.flags[wi] = flags;
    }
}

__global__ void __launch_bounds__(kPoaThreads) poa_kernel(PoaArgs a) {
    __shared__ PoaShared sh;
    extern __shared__ int s_dyn[];
    const Graph g = make_graph(a, blockIdx.x);
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) sh.best_rank = int(atomicAdd(&a.counters[0], 1u));
        __syncthreads();
        const uint32_t k = uint32_t(sh.best_rank);
        if (k >= a.nwin) break;
        poa_window(a, g, sh, a.order[k], s_dyn);
    }
}

}  // namespace

PoaEngine::PoaEngine(const DeviceInfo& dev, cudaStream_t stream, int8_t m, int8_t x, int8_t g)
    : dev_(dev), stream_(stream), match_(m), mismatch_(x), gap_(g) {
    check_cuda(cudaEventCreate(&ev0_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev2_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev3_), "cudaEventCreate");
}

PoaEngine::~PoaEngine() {
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
    cudaEventDestroy(ev2_);
    cudaEventDestroy(ev3_);
}

void PoaEngine::stage(const rb_window* wins, size_t n, int trim) {
    if (n > 0 && !wins) throw Error{RB_ERR_ARG, "rb_poa: windows is NULL"};
    nwin_ = n;
    trim_ = trim;
    // sizes
    uint64_t in_bytes = 0, nlayers = 0, out_cap = 0;
    max_len_ = 0;
    uint32_t max_nodes = 0;
    for (size_t i = 0; i < n; ++i) {
        const rb_window& w = wins[i];
        if (!w.backbone || w.backbone_length == 0 || w.backbone_length > 65535)
            throw Error{RB_ERR_ARG, "rb_poa: backbone empty, NULL or longer than 65535"};
        if (w.n_layers > 65535) throw Error{RB_ERR_ARG, "rb_poa: more than 65535 layers"};
        if (w.n_layers && (!w.layers || !w.layer_lengths || !w.begins || !w.ends))
            throw Error{RB_ERR_ARG, "rb_poa: NULL layer arrays"};
        in_bytes += 2 * ((w.backbone_length + 15) & ~15u);
        uint64_t est = w.backbone_length;
        for (uint32_t j = 0; j < w.n_layers; ++j) {
            const uint32_t l = w.layer_lengths[j];
            if (l == 0 || l > 65535 || !w.layers[j])
                throw Error{RB_ERR_ARG, "rb_poa: empty, NULL or over-long layer"};
            // racon's layers end at a matched backbone base (end <= length - 1,
            // src/polisher.cpp:450-453); the subgraph of a partial layer is
            // rooted at backbone node `end`, so it must exist.
            if (w.begins[j] >= w.ends[j] || w.ends[j] >= w.backbone_length)
                throw Error{RB_ERR_ARG, "rb_poa: layer begin and end positions are invalid"};
            in_bytes += 2 * ((l + 15) & ~15u);
            max_len_ = std::max(max_len_, l);
            est += l;
        }
        nlayers += w.n_layers;
        out_cap += 3ull * w.backbone_length + 1024;
        max_nodes = uint32_t(std::max<uint64_t>(max_nodes, std::min<uint64_t>(est, 1u << 20)));
    }
    in_bytes_ = in_bytes;
    out_cap_ = out_cap;
    max_nodes_cap_ = max_nodes;
    h_in_.reserve(std::max<uint64_t>(in_bytes, 16));
    h_desc_.reserve(std::max<size_t>(n, 1) * sizeof(PoaWinDev));
    h_layers_.reserve(std::max<uint64_t>(nlayers, 1) * sizeof(PoaLayerDev));
    h_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    uint8_t* in = h_in_.as<uint8_t>();
    PoaWinDev* wd = h_desc_.as<PoaWinDev>();
    PoaLayerDev* ld = h_layers_.as<PoaLayerDev>();
    uint64_t off = 0, lbase = 0, oo = 0;
    labels_.resize(n);
    std::vector<uint32_t> rank;
    for (size_t i = 0; i < n; ++i) {
        const rb_window& w = wins[i];
        labels_[i] = {w.id, w.rank};
        PoaWinDev& d = wd[i];
        d.bb_off = off;
        memcpy(in + off, w.backbone, w.backbone_length);
        off += (w.backbone_length + 15) & ~15u;
        if (w.backbone_quality) {
            d.bq_off = off;
            memcpy(in + off, w.backbone_quality, w.backbone_length);
            off += (w.backbone_length + 15) & ~15u;
        } else {
            d.bq_off = kNoQual;
        }
        d.bb_len = w.backbone_length;
        d.n_layers = w.n_layers;
        d.layer_base = lbase;
        d.out_off = oo;
        d.out_cap = 3u * w.backbone_length + 1024;
        oo += d.out_cap;
        d.offset = uint32_t(0.01 * w.backbone_length);
        d.tgs = w.tgs ? 1u : 0u;
        d.pad = 0;
        // racon's layer order: std::sort by begin over entries 1.. (backbone at 0)
        // (src/window.cpp:78-85); the same call on the host keeps libstdc++'s
        // order for equal begins.
        rank.resize(size_t(w.n_layers) + 1);
        for (uint32_t j = 0; j <= w.n_layers; ++j) rank[j] = j;
        std::sort(rank.begin() + 1, rank.end(), [&](uint32_t lhs, uint32_t rhs) {
            const uint32_t a = lhs == 0 ? 0u : w.begins[lhs - 1];
            const uint32_t b = rhs == 0 ? 0u : w.begins[rhs - 1];
            return a < b;
        });
        for (uint32_t j = 1; j <= w.n_layers; ++j) {
            const uint32_t s = rank[j] - 1;
            PoaLayerDev& L = ld[lbase + j - 1];
            const uint32_t l = w.layer_lengths[s];
            L.seq_off = off;
            memcpy(in + off, w.layers[s], l);
            off += (l + 15) & ~15u;
            const char* q = w.layer_qualities ? w.layer_qualities[s] : nullptr;
            if (q) {
                L.qual_off = off;
                memcpy(in + off, q, l);
                off += (l + 15) & ~15u;
            } else {
                L.qual_off = kNoQual;
            }
            L.len = l;
            L.begin = w.begins[s];
            L.end = w.ends[s];
            L.pad = 0;
        }
        lbase += w.n_layers;
    }
    // size-sorted queue: most work first
    uint32_t* order = h_order_.as<uint32_t>();
    std::iota(order, order + n, 0u);
    std::vector<uint64_t> work(n);
    for (size_t i = 0; i < n; ++i) {
        uint64_t s = 0;
        for (uint32_t j = 0; j < wd[i].n_layers; ++j) s += ld[wd[i].layer_base + j].len;
        work[i] = s * (wd[i].bb_len + s / std::max<uint32_t>(1, wd[i].n_layers));
    }
    std::sort(order, order + n, [&](uint32_t x, uint32_t y) { return work[x] != work[y] ? work[x] > work[y] : x < y; });
    d_in_.reserve(std::max<uint64_t>(off, 16));
    d_desc_.reserve(std::max<size_t>(n, 1) * sizeof(PoaWinDev));
    d_layers_.reserve(std::max<uint64_t>(nlayers, 1) * sizeof(PoaLayerDev));
    d_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(d_in_.ptr, in, off, cudaMemcpyHostToDevice, stream_), "H2D windows");
    check_cuda(cudaMemcpyAsync(d_desc_.ptr, wd, n * sizeof(PoaWinDev), cudaMemcpyHostToDevice, stream_), "H2D desc");
    check_cuda(cudaMemcpyAsync(d_layers_.ptr, ld, nlayers * sizeof(PoaLayerDev), cudaMemcpyHostToDevice, stream_),
               "H2D layers");
    check_cuda(cudaMemcpyAsync(d_order_.ptr, order, n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_),
               "H2D order");
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "stage sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.h2d_ms = ms;
    stats_.h2d_bytes = off + n * (sizeof(PoaWinDev) + 4) + nlayers * sizeof(PoaLayerDev);
    in_bytes_ = off;
}

void PoaEngine::run() {
    const size_t n = nwin_;
    stats_.launches = 0;
    stats_.items = n;
    stats_.cells = 0;
    stats_.kernel_ms = 0;
    if (n == 0) return;
    d_out_.reserve(std::max<uint64_t>(out_cap_, 16));
    d_outlen_.reserve(n * 4);
    d_flags_.reserve(n);
    d_misc_.reserve(64);
    std::vector<uint32_t> todo(n);
    const uint32_t* h_order = h_order_.as<uint32_t>();
    for (size_t i = 0; i < n; ++i) todo[i] = h_order[i];
    int ncap = 4096;
    while (uint32_t(ncap) < std::min<uint32_t>(max_nodes_cap_, 6144)) ncap *= 2;
    std::vector<uint8_t> flags(n);
    float total_ms = 0;
    while (!todo.empty()) {
        const int ecap = 2 * ncap, acap = ncap;
        const int lcap = int((max_len_ + 1 + 3) & ~3u);
        const size_t slot = walk_layout(ncap, ecap, acap, lcap, [](int, size_t) {});
        const size_t budget = size_t(24) << 30;
        size_t slots = std::min<size_t>(todo.size(), size_t(dev_.sm_count) * 4);
        // RB_POA_SLOTS caps the resident windows (smaller scratch, e.g. for
        // profiler captures); results do not depend on it
        if (const char* e = getenv("RB_POA_SLOTS")) slots = std::max<size_t>(1, std::min<size_t>(slots, strtoull(e, nullptr, 10)));
        while (slots > 1 && slots * slot > budget) slots /= 2;
        d_graph_.reserve(slots * slot);
        d_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
        DevBuf& d_todo = d_dp_;
        d_todo.reserve(todo.size() * 4);
        check_cuda(cudaMemcpyAsync(d_todo.ptr, todo.data(), todo.size() * 4, cudaMemcpyHostToDevice, stream_),
                   "H2D todo");
        PoaArgs a;
        memset(&a, 0, sizeof(a));
        a.in = d_in_.as<uint8_t>();
        a.wins = d_desc_.as<PoaWinDev>();
        a.layers = d_layers_.as<PoaLayerDev>();
        a.order = d_todo.as<uint32_t>();
        a.nwin = uint32_t(todo.size());
        a.out = d_out_.as<char>();
        a.out_len = d_outlen_.as<uint32_t>();
        a.flags = d_flags_.as<uint8_t>();
        a.scratch = d_graph_.as<uint8_t>();
        a.slot_bytes = slot;
        a.ncap = ncap;
        a.ecap = ecap;
        a.acap = acap;
        a.lcap = lcap;
        a.match = match_;
        a.mismatch = mismatch_;
        a.gap = gap_;
        a.trim = trim_;
        a.counters = d_misc_.as<unsigned int>();
        a.cells = reinterpret_cast<unsigned long long*>(d_misc_.as<unsigned int>() + 8);
        const size_t smem = size_t(2 * lcap + 8) * sizeof(int);
        if (smem > 48 * 1024) {
            check_cuda(cudaFuncSetAttribute(poa_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                       "cudaFuncSetAttribute");
        }
        check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset counters");
        check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
        poa_kernel<<<int(slots), kPoaThreads, smem, stream_>>>(a);
        check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
        ++stats_.launches;
        unsigned long long cells = 0;
        check_cuda(cudaMemcpyAsync(&cells, a.cells, 8, cudaMemcpyDeviceToHost, stream_), "D2H cells");
        check_cuda(cudaMemcpyAsync(flags.data(), d_flags_.ptr, n, cudaMemcpyDeviceToHost, stream_), "D2H flags");
        check_cuda(cudaStreamSynchronize(stream_), "poa sync");
        check_cuda(cudaGetLastError(), "poa kernel");
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0_, ev1_);
        total_ms += ms;
        stats_.cells += cells;
        std::vector<uint32_t> again;
        for (uint32_t w : todo) {
            if (flags[w] & kFailed) throw Error{RB_ERR_DEVICE, "rb_poa: window consensus failed on the device"};
            if (flags[w] & kOverflow) again.push_back(w);
        }
        if (!again.empty()) {
            if (ncap >= (1 << 20)) throw Error{RB_ERR_DEVICE, "rb_poa: window graph exceeds 2^20 nodes"};
            ncap *= 4;
        }
        todo.swap(again);
    }
    stats_.kernel_ms = total_ms;
    stats_.top_kernel_ms = total_ms;
    stats_.max_nodes = uint32_t(ncap);
}

void PoaEngine::fetch(rb_poa_result* out) {
    const size_t n = nwin_;
    std::vector<uint32_t> lens(n);
    std::vector<uint8_t> flags(n);
    h_out_.reserve(std::max<uint64_t>(out_cap_, 16));
    check_cuda(cudaEventRecord(ev2_, stream_), "cudaEventRecord");
    if (n) {
        check_cuda(cudaMemcpyAsync(lens.data(), d_outlen_.ptr, n * 4, cudaMemcpyDeviceToHost, stream_), "D2H lens");
        check_cuda(cudaMemcpyAsync(flags.data(), d_flags_.ptr, n, cudaMemcpyDeviceToHost, stream_), "D2H flags");
        check_cuda(cudaMemcpyAsync(h_out_.ptr, d_out_.ptr, out_cap_, cudaMemcpyDeviceToHost, stream_), "D2H cons");
    }
    check_cuda(cudaEventRecord(ev3_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "fetch sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev2_, ev3_);
    stats_.d2h_ms = ms;
    stats_.d2h_bytes = n * 5 + out_cap_;
    const PoaWinDev* wd = h_desc_.as<PoaWinDev>();
    const char* src = h_out_.as<char>();
    offsets_.assign(n + 1, 0);
    cons_.clear();
    polished_.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
        offsets_[i] = cons_.size();
        cons_.insert(cons_.end(), src + wd[i].out_off, src + wd[i].out_off + lens[i]);
        polished_[i] = (flags[i] & kPolished) ? 1 : 0;
        if (flags[i] & kChimeric) {
            fprintf(stderr, "[racon::Window::generate_consensus] warning: contig %lu might be chimeric in window %u!\n",
                    (unsigned long)labels_[i].first, labels_[i].second);
        }
    }
    offsets_[n] = cons_.size();
    out->consensus = cons_.data();
    out->offsets = offsets_.data();
    out->polished = polished_.data();
}

}  // namespace rb
