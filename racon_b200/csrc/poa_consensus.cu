// Window consensus on the device with the semantics of racon's
//   src/window.cpp:65-142  Window::generate_consensus
// over spoa's partial-order graph (linear-gap NW, match/mismatch/gap from
// racon's -m/-x/-g, engine built at src/polisher.cpp:181-185).
//
// Design (B200, sm_100a). One warp owns one window at a time; warps (4 per
// CTA, 12 per SM) are persistent and pull windows from a size-sorted queue.
// Each warp has a slot of global scratch (graph arrays first, then the DP
// score rows and decision bit-planes) and a 16 KB shared-memory ring.
// * Per layer: the subgraph of a partial layer, row descriptors (first
//   predecessor ranks, count, sink flag, base), the DP, the end cell, the
//   traceback and the insertion of the aligned layer, all warp-cooperative.
//   The steps that walk the graph build compact uint16 adjacency lists or
//   accumulators in the shared ring when they fit, so their dependent steps
//   read shared memory; loads of graph arrays go out 128 entries at a time.
// * The DP runs one row (graph node in a valid topological order kept
//   incrementally) at a time: lane l owns S consecutive columns, recent rows
//   sit in the ring, diagonal and vertical terms take the max over the
//   predecessors (DPX add-max forms), and the in-row gap term H[i][j] =
//   max(T[j], H[i][j-1] + g) is a max-plus prefix (in-lane sub-chains, warp
//   scan). Decisions are two bit-planes per lane and row; the walk decides
//   the rare remaining cells again from the stored scores, in spoa's order
//   (diagonal through each predecessor, then vertical, then horizontal).
// * The NW end cell is the first sink in spoa's topological order with the
//   best last-column score; spoa's DFS order is built only when tied sinks
//   belong to aligned groups.
// * After the last layer: spoa's topological order, heaviest bundle (scores
//   in shared memory), branch completion, coverages and trimming.
// Exact int32 arithmetic throughout; results are byte-identical to the CPU
// algorithm by construction.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <cstdlib>
#include <memory>
#include <numeric>

#include "rb_internal.hpp"
#include "ring_queue.cuh"

namespace rb {

// One batch of windows in the shared queue (device record, written before
// its items are published): the batch's device buffers, as PoaArgs holds
// them for a private launch.
struct PoaJobDev {
    SvcJobHead head;            // windows of the batch, generation
    const uint8_t* in;
    const PoaWinDev* wins;
    const PoaLayerDev* layers;
    char* out;
    uint32_t* out_len;
    uint8_t* flags;
    unsigned long long* cells;  // [0] DP cells, [1] edge-cells (device)
    int trim;
    uint32_t pad;
};

namespace {

// minus infinity that survives thousands of gap additions without overflow
constexpr int kNegInf = -(1 << 29);
// per-warp shared memory: the DP row ring, reused by the other steps
constexpr int kRingBytesPerWarp = 16384;
// node ranks held in the ring's shared memory during the descriptor build
constexpr int kSmemRanks = (kRingBytesPerWarp - 512) / 4;

enum PoaFlag : uint8_t {
    kPolished = 1,
    kChimeric = 2,
    kOverflow = 4,
    kFailed = 8,
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
    unsigned long long* cells;   // [0] DP cells computed, [1] edge-cells
    uint32_t per_warp_cap;       // windows a warp takes per launch (0: until the queue is empty)
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
    int4* rowdesc;  // per DP row: first three predecessor ranks (or the list offset) | count, sink, base
    int *aln_node, *aln_pos;
    long long* bscore;
    int* bpred;
    int* cons;
    // valid topological order kept incrementally (rank -> node, node -> rank),
    // its double buffer, per-rank shift counts and the new nodes of a layer
    int *ord, *ord2, *my_rank, *shift, *nw_node, *nw_slot;
    int* H;
    uint8_t* dec;
    int* lastH;   // per DP row (sinks): score of the last column
    // per-node in-edge and aligned-entry counts, owner node of each aligned
    // entry (for the compact lists built in shared memory)
    int *in_cnt, *al_cnt, *a_owner, *out_cnt;
    int ncap, ecap, acap, scap, lcap, alncap;
};

__host__ __device__ size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Decision bytes are stored in tiles of 8 rows x 128 columns (1 KiB): a
// warp still writes each row as whole 128-byte lines, and the traceback,
// which walks up and left one cell at a time through nearby rows, stays
// inside one tile for several steps. lc is a multiple of 128.
__device__ __forceinline__ size_t dec_at(int i, int j, int lc) {
    return size_t(i) * size_t(lc) + size_t(j);
}

// Decision bit-planes of dp_layer_fast: one uint2 per (row, lane), row-major
// (each row is one coalesced 256-byte store).
__device__ __forceinline__ size_t bits_at(int i, int lane) { return size_t(i) * 32u + size_t(lane); }

// Row descriptor word w: predecessor count (17 bits) | sink << 17 | base << 24.
__device__ __forceinline__ int desc_np(int w) { return w & 0x1FFFF; }
__device__ __forceinline__ bool desc_sink(int w) { return (w >> 17) & 1; }
__device__ __forceinline__ uint32_t desc_base(int w) { return uint32_t(w) >> 24; }

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
    // graph arrays (touched by the pointer-walking steps) first, packed;
    // the DP matrices, streamed once per layer, last
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
    take(N * 4, 33);       // ord
    take(N * 4, 34);       // ord2
    take(N * 4, 35);       // my_rank
    take((N + 2) * 4, 36); // shift
    take(N * 4, 37);       // nw_node
    take(N * 4, 38);       // nw_slot
    take((N + 32) * 16, 39);  // rowdesc
    take(N * 4, 40);       // in_cnt
    take(N * 4, 41);       // al_cnt
    take(A * 4, 42);       // a_owner
    take(N * 4, 43);       // out_cnt
    take((N + 2) * 4, 24); // pred_off
    take((E + N + 2) * 4, 25);  // pred_idx
    take((N + L + 2) * 4, 26);  // aln_node
    take((N + L + 2) * 4, 27);  // aln_pos
    take(N * 8, 28);       // bscore
    take(N * 4, 29);       // bpred
    take(N * 4, 30);       // cons
    take(S * 4, 23);       // stack
    take((N + 1) * L * 4, 31);  // H
    take(std::max(((N + 8) & ~size_t(7)) * L, (N + 1) * 256), 32);  // dec: bytes, or 32 uint2 per row
    take((N + 1) * 4, 44);      // lastH: last-column score of each sink row
    // whole 2 MiB pages per slot, so that a slot's graph arrays share one page
    off = (off + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    return off;
}

__device__ Graph make_graph(const PoaArgs& a, uint32_t slot) {
    uint8_t* base = a.scratch + size_t(slot) * a.slot_bytes;
    Graph g;
    void* p[45];
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
    g.ord = (int*)p[33];
    g.ord2 = (int*)p[34];
    g.my_rank = (int*)p[35];
    g.shift = (int*)p[36];
    g.nw_node = (int*)p[37];
    g.nw_slot = (int*)p[38];
    g.rowdesc = (int4*)p[39];
    g.in_cnt = (int*)p[40];
    g.al_cnt = (int*)p[41];
    g.a_owner = (int*)p[42];
    g.out_cnt = (int*)p[43];
    g.lastH = (int*)p[44];
    g.ncap = a.ncap;
    g.ecap = a.ecap;
    g.acap = a.acap;
    g.scap = a.ncap + a.ecap + a.acap + 16;
    g.lcap = a.lcap;
    g.alncap = a.ncap + a.lcap + 2;
    return g;
}

// Shared per-CTA state.
// NW end cell of one layer: first sink row (in the DP order) with the best
// last-column value, that value, and how many sinks share it.
struct EndCell {
    int row, value, ties;
    int preds;  // predecessor links over the DP rows (edge-cells = |layer| x (rows + preds))
    bool h16;   // the layer's score rows in global memory are int16
};

struct PoaShared {
    int nnodes, nedges, naligned, nseq;
    int nnew;     // new nodes of the last insertion (g.nw_node / g.nw_slot)
    int nranks;   // entries of rank_to_node (full graph order)
    int ndp;      // rows of the current DP
    int fail;     // 0 ok, else PoaFlag
    int iend;     // DP rank of the NW end cell
    int naln;
};

// ---------------- graph primitives (thread 0) ----------------

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

// Warp prefix helpers: exclusive prefix of v over lanes, and the total.
__device__ __forceinline__ int warp_excl(int v, int lane, int& total) {
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// Out-edges of nodes [0, N) as uint16 lists in shared memory: destination and
// edge id, grouped by source (order within a source is irrelevant: the lists
// answer "does u -> v exist, and which edge is it"). Loads of the edge
// arrays go four 32-edge chunks at a time. Returns false, building nothing,
// when the lists do not fit in `cap` bytes or 16-bit indices.
struct OutCsr {
    uint16_t* off;  // [N + 1]
    uint16_t* dst;  // [E]
    uint16_t* eid;  // [E]
};
__device__ bool build_out_csr(const Graph& g, int N, int E, int lane, void* smem, int cap, OutCsr& c) {
    if (N >= 65535 || E >= 65535 || 2 * (size_t(N) + 1) + 4 * size_t(E) > size_t(cap)) return false;
    c.off = reinterpret_cast<uint16_t*>(smem);
    c.dst = c.off + (N + 1);
    c.eid = c.dst + E;
    int b = 0;
    for (int c4 = 0; c4 < N; c4 += 128) {
        int cn[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int v = c4 + 32 * u + lane;
            cn[u] = v < N ? g.out_cnt[v] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int v = c4 + 32 * u + lane;
            int t = 0;
            const int x = warp_excl(cn[u], lane, t);
            if (v < N) c.off[v] = uint16_t(b + x);
            b += t;
        }
    }
    if (lane == 0) c.off[N] = uint16_t(E);
    __syncwarp();
    const unsigned below = (1u << lane) - 1u;
    for (int c4 = 0; c4 < E; c4 += 128) {
        int ss[4], ds[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = c4 + 32 * u + lane;
            ss[u] = e < E ? g.e_src[e] : -1 - lane;
            ds[u] = e < E ? g.e_dst[e] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int src = ss[u];
            const unsigned grp = __match_any_sync(0xffffffffu, src);
            const int cur = src >= 0 ? c.off[src] : 0;
            __syncwarp();
            if (src >= 0) {
                const int q = cur + __popc(grp & below);
                c.dst[q] = uint16_t(ds[u]);
                c.eid[q] = uint16_t(c4 + 32 * u + lane);
                if ((grp & below) == 0) c.off[src] = uint16_t(cur + __popc(grp));
            }
            __syncwarp();
        }
    }
    for (int c0 = ((N - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
        const int v = c0 + lane;
        const uint16_t pv = (v < N && v > 0) ? c.off[v - 1] : uint16_t(0);
        __syncwarp();
        if (v < N) c.off[v] = pv;
        __syncwarp();
    }
    return true;
}

// Graph::add_alignment for one layer, by the whole warp. A path visits every
// node and every aligned group at most once, so the per-position work is
// independent: classify each aligned base (existing node, new base, new
// member of an aligned group), number the new nodes in spoa's order (head
// bases, tail bases, then new aligned bases along the path), then in
// parallel create nodes, aligned-group links, edges P[k-1] -> P[k] with
// weight w[k-1] + w[k] (every sequence position k owns exactly one path node
// P[k]) and coverage, and list the new nodes with their order slots (see
// order_insert). Per-entry scratch lives in g.stack: [0,m) node, [m,2m) kind
// | aligned-count << 2, [2m,3m) anchor slot, [3m,4m) group start.
__device__ void add_alignment_warp(const Graph& g, PoaShared& sh, const uint8_t* seq, const uint8_t* qual,
                                   int len, int lane, int4* ring) {
    const int m = sh.naln;
    const int nold = sh.nnodes;
    if (len == 0) return;
    if (m == 0 || 4 * m + 64 > g.scap) {
        if (lane == 0) sh.fail = m == 0 ? kFailed : kOverflow;
        __syncwarp();
        return;
    }
    int* e_nid = g.stack;
    int* e_kind = g.stack + m;
    int* e_slot = g.stack + 2 * m;
    int* e_start = g.stack + 3 * m;
    const int first_pos = g.aln_pos[m - 1], last_pos = g.aln_pos[0];
    const int h = first_pos, tl = len - 1 - last_pos;
    // existing-edge lookups of step 5 from shared memory when they fit
    OutCsr oc;
    const bool ocsr = build_out_csr(g, nold, sh.nedges, lane, ring, kRingBytesPerWarp, oc);
    // 1. classify (reads only the graph as it was before this insertion);
    //    the loads of four 32-entry chunks go out together
    for (int t4 = 0; t4 < m; t4 += 128) {
        int at[4], pos[4], cd[4], rk[4], ah[4];
        uint8_t letter[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = t4 + 32 * u + lane;
            at[u] = t < m ? g.aln_node[m - 1 - t] : -1;
            pos[u] = t < m ? g.aln_pos[m - 1 - t] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = t4 + 32 * u + lane;
            letter[u] = t < m ? seq[pos[u]] : 0;
            cd[u] = at[u] >= 0 ? g.code[at[u]] : -1;
            rk[u] = at[u] >= 0 ? g.my_rank[at[u]] : 0;
            ah[u] = at[u] >= 0 ? g.al_head[at[u]] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = t4 + 32 * u + lane;
            if (t >= m) continue;
            int kind = 1, nid = -1, nal = 0, slot = INT_MIN, start = INT_MAX;
            if (at[u] != -1) {
                // the rank extent, in the incremental order, of v's aligned
                // group among the nodes that existed before this insertion
                slot = start = rk[u];
                const bool same = cd[u] == int(letter[u]);
                for (int x = ah[u]; x != -1; x = g.a_next[x]) {
                    const int y = g.a_node[x];
                    if (y < nold) {
                        const int ry = g.my_rank[y];
                        slot = max(slot, ry);
                        start = min(start, ry);
                    }
                    if (!same) {
                        ++nal;
                        if (nid == -1 && g.code[y] == letter[u]) nid = y;
                    }
                }
                if (same) {
                    kind = 0;
                    nid = at[u];
                } else {
                    kind = nid == -1 ? 2 : 0;
                }
            }
            e_nid[t] = nid;
            e_kind[t] = kind | (kind == 2 ? nal << 2 : 0);
            e_slot[t] = slot;
            e_start[t] = start;
        }
    }
    __syncwarp();
    // 2. ids of new aligned bases, aligned-pool offsets, order slots
    const int base_id = nold + h + tl;
    int nnew_e = 0, nal_tot = 0, cur_slot = INT_MIN, first_start = INT_MAX;
    for (int c0 = 0; c0 < m; c0 += 32) {
        const int t = c0 + lane;
        const int kd = t < m ? e_kind[t] : 0;
        const int kind = kd & 3;
        const bool is_new = t < m && kind != 0;
        int tot;
        const int pre = warp_excl(is_new ? 1 : 0, lane, tot);
        int atot;
        const int apre = warp_excl(kind == 2 ? 2 * (kd >> 2) + 2 : 0, lane, atot);
        // last anchor slot up to t (anchors: kind 0 or 2), carried over chunks
        int sl = (t < m && kind != 1) ? e_slot[t] : INT_MIN;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, sl, o);
            if (lane >= o) sl = max(sl, y);
        }
        sl = max(sl, cur_slot);
        int st = (t < m && kind != 1) ? e_start[t] : INT_MAX;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) st = min(st, __shfl_xor_sync(0xffffffffu, st, o));
        if (first_start == INT_MAX) first_start = st;
        if (t < m) {
            if (is_new) e_nid[t] = base_id + nnew_e + pre;
            // kind 2: own group slot; kind 1: last anchor before it (INT_MIN: none yet)
            e_slot[t] = kind == 2 ? e_slot[t] : sl;
            e_start[t] = nal_tot + apre;  // aligned-pool offset (kind 2)
        }
        cur_slot = __shfl_sync(0xffffffffu, sl, 31);
        nnew_e += tot;
        nal_tot += atot;
    }
    const int nnew = h + tl + nnew_e;
    if (nold + nnew > g.ncap || sh.nedges + len + 2 > g.ecap || sh.naligned + nal_tot > g.acap) {
        if (lane == 0) sh.fail = kOverflow;
        __syncwarp();
        return;
    }
    __syncwarp();
    // 3. new nodes
    auto path_node = [&](int k) -> int {
        if (k < first_pos) return nold + k;
        if (k > last_pos) return nold + h + (k - last_pos - 1);
        return e_nid[k - first_pos];
    };
    for (int x = lane; x < nnew; x += 32) {
        int id, k;
        if (x < h) {
            id = nold + x;
            k = x;
        } else if (x < h + tl) {
            id = nold + x;
            k = last_pos + 1 + (x - h);
        } else {
            id = nold + x;
            k = -1;
        }
        g.code[id] = k >= 0 ? seq[k] : 0;
        g.cov[id] = 0;
        g.in_head[id] = g.in_tail[id] = -1;
        g.out_head[id] = g.out_tail[id] = -1;
        g.al_head[id] = g.al_tail[id] = -1;
        g.in_cnt[id] = 0;
        g.al_cnt[id] = 0;
        g.out_cnt[id] = 0;
    }
    __syncwarp();
    for (int t = lane; t < m; t += 32) {
        if ((e_kind[t] & 3) != 0) g.code[e_nid[t]] = seq[first_pos + t];
    }
    __syncwarp();
    // 4. aligned groups: a new base joining the group of `at` links to every
    //    member, then to `at` (spoa's order)
    for (int t = lane; t < m; t += 32) {
        if ((e_kind[t] & 3) != 2) continue;
        const int at = g.aln_node[m - 1 - t];
        const int G = e_nid[t];
        int slot = sh.naligned + e_start[t];
        auto link = [&](int v, int y) {
            g.a_node[slot] = y;
            g.a_owner[slot] = v;
            g.al_cnt[v] += 1;  // one group per node and layer: no other lane links v
            g.a_next[slot] = -1;
            if (g.al_tail[v] == -1) g.al_head[v] = slot;
            else g.a_next[g.al_tail[v]] = slot;
            g.al_tail[v] = slot;
            ++slot;
        };
        for (int x = g.al_head[at]; x != -1; x = g.a_next[x]) {
            const int y = g.a_node[x];
            link(G, y);
            link(y, G);
        }
        link(G, at);
        link(at, G);
    }
    __syncwarp();
    // 5. edges P[k-1] -> P[k]: existing ones gain weight, new ones are appended
    int new_edges = 0;
    for (int c0 = 1; c0 < len; c0 += 32) {
        const int k = c0 + lane;
        int u = -1, v = -1, w = 0, found = -1;
        if (k < len) {
            u = path_node(k - 1);
            v = path_node(k);
            w = layer_weight(qual, k - 1) + layer_weight(qual, k);
            if (u < nold && v < nold) {
                if (ocsr) {
                    for (int q = oc.off[u], qe = oc.off[u + 1]; q < qe; ++q)
                        if (oc.dst[q] == v) {
                            found = oc.eid[q];
                            break;
                        }
                } else {
                    for (int e = g.out_head[u]; e != -1; e = g.e_next_out[e])
                        if (g.e_dst[e] == v) {
                            found = e;
                            break;
                        }
                }
            }
        }
        int tot;
        const int pre = warp_excl((k < len && found < 0) ? 1 : 0, lane, tot);
        __syncwarp();
        if (k < len) {
            if (found >= 0) {
                g.e_w[found] += w;
            } else {
                const int id = sh.nedges + new_edges + pre;
                g.e_src[id] = u;
                g.e_dst[id] = v;
                g.e_w[id] = w;
                g.e_next_in[id] = -1;
                g.e_next_out[id] = -1;
                if (g.out_tail[u] == -1) g.out_head[u] = id;
                else g.e_next_out[g.out_tail[u]] = id;
                g.out_tail[u] = id;
                if (g.in_tail[v] == -1) g.in_head[v] = id;
                else g.e_next_in[g.in_tail[v]] = id;
                g.in_tail[v] = id;
                g.in_cnt[v] += 1;  // at most one new edge into v per layer
                g.out_cnt[u] += 1;  // and at most one out of u
            }
        }
        new_edges += tot;
        __syncwarp();
    }
    // 6. coverage: every node of a path with at least two bases
    if (len >= 2)
        for (int k = lane; k < len; k += 32) g.cov[path_node(k)] += 1;
    // 7. new nodes with their order slots, in path order
    const int before = first_start == INT_MAX ? nold - 1 : first_start - 1;
    const int last_slot = cur_slot == INT_MIN ? before : cur_slot;
    for (int x = lane; x < h; x += 32) {
        g.nw_node[x] = nold + x;
        g.nw_slot[x] = before;
    }
    for (int t = lane; t < m; t += 32) {
        if ((e_kind[t] & 3) == 0) continue;
        const int id = e_nid[t];
        const int at = id - base_id;  // position among the new aligned bases
        const int sl = e_slot[t];
        g.nw_node[h + at] = id;
        g.nw_slot[h + at] = sl == INT_MIN ? before : sl;
    }
    for (int x = lane; x < tl; x += 32) {
        g.nw_node[h + nnew_e + x] = nold + h + x;
        g.nw_slot[h + nnew_e + x] = last_slot;
    }
    __syncwarp();
    if (lane == 0) {
        sh.nnodes = nold + nnew;
        sh.nedges += new_edges;
        sh.naligned += nal_tot;
        sh.nnew = nnew;
        sh.nseq += 1;
    }
    __syncwarp();
}

// Splices the new nodes of the last insertion into the incremental order
// (warp): an old node at rank r moves up by the number of new nodes with slot
// < r, the k-th new node (slots sorted) lands at slot + 1 + k.
__device__ void order_insert(const Graph& g, const PoaShared& sh, int nold, int lane, int4* ring) {
    const int nnew = sh.nnew, n = nold + nnew;
    // shift counts in shared memory when they fit (the ring is free here)
    int* const shift = size_t(nold + 1) * 4 <= size_t(kRingBytesPerWarp) ? reinterpret_cast<int*>(ring) : g.shift;
    for (int r = lane; r <= nold; r += 32) shift[r] = 0;
    __syncwarp();
    for (int k = lane; k < nnew; k += 32) {
        const int at = g.nw_slot[k] + 1;
        if (at < nold) atomicAdd(&shift[at], 1);
    }
    __syncwarp();
    int base = 0;
    for (int c4 = 0; c4 < nold; c4 += 128) {
        int ov[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = c4 + 32 * u + lane;
            ov[u] = r < nold ? g.ord[r] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = c4 + 32 * u + lane;
            int v = r < nold ? shift[r] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += y;
            }
            if (r < nold) g.ord2[r + base + v] = ov[u];
            base += __shfl_sync(0xffffffffu, v, 31);
        }
    }
    for (int k = lane; k < nnew; k += 32) g.ord2[g.nw_slot[k] + 1 + k] = g.nw_node[k];
    __syncwarp();
    for (int x4 = 0; x4 < n; x4 += 128) {
        int vv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = x4 + 32 * u + lane;
            vv[u] = x < n ? g.ord2[x] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = x4 + 32 * u + lane;
            if (x < n) {
                g.ord[x] = vv[u];
                g.my_rank[vv[u]] = x;
            }
        }
    }
    __syncwarp();
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

// Predecessor p (in in-edge order) of a DP row from its descriptor: DP rank
// (0 = the empty prefix row when the row has no predecessor).
__device__ __forceinline__ int desc_pred(const Graph& g, const int4& d, int p) {
    const int np = desc_np(d.w);
    if (np == 0) return 0;
    if (np > 3) return p == 0 ? d.y : g.pred_idx[d.x + p];
    return p == 0 ? d.x : (p == 1 ? d.y : d.z);
}

// ---------------- DP of one layer (one warp) ----------------

// Columns covered by one warp pass: S cells per lane, S a multiple of 4.
__host__ __device__ inline int seg_cells(int wc) {
    const int s = (wc + 31) / 32;
    return s <= 24 ? ((s + 3) & ~3) : 24;
}
__host__ __device__ inline int row_cover(int wc) {
    const int s = seg_cells(wc);
    const int ch = 32 * s;
    return ((wc + ch - 1) / ch) * ch;
}

constexpr uint32_t kNoPred = 0xFFu;
constexpr uint32_t kEscape = 63u;  // predecessor index >= 63: decide again in the walk

// DP of one layer against rows order[0..ndp) (ranks 1..ndp; rank 0 = empty
// prefix row). Lane l owns columns [c + l*S, c + l*S + S) of each chunk c of
// 32*S columns. Per cell it keeps T = max over predecessors of the diagonal
// and vertical terms, the first predecessor giving T diagonally and the first
// giving it vertically; the horizontal term is a max-plus scan: in-lane
// prefix, then a warp shuffle scan of lane aggregates. Decision byte: p
// (diagonal via predecessor p), 64 + p (vertical), 128 (horizontal), 255
// (predecessor index >= 63). Returns the rank of the NW end cell (first sink
// in rank order with the best last-column value).
template <int S>
__device__ EndCell dp_layer(const PoaArgs& a, const Graph& g, const int* order, int ndp, const uint8_t* seq, int L,
                        int lane) {
    static_assert(S % 4 == 0 && S >= 4 && S <= 32, "segment");
    constexpr unsigned kFull = 0xffffffffu;
    const int lc = g.lcap;
    int* const Hm = g.H;
    uint8_t* const Dm = g.dec;
    const int wc = L + 1;
    const int ch = 32 * S;
    const int nch = (wc + ch - 1) / ch;
    const int gap = a.gap, mt = a.match, mm = a.mismatch;
    // virtual row 0: j * gap
    for (int j = lane; j < nch * ch; j += 32) Hm[j] = j * gap;
    __syncwarp();
    const int lane_l = (L % ch) / S, k_l = L % S, ch_l = L / ch;
    int best_v = kNegInf, best_r = INT_MAX, ties = 0, npreds = 0;
    for (int i = 1; i <= ndp; ++i) {
        const int4 d = g.rowdesc[i - 1];
        const uint32_t cmask = desc_base(d.w) * 0x01010101u;
        const int np = desc_np(d.w);
        npreds += np;
        const int cnt = np == 0 ? 1 : np;
        const bool is_sink = desc_sink(d.w);
        int carry_in = kNegInf;  // final H of the last column of the previous chunk
        for (int c = 0; c < nch; ++c) {
            const int j0 = c * ch + lane * S;
            // sequence chars of columns j0 .. j0+S-1 (column j compares seq[j-1])
            uint32_t eq[S / 4];
#pragma unroll
            for (int q = 0; q < S / 4; ++q) {
                uint32_t w = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int j = j0 + 4 * q + b;
                    const uint32_t ch8 = (j >= 1 && j <= L) ? uint32_t(seq[j - 1]) : 0u;
                    w |= ch8 << (8 * b);
                }
                eq[q] = __vcmpeq4(w, cmask);
            }
            int T[S];
            uint32_t code[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                T[k] = kNegInf;
                code[k] = 0xFFFFu;
            }
            for (int p = 0; p < cnt; ++p) {
                const int r = desc_pred(g, d, p);
                const int4* hp4 = reinterpret_cast<const int4*>(Hm + r * lc + j0);
                int hv[S];
#pragma unroll
                for (int q = 0; q < S / 4; ++q) {
                    const int4 t4 = hp4[q];
                    hv[4 * q] = t4.x;
                    hv[4 * q + 1] = t4.y;
                    hv[4 * q + 2] = t4.z;
                    hv[4 * q + 3] = t4.w;
                }
                int left = __shfl_up_sync(kFull, hv[S - 1], 1);
                if (lane == 0) left = j0 > 0 ? Hm[r * lc + j0 - 1] : kNegInf;
                const uint32_t pc = p < int(kEscape) ? uint32_t(p) : kEscape;
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    const int prev = k == 0 ? left : hv[k - 1];
                    const bool same = (eq[k / 4] >> (8 * (k % 4))) & 1u;
                    const int dg = prev <= kNegInf / 2 ? kNegInf : prev + (same ? mt : mm);
                    const int vt = hv[k] + gap;
                    const int mx = max(dg, vt);
                    if (mx > T[k]) {
                        T[k] = mx;
                        code[k] = (dg == mx ? pc : kNoPred) | ((vt == mx ? pc : kNoPred) << 8);
                    } else if (mx == T[k]) {
                        if ((code[k] & 0xFFu) == kNoPred && dg == mx) code[k] = (code[k] & 0xFF00u) | pc;
                        if ((code[k] >> 8) == kNoPred && vt == mx) code[k] = (code[k] & 0xFFu) | (pc << 8);
                    }
                }
            }
            // horizontal term: in-lane prefix, warp scan of lane aggregates
            int hk[S];
            int run = kNegInf;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                run = max(T[k], run <= kNegInf / 2 ? kNegInf : run + gap);
                hk[k] = run;
            }
            int x = run;
            if (lane == 0 && carry_in > kNegInf / 2) x = max(x, carry_in + S * gap);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, x, o);
                if (lane >= o && y > kNegInf / 2) x = max(x, y + o * S * gap);
            }
            int carry = __shfl_up_sync(kFull, x, 1);
            if (lane == 0) carry = carry_in;
            int hrow[S];
            uint32_t dec4[S / 4];
#pragma unroll
            for (int q = 0; q < S / 4; ++q) dec4[q] = 0;
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int cin = carry <= kNegInf / 2 ? kNegInf : carry + (k + 1) * gap;
                const int h = max(hk[k], cin);
                hrow[k] = h;
                uint32_t d;
                if (h > T[k]) {
                    d = 128u;
                } else if ((code[k] & 0xFFu) != kNoPred) {
                    d = code[k] & 0xFFu;
                    if (d == kEscape) d = 255u;
                } else {
                    d = (code[k] >> 8);
                    d = d == kEscape ? 255u : 64u + d;
                }
                dec4[k / 4] |= d << (8 * (k % 4));
            }
            int4* out4 = reinterpret_cast<int4*>(Hm + i * lc + j0);
#pragma unroll
            for (int q = 0; q < S / 4; ++q)
                out4[q] = make_int4(hrow[4 * q], hrow[4 * q + 1], hrow[4 * q + 2], hrow[4 * q + 3]);
#pragma unroll
            for (int q = 0; q < S / 4; ++q) *reinterpret_cast<uint32_t*>(Dm + dec_at(i, j0 + 4 * q, lc)) = dec4[q];
            if (c == ch_l && lane == lane_l && is_sink) {
                int val = kNegInf;
#pragma unroll
                for (int k = 0; k < S; ++k)
                    if (k == k_l) val = hrow[k];
                g.lastH[i] = val;
                if (val > best_v) {
                    best_v = val;
                    best_r = i;
                    ties = 1;
                } else if (val == best_v) {
                    ++ties;
                }
            }
            carry_in = __shfl_sync(kFull, hrow[S - 1], 31);
        }
        __syncwarp();
    }
    // the owner lane of column L holds the end cell (int32 score rows)
    return EndCell{__shfl_sync(kFull, best_r, lane_l), __shfl_sync(kFull, best_v, lane_l),
                   __shfl_sync(kFull, ties, lane_l), npreds, false};
}

// Score rows in global memory (read back for rows beyond the ring and by
// the walk's re-decisions) are int16 for a layer whose scores provably fit:
// every score lies between gap x (rows + columns) (the all-gap path, which
// the maximum includes) and max(match, 0) x columns, so with
// (ndp + L) x |gap| <= 32767 and max(match, 0) x L <= 32767 no score leaves
// [-32767, 32767]. Other layers are promoted to int32 rows. Stores saturate,
// so minus infinity (kNegInf and what is derived from it) becomes -32768,
// which no score reaches and which reads back as kNegInf. The DP itself
// stays int32 in registers and in the ring.
__device__ __forceinline__ bool layer_fits_s16(const PoaArgs& a, int ndp, int L) {
    return a.gap <= 0 && (long long)(ndp + L) * (long long)(-a.gap) <= 32767 &&
           (long long)max(int(a.match), 0) * (long long)L <= 32767;
}
// two scores in one word, lo in bits 0..15 and hi in bits 16..31, saturated
__device__ __forceinline__ uint32_t pack_s16(int lo, int hi) {
    uint32_t d;
    asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(hi), "r"(lo));
    return d;
}
__device__ __forceinline__ int s16_score(int v) { return v == -32768 ? kNegInf : v; }
__device__ __forceinline__ int unpack_lo(uint32_t w) { return s16_score(int(w << 16) >> 16); }
__device__ __forceinline__ int unpack_hi(uint32_t w) { return s16_score(int(w) >> 16); }
// score (row r, column j) as the layer stored it
__device__ __forceinline__ int h_at(const Graph& g, int r, int j, bool h16) {
    if (h16) return s16_score(reinterpret_cast<const int16_t*>(g.H)[r * g.lcap + j]);
    return g.H[r * g.lcap + j];
}

// last 512 bytes of each warp's ring hold the 32-row descriptor block
constexpr int kRingDescOffset = (kRingBytesPerWarp - 512) / 16;

// Single-pass form of dp_layer for rows of at most 32*S columns. A lane only
// ever reads its own column segment of earlier rows (the left neighbour
// comes by shuffle), so rows are served without any cross-lane memory
// ordering: the last R rows sit in a shared-memory ring laid out
// [row][S/4][lane] (conflict-free int4), older rows come from global memory.
// Row descriptors are prefetched 32 rows at a time.
// Per cell: T = max over predecessors of the diagonal (H[p][j-1] + s) and
// vertical (H[p][j] + g) terms, with the DPX forms max(a + b, c) and
// max-with-predicate doing the add/max pairs; the horizontal term is a
// max-plus scan (in-lane prefix as 4 independent sub-chains, warp scan of the
// lane aggregates, one fix-up per cell). Decisions are two bit-planes per lane
// and row (one uint2): bit k of .x = horizontal (h > T), bit k of .y = the
// diagonal through predecessor 0 gives T (spoa tests it first). The walk
// reads the rest from the row's predecessor count: a single predecessor
// makes every other cell vertical through it; with several it decides again
// from H. Requires match >= mismatch and match - mismatch <= 255.
template <int S, bool H16>
__device__ EndCell dp_layer_fast(const PoaArgs& a, const Graph& g, const int* order, int ndp, const uint8_t* seq, int L,
                             int lane, int4* ring) {
    static_assert(S % 4 == 0 && S >= 4 && S <= 24, "segment");
    constexpr unsigned kFull = 0xffffffffu;
    constexpr int Q = S / 4;
    constexpr int R = (kRingBytesPerWarp - 512) / (S * 128);
    static_assert(R >= 2, "ring");
    const int lc = g.lcap;
    int* const Hm = g.H;
    uint2* const D2 = reinterpret_cast<uint2*>(g.dec);
    const int* const pred_idx = g.pred_idx;
    const int gap = a.gap, mm = a.mismatch;
    const uint32_t diff4 = uint32_t(a.match - a.mismatch) * 0x01010101u;
    const int j0 = lane * S;
    uint32_t sc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        uint32_t w = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = j0 + 4 * q + b;
            w |= ((j >= 1 && j <= L) ? uint32_t(seq[j - 1]) : 0u) << (8 * b);
        }
        sc[q] = w;
    }
    int16_t* const Hs = reinterpret_cast<int16_t*>(g.H);  // the same rows as int16 (H16)
    // row 0 (empty graph prefix) in global memory for the traceback
#pragma unroll
    for (int k = 0; k < S; ++k) {
        if (H16) {
            Hs[j0 + k] = int16_t((j0 + k) * gap);
        } else {
            Hm[j0 + k] = (j0 + k) * gap;
        }
    }
    const int lane_l = L / S, k_l = L % S;
    int best_v = kNegInf, best_r = INT_MAX, ties = 0, npreds = 0;
    int4* const dblk = ring + kRingDescOffset;
    const int4* const rowdesc = g.rowdesc;
    int4 pre = lane < ndp ? rowdesc[lane] : make_int4(0, 0, 0, 0);
    // hv holds the previous row's final scores between iterations (row 0
    // first), and left_prev that row's score left of the lane's segment: a
    // row whose first predecessor is the row just computed (the common
    // chain) reads both from registers instead of the ring and a shuffle
    int hv[S];
#pragma unroll
    for (int k = 0; k < S; ++k) hv[k] = (j0 + k) * gap;
    int left_prev = lane == 0 ? kNegInf : (j0 - 1) * gap;
    // the next row's descriptor is read while this row's scan and stores
    // are in flight (from the staged block, or from `pre` at a block edge)
    int4 dnext = make_int4(__shfl_sync(kFull, pre.x, 0), __shfl_sync(kFull, pre.y, 0),
                           __shfl_sync(kFull, pre.z, 0), __shfl_sync(kFull, pre.w, 0));
    for (int i = 1; i <= ndp; ++i) {
        const int bi = (i - 1) & 31;
        if (bi == 0) {
            __syncwarp();
            dblk[lane] = pre;
            __syncwarp();
            const int nx = i - 1 + 32 + lane;
            pre = nx < ndp ? rowdesc[nx] : make_int4(0, 0, 0, 0);
        }
        const int4 d = dnext;
        const int np = desc_np(d.w);
        npreds += np;
        const bool is_sink = desc_sink(d.w);
        const uint32_t cmask = desc_base(d.w) * 0x01010101u;
        const int p0 = np > 3 ? d.y : d.x;
        // per cell: match - mismatch where the base matches, else 0 (bytes)
        uint32_t sw[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) sw[q] = __vcmpeq4(sc[q], cmask) & diff4;
        int T[S];
        uint32_t dbit = 0;
        // row r's scores of the lane's segment into dst
        auto load_row = [&](int r, int (&dst)[S]) {
            if (r == 0) {
#pragma unroll
                for (int k = 0; k < S; ++k) dst[k] = (j0 + k) * gap;
            } else if (i - r <= R) {
                // separate shared and global paths (warp-uniform branch), so
                // the ring is read with shared-memory loads, not generic ones
                const int4* src = ring + (r % R) * Q * 32 + lane;
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int4 t4 = src[q * 32];
                    dst[4 * q] = t4.x;
                    dst[4 * q + 1] = t4.y;
                    dst[4 * q + 2] = t4.z;
                    dst[4 * q + 3] = t4.w;
                }
            } else if (H16) {
                const uint2* src = reinterpret_cast<const uint2*>(Hs + r * lc + j0);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const uint2 t2 = src[q];
                    dst[4 * q] = unpack_lo(t2.x);
                    dst[4 * q + 1] = unpack_hi(t2.x);
                    dst[4 * q + 2] = unpack_lo(t2.y);
                    dst[4 * q + 3] = unpack_hi(t2.y);
                }
            } else {
                const int4* src = reinterpret_cast<const int4*>(Hm + r * lc + j0);
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int4 t4 = src[q];
                    dst[4 * q] = t4.x;
                    dst[4 * q + 1] = t4.y;
                    dst[4 * q + 2] = t4.z;
                    dst[4 * q + 3] = t4.w;
                }
            }
        };
        auto sbyte = [&](int k) -> int { return int((sw[k >> 2] >> (8 * (k & 3))) & 0xFFu); };
        {
            const int r0 = np == 0 ? 0 : p0;
            int left = left_prev;
            if (r0 != i - 1) {
                load_row(r0, hv);
                left = __shfl_up_sync(kFull, hv[S - 1], 1);
                if (lane == 0) left = kNegInf;
            }
            // Several predecessors: the maximum over them of the diagonal
            // (H[p][j-1] + s) and vertical (H[p][j] + g) terms is the
            // diagonal and vertical term of their elementwise maximum row M,
            // so each further row costs one max per cell. hv and left become
            // M; p0m / p0left mark the columns where the first predecessor
            // holds M, which is where its diagonal can give T.
            uint32_t p0m = ~0u;
            bool p0left = true;
            for (int p = 1; p < np; ++p) {
                load_row(np > 3 ? pred_idx[d.x + p] : (p == 1 ? d.y : d.z), T);
                int lft = __shfl_up_sync(kFull, T[S - 1], 1);
                if (lane == 0) lft = kNegInf;
                uint32_t lq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    bool keep;
                    hv[k] = __vibmax_s32(hv[k], T[k], &keep);
                    lq[k & 3] |= uint32_t(!keep) << k;
                }
                bool keepl;
                left = __vibmax_s32(left, lft, &keepl);
                p0left = p0left && keepl;
                p0m &= ~((lq[0] | lq[1]) | (lq[2] | lq[3]));
            }
            // T = max(M[j-1] + s, M[j] + g); the diagonal of predecessor 0
            // gives T where it holds M[j-1] and the diagonal is not below the
            // vertical. Decision bits gathered in four independent words.
            uint32_t dq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int pv = k == 0 ? left : hv[k - 1];
                const int dg = pv + mm + sbyte(k);
                bool dge;
                T[k] = __vibmax_s32(dg, hv[k] + gap, &dge);
                dq[k & 3] |= uint32_t(dge) << k;
            }
            dbit = ((dq[0] | dq[1]) | (dq[2] | dq[3])) & ((p0m << 1) | (p0left ? 1u : 0u));
        }
        // horizontal term
        constexpr int C = S / 4;  // cells per sub-chain
        int agg[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            int run = T[c * C];
            hv[c * C] = run;
#pragma unroll
            for (int k = c * C + 1; k < (c + 1) * C; ++k) {
                run = __viaddmax_s32(run, gap, T[k]);
                hv[k] = run;
            }
            agg[c] = run;
        }
        int x = agg[0];
#pragma unroll
        for (int c = 1; c < 4; ++c) x = __viaddmax_s32(x, C * gap, agg[c]);
        // max-plus prefix of the lane aggregates (penalty S * gap per lane),
        // rounds of offset 1, 2, 4, 8, 16, stopping at the first round in
        // which no lane changes: with a uniform penalty per lane, a round of
        // offset o that changes nothing means x_(l-o) + o S gap <= x_l for
        // every l, so x_(l-2o) + 2o S gap <= x_(l-o) + o S gap <= x_l and no
        // later round can change anything either. Horizontal runs rarely
        // cross a whole lane segment, so most rows stop after one round; a
        // run across many lanes takes at most five.
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, x, o);
            if (lane < o) y = kNegInf;
            const int nx = __viaddmax_s32(y, o * S * gap, x);
            const bool changed = nx != x;
            x = nx;
            if (!__any_sync(kFull, changed)) break;
        }
        int cin = __shfl_up_sync(kFull, x, 1);  // final value left of the segment
        if (lane == 0) cin = kNegInf;
        left_prev = cin;
        if (i < ndp) {
            const int bn = i & 31;  // slot of row i + 1 in the staged block
            if (bn == 0) {
                dnext = make_int4(__shfl_sync(kFull, pre.x, 0), __shfl_sync(kFull, pre.y, 0),
                                  __shfl_sync(kFull, pre.z, 0), __shfl_sync(kFull, pre.w, 0));
            } else {
                dnext = dblk[bn];
            }
        }
        uint32_t hq[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int next = __viaddmax_s32(cin, C * gap, agg[c]);
#pragma unroll
            for (int k = c * C; k < (c + 1) * C; ++k) {
                hv[k] = __viaddmax_s32(cin, (k - c * C + 1) * gap, hv[k]);
                hq[k & 3] |= uint32_t(hv[k] > T[k]) << k;
            }
            cin = next;
        }
        const uint32_t hbit = (hq[0] | hq[1]) | (hq[2] | hq[3]);
        int4* dst_g = reinterpret_cast<int4*>(Hm + i * lc + j0);
        uint2* dst_s = reinterpret_cast<uint2*>(Hs + i * lc + j0);
        int4* dst_r = ring + (i % R) * Q * 32 + lane;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int4 v4 = make_int4(hv[4 * q], hv[4 * q + 1], hv[4 * q + 2], hv[4 * q + 3]);
            // streamed: keep the graph arrays in L2
            if (H16) {
                __stcs(dst_s + q, make_uint2(pack_s16(v4.x, v4.y), pack_s16(v4.z, v4.w)));
            } else {
                __stcs(dst_g + q, v4);
            }
            dst_r[q * 32] = v4;
        }
        __stcs(D2 + bits_at(i, lane), make_uint2(hbit, dbit));
        if (lane == lane_l && is_sink) {
            int val = kNegInf;
#pragma unroll
            for (int k = 0; k < S; ++k)
                if (k == k_l) val = hv[k];
            g.lastH[i] = val;
            if (val > best_v) {
                best_v = val;
                best_r = i;
                ties = 1;
            } else if (val == best_v) {
                ++ties;
            }
        }
    }
    __syncwarp();
    return EndCell{__shfl_sync(kFull, best_r, lane_l), __shfl_sync(kFull, best_v, lane_l),
                   __shfl_sync(kFull, ties, lane_l), npreds, H16};
}

// True when the layer's DP runs in dp_layer_fast (bit-plane decisions).
__device__ __forceinline__ bool fast_dp(const PoaArgs& a, int L) {
    return L + 1 <= 32 * 24 && a.match >= a.mismatch && a.match - a.mismatch <= 255;
}

__device__ EndCell dp_dispatch(const PoaArgs& a, const Graph& g, const int* order, int ndp, const uint8_t* seq, int L,
                           int lane, int4* ring) {
    if (fast_dp(a, L)) {
        if (layer_fits_s16(a, ndp, L)) {
            switch (seg_cells(L + 1)) {
                case 4: return dp_layer_fast<4, true>(a, g, order, ndp, seq, L, lane, ring);
                case 8: return dp_layer_fast<8, true>(a, g, order, ndp, seq, L, lane, ring);
                case 12: return dp_layer_fast<12, true>(a, g, order, ndp, seq, L, lane, ring);
                case 16: return dp_layer_fast<16, true>(a, g, order, ndp, seq, L, lane, ring);
                case 20: return dp_layer_fast<20, true>(a, g, order, ndp, seq, L, lane, ring);
                default: return dp_layer_fast<24, true>(a, g, order, ndp, seq, L, lane, ring);
            }
        }
        switch (seg_cells(L + 1)) {
            case 4: return dp_layer_fast<4, false>(a, g, order, ndp, seq, L, lane, ring);
            case 8: return dp_layer_fast<8, false>(a, g, order, ndp, seq, L, lane, ring);
            case 12: return dp_layer_fast<12, false>(a, g, order, ndp, seq, L, lane, ring);
            case 16: return dp_layer_fast<16, false>(a, g, order, ndp, seq, L, lane, ring);
            case 20: return dp_layer_fast<20, false>(a, g, order, ndp, seq, L, lane, ring);
            default: return dp_layer_fast<24, false>(a, g, order, ndp, seq, L, lane, ring);
        }
    }
    return dp_layer<24>(a, g, order, ndp, seq, L, lane);
}

// Walk back from (iend, L) over the decision bytes (lane 0). Writes the
// sequence-consuming steps of the alignment (node id or -1 for an inserted
// base, sequence position), end of path first; vertical steps (a graph node
// against a gap) consume no position and add nothing to the graph. Each step
// loads the cell's decision byte and its row's descriptor (independent
// loads); the next row comes from the descriptor. Used for the byte
// decisions of the chunked dp_layer (rows over 768 columns).
__device__ bool traceback(const PoaArgs& a, const Graph& g, PoaShared& sh, const int* order, const uint8_t* seq,
                          int L, int iend) {
    const int lc = g.lcap;
    int i = iend, j = L, n = 0;
    if (iend == INT_MAX || iend < 1) return false;
    while (!(i == 0 && j == 0)) {
        if (n >= g.alncap) return false;
        if (i == 0) {
            g.aln_node[n] = -1;
            g.aln_pos[n] = j - 1;
            ++n;
            --j;
            continue;
        }
        const int4 d = g.rowdesc[i - 1];
        const int v = order[i - 1];
        const int np = desc_np(d.w);
        uint32_t code = g.dec[dec_at(i, j, lc)];
        if (code == 255u) {  // decide again from H: diagonal, then vertical, preds in order
            const int h = g.H[i * lc + j];
            const int s = j > 0 ? (uint32_t(seq[j - 1]) == desc_base(d.w) ? a.match : a.mismatch) : 0;
            const int cnt = np == 0 ? 1 : np;
            code = 128u;
            int pick = -1;
            if (cnt <= 3) {
                // all candidate values loaded at once (independent loads)
                int hd[3], hvv[3];
#pragma unroll
                for (int p = 0; p < 3; ++p) {
                    const int r = p < cnt ? desc_pred(g, d, p) : 0;
                    hd[p] = (p < cnt && j > 0) ? g.H[r * lc + j - 1] : kNegInf;
                    hvv[p] = p < cnt ? g.H[r * lc + j] : kNegInf;
                }
#pragma unroll
                for (int p = 2; p >= 0; --p)
                    if (j > 0 && hd[p] + s == h) pick = p;
                if (pick >= 0) {
                    code = 1000u + uint32_t(pick);
                } else {
#pragma unroll
                    for (int p = 2; p >= 0; --p)
                        if (hvv[p] + a.gap == h) pick = p;
                    if (pick >= 0) code = 2000u + uint32_t(pick);
                }
            } else {
                if (j > 0)
                    for (int p = 0; p < cnt && pick < 0; ++p)
                        if (g.H[desc_pred(g, d, p) * lc + j - 1] + s == h) pick = p;
                if (pick >= 0) {
                    code = 1000u + uint32_t(pick);
                } else {
                    for (int p = 0; p < cnt && pick < 0; ++p)
                        if (g.H[desc_pred(g, d, p) * lc + j] + a.gap == h) pick = p;
                    if (pick >= 0) code = 2000u + uint32_t(pick);
                }
            }
        }
        if (code < 64u || (code >= 1000u && code < 2000u)) {
            const int p = code < 64u ? int(code) : int(code - 1000u);
            g.aln_node[n] = v;
            g.aln_pos[n] = j - 1;
            ++n;
            i = desc_pred(g, d, p);
            --j;
        } else if (code < 128u || code >= 2000u) {
            const int p = code < 128u ? int(code - 64u) : int(code - 2000u);
            i = desc_pred(g, d, p);  // vertical: no sequence position
        } else {
            if (j == 0) return false;
            g.aln_node[n] = -1;
            g.aln_pos[n] = j - 1;
            ++n;
            --j;
        }
    }
    sh.naln = n;
    return true;
}

// ---------------- compact adjacency in shared memory ----------------

// In-edge sources and aligned nodes of every node as uint16 CSR lists in a
// warp's shared memory, in the graph's own list order (in-edges by edge id,
// aligned entries by slot: both are append-only), plus one flag byte per
// node. The DFS steps then read shared memory instead of chasing linked
// lists through global memory.
struct SmemCsr {
    uint16_t* in_off;  // [N + 1]
    uint16_t* al_off;  // [N + 1]
    uint16_t* in_src;  // [E]
    uint16_t* al_x;    // [A]
    uint8_t* flag;     // [N]: mark (bits 0-1), primary (bit 2), member (bit 3)
};

__device__ __forceinline__ size_t csr_bytes(int N, int E, int A) {
    return 2 * (size_t(N) + 1) * 2 + 2 * size_t(E) + 2 * size_t(A) + size_t(N);
}

// Builds the lists (warp). Returns false, building nothing, when the graph
// does not fit in `cap` bytes or 16-bit indices.
__device__ bool build_csr(const Graph& g, const PoaShared& sh, int lane, void* smem, int cap, SmemCsr& c) {
    const int N = sh.nnodes, E = sh.nedges, A = sh.naligned;
    if (N >= 65535 || E >= 65535 || A >= 65535 || csr_bytes(N, E, A) > size_t(cap)) return false;
    uint16_t* base = reinterpret_cast<uint16_t*>(smem);
    c.in_off = base;
    c.al_off = base + (N + 1);
    c.in_src = base + 2 * (N + 1);
    c.al_x = c.in_src + E;
    c.flag = reinterpret_cast<uint8_t*>(c.al_x + A);
    // starts: exclusive prefix of the counts
    // (graph-array loads are issued four 32-element chunks at a time)
    int bi = 0, ba = 0;
    for (int c4 = 0; c4 < N; c4 += 128) {
        int ci[4], ca[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int v = c4 + 32 * u + lane;
            ci[u] = v < N ? g.in_cnt[v] : 0;
            ca[u] = v < N ? g.al_cnt[v] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int v = c4 + 32 * u + lane;
            int ti = 0, ta = 0;
            const int xi = warp_excl(ci[u], lane, ti);
            const int xa = warp_excl(ca[u], lane, ta);
            if (v < N) {
                c.in_off[v] = uint16_t(bi + xi);
                c.al_off[v] = uint16_t(ba + xa);
            }
            bi += ti;
            ba += ta;
        }
    }
    if (lane == 0) {
        c.in_off[N] = uint16_t(E);
        c.al_off[N] = uint16_t(A);
    }
    __syncwarp();
    // stable fill by owner: the offsets serve as cursors and end up at the
    // next node's start
    const unsigned below = (1u << lane) - 1u;
    for (int c4 = 0; c4 < E; c4 += 128) {
        int ds[4], ss[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = c4 + 32 * u + lane;
            ds[u] = e < E ? g.e_dst[e] : -1 - lane;
            ss[u] = e < E ? g.e_src[e] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int dst = ds[u];
            const unsigned grp = __match_any_sync(0xffffffffu, dst);
            const int cur = dst >= 0 ? c.in_off[dst] : 0;
            __syncwarp();
            if (dst >= 0) {
                c.in_src[cur + __popc(grp & below)] = uint16_t(ss[u]);
                if ((grp & below) == 0) c.in_off[dst] = uint16_t(cur + __popc(grp));
            }
            __syncwarp();
        }
    }
    for (int c4 = 0; c4 < A; c4 += 128) {
        int os[4], ys[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = c4 + 32 * u + lane;
            os[u] = x < A ? g.a_owner[x] : -1 - lane;
            ys[u] = x < A ? g.a_node[x] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int own = os[u];
            const unsigned grp = __match_any_sync(0xffffffffu, own);
            const int cur = own >= 0 ? c.al_off[own] : 0;
            __syncwarp();
            if (own >= 0) {
                c.al_x[cur + __popc(grp & below)] = uint16_t(ys[u]);
                if ((grp & below) == 0) c.al_off[own] = uint16_t(cur + __popc(grp));
            }
            __syncwarp();
        }
    }
    // shift the cursors back to starts (off[v] = end of v - 1), top chunk first
    for (int c0 = ((N - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
        const int v = c0 + lane;
        uint16_t pi = 0, pa = 0;
        if (v < N && v > 0) {
            pi = c.in_off[v - 1];
            pa = c.al_off[v - 1];
        }
        __syncwarp();
        if (v < N) {
            c.in_off[v] = pi;
            c.al_off[v] = pa;
        }
        __syncwarp();
    }
    return true;
}

// g_topo_sort over the shared-memory lists (lane 0; flags initialised by the
// caller: mark 0, primary set, member bit for the nodes taking part).
__device__ int g_topo_sort_csr(const Graph& g, const SmemCsr& c, int N, bool all_nodes, int* out) {
    int nr = 0;
    int sp = 0;
    auto member = [&](int x) { return all_nodes || (c.flag[x] & 8); };
    auto mark = [&](int x) { return c.flag[x] & 3; };
    auto set_mark = [&](int x, int m) { c.flag[x] = uint8_t((c.flag[x] & ~3) | m); };
    for (int i = 0; i < N; ++i) {
        if (!member(i) || mark(i) != 0) continue;
        g.stack[sp++] = i;
        while (sp > 0) {
            const int v = g.stack[sp - 1];
            bool valid = true;
            if (mark(v) != 2) {
                for (int q = c.in_off[v], qe = c.in_off[v + 1]; q < qe; ++q) {
                    const int u = c.in_src[q];
                    if (!member(u)) continue;
                    if (mark(u) != 2) {
                        if (sp >= g.scap) return -1;
                        g.stack[sp++] = u;
                        valid = false;
                    }
                }
                if (c.flag[v] & 4) {
                    for (int q = c.al_off[v], qe = c.al_off[v + 1]; q < qe; ++q) {
                        const int y = c.al_x[q];
                        if (!member(y)) continue;
                        if (mark(y) != 2) {
                            if (sp >= g.scap) return -1;
                            g.stack[sp++] = y;
                            c.flag[y] &= uint8_t(~4);
                            valid = false;
                        }
                    }
                }
                if (valid) {
                    set_mark(v, 2);
                    if (c.flag[v] & 4) {
                        out[nr++] = v;
                        for (int q = c.al_off[v], qe = c.al_off[v + 1]; q < qe; ++q) {
                            const int y = c.al_x[q];
                            if (!member(y)) continue;
                            out[nr++] = y;
                        }
                    }
                } else {
                    set_mark(v, 1);
                }
            }
            if (valid) --sp;
        }
    }
    return nr;
}

// spoa's topological order of the graph (all_nodes) or of the member nodes,
// into out; shared-memory lists when they fit in the warp's ring, else the
// global-memory walk. Warp-collective; the count is returned on every lane
// (-1 on stack overflow).
__device__ int topo_sort_warp(const Graph& g, PoaShared& sh, bool all_nodes, int* out, int lane, int4* ring) {
    const int N = sh.nnodes;
    SmemCsr c;
    int nr = 0;
    if (build_csr(g, sh, lane, ring, kRingBytesPerWarp, c)) {
        for (int i = lane; i < N; i += 32) c.flag[i] = uint8_t(4 | (all_nodes || g.member[i] ? 8 : 0));
        __syncwarp();
        if (lane == 0) nr = g_topo_sort_csr(g, c, N, all_nodes, out);
    } else {
        for (int i = lane; i < N; i += 32) {
            g.mark[i] = 0;
            g.prim[i] = 1;
        }
        __syncwarp();
        if (lane == 0) nr = g_topo_sort(g, sh, all_nodes, out);
    }
    return __shfl_sync(0xffffffffu, nr, 0);
}

// spoa's subgraph node set (g_mark_subgraph) into g.member, over the
// shared-memory lists when they fit. Warp-collective; false on stack
// overflow (on every lane).
__device__ bool mark_subgraph_warp(const Graph& g, PoaShared& sh, int begin_node, int end_node, int lane, int4* ring) {
    const int N = sh.nnodes;
    if (end_node < 0 || end_node >= N) {
        if (lane == 0) sh.fail = kFailed;
        __syncwarp();
        return true;
    }
    SmemCsr c;
    bool ok = true;
    if (build_csr(g, sh, lane, ring, kRingBytesPerWarp, c)) {
        for (int i = lane; i < N; i += 32) c.flag[i] = 0;
        __syncwarp();
        if (lane == 0) {
            int sp = 0;
            g.stack[sp++] = end_node;
            while (sp > 0 && ok) {
                const int v = g.stack[--sp];
                if (!(c.flag[v] & 8) && v >= begin_node) {
                    for (int q = c.in_off[v], qe = c.in_off[v + 1]; q < qe; ++q) {
                        if (sp >= g.scap) {
                            ok = false;
                            break;
                        }
                        g.stack[sp++] = c.in_src[q];
                    }
                    for (int q = c.al_off[v], qe = c.al_off[v + 1]; q < qe && ok; ++q) {
                        if (sp >= g.scap) {
                            ok = false;
                            break;
                        }
                        g.stack[sp++] = c.al_x[q];
                    }
                    c.flag[v] |= 8;
                }
            }
        }
        __syncwarp();
        for (int i = lane; i < N; i += 32) g.member[i] = (c.flag[i] & 8) ? 1 : 0;
    } else if (lane == 0) {
        ok = g_mark_subgraph(g, sh, begin_node, end_node);
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
}

// Row descriptors with shared-memory accumulators (the ring is free until the
// DP): node ranks as uint16 (bit 15 marks a node with a successor row) and,
// per row, the first three predecessor ranks and the count. Loads of graph
// arrays are issued four 32-element chunks at a time, so one memory latency
// covers 128 edges or rows. Same order rules as the global form below.
// Returns false, building nothing, when the graph does not fit.
__device__ bool descriptors_smem(const Graph& g, const PoaShared& sh, const int* order, int N, int ndp, int lane,
                                 int4* ring) {
    constexpr unsigned kFull = 0xffffffffu;
    const size_t rk_bytes = size_t((N + 3) / 4) * 8;
    if (ndp >= 32768 || sh.nseq >= 65535 || rk_bytes + size_t(8) * ndp > size_t(kRingBytesPerWarp)) return false;
    uint16_t* const rk = reinterpret_cast<uint16_t*>(ring);
    ushort4* const acc = reinterpret_cast<ushort4*>(reinterpret_cast<uint8_t*>(ring) + rk_bytes);
    for (int i = lane; i < N; i += 32) rk[i] = 0;
    for (int i = lane; i < ndp; i += 32) acc[i] = make_ushort4(0, 0, 0, 0);
    __syncwarp();
    for (int c0 = 0; c0 < ndp; c0 += 128) {
        int v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = c0 + 32 * u + lane;
            v[u] = i < ndp ? order[i] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (v[u] >= 0) rk[v[u]] = uint16_t(c0 + 32 * u + lane + 1);
    }
    __syncwarp();
    const int E = sh.nedges;
    const unsigned below = (1u << lane) - 1u;
    bool any_long = false;
    for (int c0 = 0; c0 < E; c0 += 128) {
        int es[4], ed[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = c0 + 32 * u + lane;
            es[u] = e < E ? g.e_src[e] : -1;
            ed[u] = e < E ? g.e_dst[e] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int src = es[u], dst = ed[u];
            int rs = 0, rd = 0;
            if (src >= 0) {
                rs = rk[src] & 0x7FFF;
                rd = rs > 0 ? rk[dst] & 0x7FFF : 0;
            }
            const bool q = rs > 0 && rd > 0;
            const unsigned grp = __match_any_sync(kFull, q ? rd : -1 - lane);
            int cnt = 0;
            if (q) cnt = acc[rd - 1].w;
            __syncwarp();
            if (q) {
                rk[src] = uint16_t(rs | 0x8000);  // every writer stores the same value
                const int pos = cnt + __popc(grp & below);
                uint16_t* a4 = reinterpret_cast<uint16_t*>(&acc[rd - 1]);
                if (pos < 3) a4[pos] = uint16_t(rs);
                if ((grp & below) == 0) {
                    const int tot = cnt + __popc(grp);
                    a4[3] = uint16_t(tot);
                    any_long |= tot > 3;
                }
            }
            __syncwarp();
        }
    }
    any_long = __any_sync(kFull, any_long);
    int list_base = 0;
    for (int c0 = 0; c0 < ndp; c0 += 128) {
        int v[4], code[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = c0 + 32 * u + lane;
            v[u] = i < ndp ? order[i] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) code[u] = c0 + 32 * u + lane < ndp ? g.code[v[u]] : 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (c0 + 32 * u >= ndp) break;
            const int i = c0 + 32 * u + lane;
            const ushort4 dd = i < ndp ? acc[i] : make_ushort4(0, 0, 0, 0);
            const int np = dd.w;
            int off = 0;
            if (any_long) {
                int tot = 0;
                const int cntl = (i < ndp && np > 3) ? np : 0;
                off = list_base + warp_excl(cntl, lane, tot);
                list_base += tot;
                if (cntl) g.bpred[v[u]] = off;  // list cursor of the node
            }
            if (i < ndp) {
                const bool sink = (rk[v[u]] & 0x8000) == 0;
                g.sink[i] = sink ? 1 : 0;
                // long rows: x = list offset, y = first predecessor
                g.rowdesc[i] = make_int4(np > 3 ? off : dd.x, np > 3 ? dd.x : dd.y, dd.z,
                                         int(uint32_t(np) | (uint32_t(sink) << 17) | (uint32_t(code[u]) << 24)));
            }
        }
    }
    __syncwarp();
    if (any_long) {
        for (int c0 = 0; c0 < E; c0 += 32) {
            const int e = c0 + lane;
            int rs = 0, dst = 0;
            bool q = false;
            if (e < E) {
                dst = g.e_dst[e];
                const int rd = rk[dst] & 0x7FFF;
                if (rd > 0 && acc[rd - 1].w > 3) {
                    rs = rk[g.e_src[e]] & 0x7FFF;
                    q = rs > 0;
                }
            }
            const unsigned grp = __match_any_sync(kFull, q ? dst : -1 - lane);
            int cur = 0;
            if (q) cur = g.bpred[dst];
            __syncwarp();
            if (q) {
                g.pred_idx[cur + __popc(grp & below)] = rs;
                if ((grp & below) == 0) g.bpred[dst] = cur + __popc(grp);
            }
            __syncwarp();
        }
    }
    __syncwarp();
    return true;
}

// Heaviest bundle (g_heaviest_bundle) with the scores in shared memory: per
// node an int32 score and a uint16 predecessor, and for each chunk of 32 ranks
// the in-edges (source, weight) staged by the lanes in parallel, so the
// serial pass of lane 0 touches no global memory. Scores are bounded by
// sequences x 186 x nodes (two Phred values per sequence and edge, summed
// along a path), checked against int32. When branch completion is needed, or
// the graph does not fit, the global form finishes or does the work.
// Warp-collective; returns the path length (-1 on failure) on every lane.
__device__ int heaviest_bundle_warp(const Graph& g, PoaShared& sh, int lane, int4* ring) {
    constexpr int D = 8;  // staged in-edges per node
    const int N = sh.nnodes, R = sh.nranks;
    uint8_t* base = reinterpret_cast<uint8_t*>(ring);
    int* const bs = reinterpret_cast<int*>(base);                             // [N]
    uint16_t* const bp = reinterpret_cast<uint16_t*>(base + 4 * size_t(N));   // [N], 0xFFFF = none
    const size_t st_off = (6 * size_t(N) + 15) & ~size_t(15);
    int* const sw = reinterpret_cast<int*>(base + st_off);                    // [32][D] weights
    uint16_t* const su = reinterpret_cast<uint16_t*>(sw + 32 * D);            // [32][D] sources
    int* const sv = reinterpret_cast<int*>(su + 32 * D);                      // [32] node
    int* const sd = sv + 32;                                                  // [32] degree, D + 1 = more
    const size_t need = st_off + 32 * D * 6 + 32 * 8;
    const bool fits = N < 65535 && need <= size_t(kRingBytesPerWarp) &&
                      double(sh.nseq + 1) * 186.0 * double(N + 1) < 2.0e9;
    if (!fits) {
        int len = 0;
        if (lane == 0) len = g_heaviest_bundle(g, sh);
        return __shfl_sync(0xffffffffu, len, 0);
    }
    for (int i = lane; i < N; i += 32) {
        bs[i] = -1;
        bp[i] = 0xFFFF;
    }
    __syncwarp();
    int best_id = 0;
    for (int r0 = 0; r0 < R; r0 += 32) {
        const int r = r0 + lane;
        if (r < R) {
            const int v = g.rank_to_node[r];
            int deg = 0;
            for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) {
                if (deg == D) {
                    deg = D + 1;
                    break;
                }
                su[lane * D + deg] = uint16_t(g.e_src[e]);
                sw[lane * D + deg] = g.e_w[e];
                ++deg;
            }
            sv[lane] = v;
            sd[lane] = deg;
        }
        __syncwarp();
        if (lane == 0) {
            const int cnt = min(32, R - r0);
            for (int t = 0; t < cnt; ++t) {
                const int v = sv[t];
                const int deg = sd[t];
                int sv_ = bs[v], pv_ = bp[v] == 0xFFFF ? -1 : int(bp[v]);
                auto consider = [&](int u, int w) {
                    if (sv_ < w || (sv_ == w && pv_ != -1 && bs[pv_] <= bs[u])) {
                        sv_ = w;
                        pv_ = u;
                    }
                };
                if (deg <= D) {
                    for (int q = 0; q < deg; ++q) consider(su[t * D + q], sw[t * D + q]);
                } else {
                    for (int e = g.in_head[v]; e != -1; e = g.e_next_in[e]) consider(g.e_src[e], g.e_w[e]);
                }
                if (pv_ != -1) sv_ += bs[pv_];
                bs[v] = sv_;
                bp[v] = pv_ < 0 ? uint16_t(0xFFFF) : uint16_t(pv_);
                if (bs[best_id] < sv_) best_id = v;
            }
        }
        __syncwarp();
    }
    best_id = __shfl_sync(0xffffffffu, best_id, 0);
    const bool complete = g.out_head[best_id] != -1;
    if (complete) {
        // branch completion works on the global arrays
        for (int i = lane; i < N; i += 32) {
            g.bscore[i] = bs[i];
            g.bpred[i] = bp[i] == 0xFFFF ? -1 : int(bp[i]);
        }
        __syncwarp();
        int len = 0;
        if (lane == 0) {
            for (int r = 0; r < R; ++r) g.node_rank[g.rank_to_node[r]] = r;
            int guard = 0;
            len = 1;
            while (g.out_head[best_id] != -1) {
                best_id = g_branch_completion(g, sh, g.node_rank[best_id]);
                if (++guard > N + 1) {
                    len = -1;
                    break;
                }
            }
            if (len > 0) {
                len = 0;
                while (g.bpred[best_id] != -1) {
                    g.cons[len++] = best_id;
                    best_id = g.bpred[best_id];
                    if (len > N) {
                        len = -1;
                        break;
                    }
                }
                if (len >= 0) g.cons[len++] = best_id;
            }
            for (int i = 0, j = len - 1; i < j; ++i, --j) {
                const int t = g.cons[i];
                g.cons[i] = g.cons[j];
                g.cons[j] = t;
            }
        }
        return __shfl_sync(0xffffffffu, len, 0);
    }
    int len = 0;
    if (lane == 0) {
        int v = best_id;
        while (bp[v] != 0xFFFF) {
            g.cons[len++] = v;
            v = bp[v];
            if (len > N) {
                len = -1;
                break;
            }
        }
        if (len >= 0) {
            g.cons[len++] = v;
            for (int i = 0, j = len - 1; i < j; ++i, --j) {
                const int t = g.cons[i];
                g.cons[i] = g.cons[j];
                g.cons[j] = t;
            }
        }
    }
    return __shfl_sync(0xffffffffu, len, 0);
}

// Escape decision from H for a row of several predecessors (warp, uniform
// arguments): the first predecessor whose diagonal gives H[i][j],
// else the first whose vertical does, else horizontal. Returns 1000 + p,
// 2000 + p or 128. Lanes load the candidates of 32 predecessors at a time.
__device__ uint32_t decide_from_h(const PoaArgs& a, const Graph& g, const int4& d, const uint8_t* seq, int i, int j,
                                  int lane, bool h16) {
    const int np = desc_np(d.w);
    const int h = h_at(g, i, j, h16);
    const int s = j > 0 ? (uint32_t(seq[j - 1]) == desc_base(d.w) ? a.match : a.mismatch) : 0;
    const int cnt = np == 0 ? 1 : np;
    int vpick = -1;
    for (int p0 = 0; p0 < cnt; p0 += 32) {
        const int p = p0 + lane;
        bool dm = false, vm = false;
        if (p < cnt) {
            const int r = desc_pred(g, d, p);
            dm = j > 0 && h_at(g, r, j - 1, h16) + s == h;
            vm = h_at(g, r, j, h16) + a.gap == h;
        }
        const unsigned bd = __ballot_sync(0xffffffffu, dm);
        if (bd) return 1000u + uint32_t(p0 + __ffs(bd) - 1);
        const unsigned bv = __ballot_sync(0xffffffffu, vm);
        if (bv && vpick < 0) vpick = p0 + __ffs(bv) - 1;
    }
    return vpick >= 0 ? 2000u + uint32_t(vpick) : 128u;
}

// Warp form of the walk over dp_layer_fast's bit-plane decisions. The walk is
// a chain of dependent steps through nearby rows and columns, so the warp
// stages a window in shared memory with one parallel load: descriptors,
// node ids and the decision words of rows [wlo, wlo + 64) in column segments
// wseg and wseg - 1. Every lane then runs the same walk over the window
// (uniform control flow); lane 0 writes the alignment. A step that leaves
// the window reloads it. Decoding: horizontal plane, else the diagonal of
// predecessor 0; rows of one predecessor are otherwise vertical through it,
// rows of several decide again from H. Returns false on a broken walk.
__device__ bool traceback_warp(const PoaArgs& a, const Graph& g, PoaShared& sh, const int* order, const uint8_t* seq,
                               int L, int iend, int lane, int4* ring, bool h16) {
    constexpr int W = 64;
    const int S = seg_cells(L + 1);
    int4* const w_desc = ring;                                           // [W]
    int* const w_node = reinterpret_cast<int*>(ring + W);               // [W]
    uint2* const w_bits = reinterpret_cast<uint2*>(ring + W + W / 4);   // [2][W]
    const uint2* const D2 = reinterpret_cast<const uint2*>(g.dec);
    int i = iend, j = L, n = 0;
    if (iend == INT_MAX || iend < 1) return false;
    int seg = L / S, k = L % S;
    int wlo = INT_MAX, wseg = -1;
    bool ok = true;
    auto step_left = [&]() {
        --j;
        if (k == 0) {
            k = S - 1;
            --seg;
        } else {
            --k;
        }
    };
    while (!(i == 0 && j == 0)) {
        if (n >= g.alncap) {
            ok = false;
            break;
        }
        if (i == 0) {
            if (lane == 0) {
                g.aln_node[n] = -1;
                g.aln_pos[n] = j - 1;
            }
            ++n;
            step_left();
            continue;
        }
        if (i < wlo || seg < wseg - 1 || seg > wseg) {
            // stage rows [i - 63, i] (clamped at 1) for segments seg, seg - 1
            __syncwarp();
            wlo = max(1, i - (W - 1));
            wseg = seg;
#pragma unroll
            for (int h = 0; h < W / 32; ++h) {
                const int o = h * 32 + lane;
                const int r = wlo + o;
                if (r <= i) {
                    w_desc[o] = g.rowdesc[r - 1];
                    w_node[o] = order[r - 1];
                    w_bits[o] = D2[bits_at(r, seg)];
                    w_bits[W + o] = seg > 0 ? D2[bits_at(r, seg - 1)] : make_uint2(0, 0);

                }
            }
            __syncwarp();
        }
        const int o = i - wlo;
        const int4 d = w_desc[o];
        const int v = w_node[o];
        const uint2 w = w_bits[(seg == wseg ? 0 : W) + o];
        const int np = desc_np(d.w);
        uint32_t code;
        if ((w.x >> k) & 1u) {
            code = 128u;
        } else if ((w.y >> k) & 1u) {
            code = 0u;  // diagonal through predecessor 0
        } else if (np <= 1) {
            code = 64u;  // vertical through the only predecessor
        } else {
            code = decide_from_h(a, g, d, seq, i, j, lane, h16);
        }
        if (code < 64u || (code >= 1000u && code < 2000u)) {
            const int p = code < 64u ? int(code) : int(code - 1000u);
            if (lane == 0) {
                g.aln_node[n] = v;
                g.aln_pos[n] = j - 1;
            }
            ++n;
            i = desc_pred(g, d, p);
            step_left();
        } else if (code < 128u || code >= 2000u) {
            const int p = code < 128u ? int(code - 64u) : int(code - 2000u);
            i = desc_pred(g, d, p);  // vertical: no sequence position
        } else {
            if (j == 0) {
                ok = false;
                break;
            }
            if (lane == 0) {
                g.aln_node[n] = -1;
                g.aln_pos[n] = j - 1;
            }
            ++n;
            step_left();
        }
    }
    __syncwarp();
    if (lane == 0) sh.naln = n;
    return ok;
}

// ---------------- one window (one warp) ----------------

__device__ void poa_window(const PoaArgs& a, const Graph& g, PoaShared& sh, uint32_t wi, int lane, int4* ring) {
    const PoaWinDev W = a.wins[wi];
    const uint8_t* bb = a.in + W.bb_off;
    const uint8_t* bq = W.bq_off == kNoQual ? nullptr : a.in + W.bq_off;
    uint8_t* outp = reinterpret_cast<uint8_t*>(a.out) + W.out_off;
    const int B = int(W.bb_len);
    if (W.n_layers < 2) {
        for (int i = lane; i < B; i += 32) outp[i] = bb[i];
        if (lane == 0) {
            a.out_len[wi] = uint32_t(B);
            a.flags[wi] = 0;
        }
        return;
    }
    if (B > g.ncap) {
        if (lane == 0) {
            a.flags[wi] = kOverflow;
            a.out_len[wi] = 0;
        }
        return;
    }
    // backbone: chain of B nodes, edge weights from quality (0 with the dummy)
    for (int i = lane; i < B; i += 32) {
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
        g.ord[i] = i;
        g.my_rank[i] = i;
        g.in_cnt[i] = i > 0 ? 1 : 0;
        g.al_cnt[i] = 0;
        g.out_cnt[i] = i + 1 < B ? 1 : 0;
    }
    if (lane == 0) {
        sh.nnodes = B;
        sh.nedges = B - 1;
        sh.naligned = 0;
        sh.nseq = 1;
        sh.nranks = B;
        sh.fail = 0;
    }
    __syncwarp();
    unsigned long long cells = 0, edge_cells = 0;

    for (uint32_t li = 0; li < W.n_layers; ++li) {
        const PoaLayerDev Lr = a.layers[W.layer_base + li];
        const uint8_t* seq = a.in + Lr.seq_off;
        const uint8_t* qual = Lr.qual_off == kNoQual ? nullptr : a.in + Lr.qual_off;
        const int L = int(Lr.len);
        const bool full = Lr.begin < W.offset && Lr.end > uint32_t(B) - W.offset;
        const int N = sh.nnodes;
        for (int i = lane; i < N; i += 32) {
            g.member[i] = full ? 1 : 0;
        }
        __syncwarp();
        if (!full && !mark_subgraph_warp(g, sh, int(Lr.begin), int(Lr.end), lane, ring) && lane == 0)
            sh.fail = kOverflow;
        __syncwarp();
        if (lane == 0 && !sh.fail && row_cover(L + 1) > g.lcap) sh.fail = kOverflow;
        __syncwarp();
        if (sh.fail) break;
        // DP rows: the incremental order, restricted to the subgraph for a
        // partial layer (any topological order gives the same DP values)
        int ndp = N;
        const int* order = g.ord;
        if (!full) {
            // compaction of the member nodes in order; the loads of four
            // 32-entry chunks go out together
            int base = 0;
            for (int c4 = 0; c4 < N; c4 += 128) {
                int vv[4];
                bool in[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = c4 + 32 * u + lane;
                    vv[u] = r < N ? g.ord[r] : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) in[u] = c4 + 32 * u + lane < N && g.member[vv[u]];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const unsigned m = __ballot_sync(0xffffffffu, in[u]);
                    if (in[u]) g.dporder[base + __popc(m & ((1u << lane) - 1u))] = vv[u];
                    base += __popc(m);
                }
            }
            ndp = base;
            order = g.dporder;
            __syncwarp();
        }
        // Row descriptors: shared-memory accumulators when the graph fits,
        // else the global form below.
        if (!descriptors_smem(g, sh, order, N, ndp, lane, ring)) {
            // Row descriptors. DP ranks of the nodes live in shared memory (the
            // row ring is free until the DP) when they fit, else in global
            // scratch; bit 31 marks a node with a successor among the rows.
            int* const dpr = N <= kSmemRanks ? reinterpret_cast<int*>(ring) : g.dprank;
            for (int i = lane; i < N; i += 32) dpr[i] = 0;
            __syncwarp();
            for (int i = lane; i < ndp; i += 32) dpr[order[i]] = i + 1;
            __syncwarp();
            // Predecessors by one pass over the edges in id order. A node's
            // in-edge list is in edge-id order (each layer adds at most one edge
            // into a node, with a fresh, larger id), which is spoa's predecessor
            // order. Lanes take 32 consecutive edges; edges into the same row
            // are ranked by lane, so the order is deterministic. rowdesc[r - 1]
            // collects the first three predecessor ranks (x, y, z) and the count
            // (w) of row r; bit 31 of dpr marks a node with a successor row.
            for (int i = lane; i < ndp; i += 32) g.rowdesc[i] = make_int4(0, 0, 0, 0);
            __syncwarp();
            const int E = sh.nedges;
            const unsigned below = (1u << lane) - 1u;
            bool any_long = false;
            for (int c0 = 0; c0 < E; c0 += 32) {
                const int e = c0 + lane;
                int rs = 0, rd = 0, src = 0;
                if (e < E) {
                    src = g.e_src[e];
                    const int dst = g.e_dst[e];
                    rs = dpr[src] & 0x7FFFFFFF;
                    rd = rs > 0 ? dpr[dst] & 0x7FFFFFFF : 0;
                }
                const bool q = rs > 0 && rd > 0;
                const unsigned grp = __match_any_sync(0xffffffffu, q ? rd : -1 - lane);
                int cnt = 0;
                if (q) {
                    atomicOr(reinterpret_cast<unsigned*>(&dpr[src]), 0x80000000u);
                    cnt = g.rowdesc[rd - 1].w;
                }
                __syncwarp();
                if (q) {
                    const int pos = cnt + __popc(grp & below);
                    int* rdw = reinterpret_cast<int*>(&g.rowdesc[rd - 1]);
                    if (pos < 3) rdw[pos] = rs;
                    if ((grp & below) == 0) {
                        const int tot = cnt + __popc(grp);
                        rdw[3] = tot;
                        any_long |= tot > 3;
                    }
                }
                __syncwarp();
            }
            any_long = __any_sync(0xffffffffu, any_long);
            // final descriptors; rows with more than three predecessors get their
            // full list in pred_idx at an offset from a warp prefix of the counts
            int list_base = 0;
            for (int c0 = 0; c0 < ndp; c0 += 32) {
                const int i = c0 + lane;
                int4 dd = i < ndp ? g.rowdesc[i] : make_int4(0, 0, 0, 0);
                const int v = i < ndp ? order[i] : 0;
                int off = 0;
                if (any_long) {
                    int tot = 0;
                    const int cntl = (i < ndp && dd.w > 3) ? dd.w : 0;
                    off = list_base + warp_excl(cntl, lane, tot);
                    list_base += tot;
                    if (cntl) g.bpred[v] = off;  // list cursor of the node
                }
                if (i < ndp) {
                    const bool sink = (dpr[v] & 0x80000000) == 0;
                    g.sink[i] = sink ? 1 : 0;
                    // long rows: x = list offset, y = first predecessor
                    g.rowdesc[i] = make_int4(dd.w > 3 ? off : dd.x, dd.w > 3 ? dd.x : dd.y, dd.z,
                                             int(uint32_t(dd.w) | (uint32_t(sink) << 17) | (uint32_t(g.code[v]) << 24)));
                }
            }
            __syncwarp();
            if (any_long) {
                // second pass over the edges for the long lists, same ranking
                for (int c0 = 0; c0 < E; c0 += 32) {
                    const int e = c0 + lane;
                    int rs = 0, dst = 0;
                    bool q = false;
                    if (e < E) {
                        dst = g.e_dst[e];
                        const int rd = dpr[dst] & 0x7FFFFFFF;
                        if (rd > 0 && desc_np(g.rowdesc[rd - 1].w) > 3) {
                            rs = dpr[g.e_src[e]] & 0x7FFFFFFF;
                            q = rs > 0;
                        }
                    }
                    const unsigned grp = __match_any_sync(0xffffffffu, q ? dst : -1 - lane);
                    int cur = 0;
                    if (q) cur = g.bpred[dst];
                    __syncwarp();
                    if (q) {
                        g.pred_idx[cur + __popc(grp & below)] = rs;
                        if ((grp & below) == 0) g.bpred[dst] = cur + __popc(grp);
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
        }
        const EndCell ec = dp_dispatch(a, g, order, ndp, seq, L, lane, ring);
        cells += (unsigned long long)ndp * (unsigned long long)L;
        edge_cells += (unsigned long long)(ndp + ec.preds) * (unsigned long long)L;
        int iend = ec.row;
        if (ec.ties > 1) {
            // several sinks share the best last-column value: spoa takes the
            // first in its own topological order of the aligned (sub)graph.
            // A sink outside every aligned group is reached by spoa's DFS
            // only as a root (no member lists it as an in-edge tail, and
            // aligned links are symmetric), so such sinks are ranked by node
            // id; only a tie that involves an aligned sink needs the DFS.
            int low_id = INT_MAX, low_i = iend;
            bool grouped = false;
            for (int i = 1 + lane; i <= ndp; i += 32) {
                if (!g.sink[i - 1] || g.lastH[i] != ec.value) continue;
                const int v = order[i - 1];
                grouped |= g.al_cnt[v] != 0;
                if (v < low_id) {
                    low_id = v;
                    low_i = i;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const int ov = __shfl_xor_sync(0xffffffffu, low_id, o);
                const int oi = __shfl_xor_sync(0xffffffffu, low_i, o);
                if (ov < low_id) {
                    low_id = ov;
                    low_i = oi;
                }
            }
            grouped = __any_sync(0xffffffffu, grouped);
            const int nr = grouped ? topo_sort_warp(g, sh, full, g.rank_to_node, lane, ring) : 0;
            if (!grouped) {
                iend = low_i;
            } else if (nr < 0) {
                if (lane == 0) sh.fail = kOverflow;
            } else {
                for (int r = lane; r < nr; r += 32) g.node_rank[g.rank_to_node[r]] = r;
                __syncwarp();
                // the tied sink of lowest rank (ranks are distinct)
                int best = INT_MAX, bi = iend;
                for (int i = 1 + lane; i <= ndp; i += 32) {
                    if (!g.sink[i - 1] || g.lastH[i] != ec.value) continue;
                    const int rr = g.node_rank[order[i - 1]];
                    if (rr < best) {
                        best = rr;
                        bi = i;
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const int ob = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ob < best) {
                        best = ob;
                        bi = oi;
                    }
                }
                iend = bi;
            }
            __syncwarp();
        }
        if (fast_dp(a, L)) {
            if (!sh.fail && !traceback_warp(a, g, sh, order, seq, L, iend, lane, ring, ec.h16) && lane == 0)
                sh.fail = kFailed;
        } else if (lane == 0 && !sh.fail && !traceback(a, g, sh, order, seq, L, iend)) {
            sh.fail = kFailed;
        }
        __syncwarp();
        if (sh.fail) break;
        add_alignment_warp(g, sh, seq, qual, L, lane, ring);
        if (sh.fail) break;
        order_insert(g, sh, N, lane, ring);
    }
    // spoa's topological order of the final graph for the consensus
    if (!sh.fail) {
        const int nr = topo_sort_warp(g, sh, true, g.rank_to_node, lane, ring);
        if (lane == 0) {
            if (nr < 0) sh.fail = kOverflow;
            sh.nranks = nr;
        }
        __syncwarp();
    }
    if (lane == 0 && cells) {
        atomicAdd(a.cells, cells);
        atomicAdd(a.cells + 1, edge_cells);
    }
    if (sh.fail) {
        if (lane == 0) {
            a.flags[wi] = uint8_t(sh.fail);
            a.out_len[wi] = 0;
        }
        return;
    }
    // ---- consensus ----
    const int N = sh.nnodes;
    for (int i = lane; i < N; i += 32) {
        g.bscore[i] = -1;
        g.bpred[i] = -1;
    }
    __syncwarp();
    const int hb_len = heaviest_bundle_warp(g, sh, lane, ring);
    if (lane == 0) {
        const int len = hb_len;
        uint8_t flags = kPolished;
        if (len < 0) {
            flags = kFailed;
            a.out_len[wi] = 0;
        } else {
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
    __syncwarp();
}

constexpr int kWarpsPerCta = 4;
// resident CTAs per SM the register budget is sized for
constexpr int kCtasPerSm = 3;

__global__ void __launch_bounds__(32 * kWarpsPerCta, kCtasPerSm) poa_kernel(PoaArgs a) {
    __shared__ PoaShared sh_all[kWarpsPerCta];
    // the per-warp view of its scratch slot lives in shared memory so the
    // ~35 array pointers are not held in registers across the DP
    __shared__ Graph g_all[kWarpsPerCta];
    extern __shared__ int4 ring_all[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int4* ring = ring_all + wid * (kRingBytesPerWarp / 16);
    PoaShared& sh = sh_all[wid];
    const uint32_t slot = blockIdx.x * kWarpsPerCta + wid;
    if (lane == 0) g_all[wid] = make_graph(a, slot);
    __syncwarp();
    const Graph& g = g_all[wid];
    // with a cap the CTA retires after that many windows per warp, so other
    // streams' kernels get SMs between launches (the host launches enough)
    for (uint32_t done = 0; a.per_warp_cap == 0 || done < a.per_warp_cap; ++done) {
        unsigned k = 0;
        if (lane == 0) k = atomicAdd(&a.counters[0], 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= a.nwin) break;
        poa_window(a, g, sh, a.order[k], lane, ring);
    }
}

// Plain comparison form: one window per one-warp block, block b takes window
// order[b] with scratch slot b, one launch per batch, no work queue. Same
// per-window code as poa_kernel, so results are identical.
__global__ void __launch_bounds__(32 * kWarpsPerCta, kCtasPerSm) poa_plain_kernel(PoaArgs a) {
    __shared__ PoaShared sh;
    __shared__ Graph g;
    extern __shared__ int4 ring_all[];
    const int lane = threadIdx.x & 31;
    if (blockIdx.x >= a.nwin) return;
    if (lane == 0) g = make_graph(a, blockIdx.x);
    __syncwarp();
    poa_window(a, g, sh, a.order[blockIdx.x], lane, ring_all);
}

// ---------------- shared queue (serving) ----------------

// The consensus service's kernel arguments: scoring, capacities and scratch
// slots, the batch records, and the queue.
struct PoaSvcArgs {
    PoaArgs base;
    const PoaJobDev* jobs;
    SvcQueueDev q;
};

// Persistent consensus over the shared queue: each warp owns one scratch
// slot and takes windows of any job until the queue stays empty. Sized for
// at most kSvcCtasPerSm resident CTAs per SM, so that the rest of each SM
// stays free for the alignment and layer kernels of newly admitted jobs.
constexpr int kSvcCtasPerSm = 3;
__global__ void __launch_bounds__(32 * kWarpsPerCta, kSvcCtasPerSm) poa_service_kernel(PoaSvcArgs s) {
    __shared__ PoaShared sh_all[kWarpsPerCta];
    __shared__ Graph g_all[kWarpsPerCta];
    __shared__ PoaArgs a_all[kWarpsPerCta];
    extern __shared__ int4 ring_all[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int4* ring = ring_all + wid * (kRingBytesPerWarp / 16);
    PoaShared& sh = sh_all[wid];
    const uint32_t slot = blockIdx.x * kWarpsPerCta + wid;
    if (lane == 0) g_all[wid] = make_graph(s.base, slot);
    __syncwarp();
    for (;;) {
        unsigned long long it = 0;
        if (lane == 0) it = svc_claim(s.q, slot);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it == ~0ull) break;
        const uint32_t job = uint32_t(it >> 32), win = uint32_t(it);
        uint32_t total = 0, gen = 0;
        if (lane == 0) {
            // the record is rewritten for every batch that reuses the slot:
            // read it past L1
            const volatile PoaJobDev& J = s.jobs[job];
            PoaArgs a = s.base;
            a.in = const_cast<const uint8_t*>(J.in);
            a.wins = const_cast<const PoaWinDev*>(J.wins);
            a.layers = const_cast<const PoaLayerDev*>(J.layers);
            a.out = const_cast<char*>(J.out);
            a.out_len = const_cast<uint32_t*>(J.out_len);
            a.flags = const_cast<uint8_t*>(J.flags);
            a.trim = J.trim;
            a.cells = const_cast<unsigned long long*>(J.cells);
            total = J.head.total;
            gen = J.head.generation;
            a.nwin = total;
            a_all[wid] = a;
        }
        __syncwarp();
        poa_window(a_all[wid], g_all[wid], sh, win, lane, ring);
        __threadfence();
        __syncwarp();
        if (lane == 0) svc_item_done(s.q, job, total, gen);
    }
}

}  // namespace

size_t PoaEngine::slot_bytes_for(uint32_t max_layer_length) {
    const int ncap = 4096;
    return walk_layout(ncap, 2 * ncap, ncap, row_cover(int(max_layer_length) + 1), [](int, size_t) {});
}

PoaEngine::PoaEngine(const DeviceInfo& dev, cudaStream_t stream, int8_t m, int8_t x, int8_t g)
    : dev_(dev), stream_(stream), match_(m), mismatch_(x), gap_(g) {
    check_cuda(cudaEventCreate(&ev0_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev2_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev3_), "cudaEventCreate");
    prefer_max_shared(reinterpret_cast<const void*>(poa_kernel));
    prefer_max_shared(reinterpret_cast<const void*>(poa_plain_kernel));
}

PoaEngine::~PoaEngine() {
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
    cudaEventDestroy(ev2_);
    cudaEventDestroy(ev3_);
}

// Phred+33 bytes '!'..'~': the window graph weights are quality - 33 in
// 0..93 (spoa's uint32 weights of other bytes are not modelled).
static bool phred_bytes(const char* q, uint32_t n) {
    uint8_t bad = 0;
    for (uint32_t k = 0; k < n; ++k) bad |= uint8_t(uint8_t(q[k] - 33) > 93);
    return bad == 0;
}

void PoaEngine::stage(const rb_window* wins, size_t n, int trim) {
    if (n > 0 && !wins) throw Error{RB_ERR_ARG, "rb_poa: windows is NULL"};
    forget();
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
            if (!phred_bytes(w.backbone_quality, w.backbone_length))
                throw Error{RB_ERR_ARG, "rb_poa: quality values outside '!'..'~' (Phred+33 0..93)"};
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
                if (!phred_bytes(q, l))
                    throw Error{RB_ERR_ARG, "rb_poa: quality values outside '!'..'~' (Phred+33 0..93)"};
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
    in_ptr_ = d_in_.as<uint8_t>();
    layers_ptr_ = d_layers_.as<PoaLayerDev>();
    nwin_ = n;
}

void PoaEngine::stage_device(const uint8_t* d_in, const PoaWinDev* wins, size_t n, const PoaLayerDev* d_layers,
                             const uint64_t* sum_len, const std::vector<std::pair<uint64_t, uint32_t>>& labels,
                             uint32_t max_len, int trim) {
    forget();
    trim_ = trim;
    max_len_ = max_len;
    uint64_t out_cap = 0;
    uint32_t max_nodes = 0;
    for (size_t i = 0; i < n; ++i) {
        out_cap = std::max<uint64_t>(out_cap, wins[i].out_off + wins[i].out_cap);
        max_nodes = uint32_t(std::max<uint64_t>(max_nodes, std::min<uint64_t>(wins[i].bb_len + sum_len[i], 1u << 20)));
    }
    out_cap_ = out_cap;
    max_nodes_cap_ = max_nodes;
    labels_.assign(labels.begin(), labels.begin() + n);
    h_desc_.reserve(std::max<size_t>(n, 1) * sizeof(PoaWinDev));
    h_order_.reserve(std::max<size_t>(n, 1) * sizeof(uint32_t));
    PoaWinDev* wd = h_desc_.as<PoaWinDev>();
    if (n) memcpy(wd, wins, n * sizeof(PoaWinDev));
    // size-sorted queue, the same work estimate as stage()
    uint32_t* order = h_order_.as<uint32_t>();
    std::iota(order, order + n, 0u);
    std::vector<uint64_t> work(n);
    for (size_t i = 0; i < n; ++i) {
        const uint64_t s = sum_len[i];
        work[i] = s * (wd[i].bb_len + s / std::max<uint32_t>(1, wd[i].n_layers));
    }
    std::sort(order, order + n, [&](uint32_t x, uint32_t y) { return work[x] != work[y] ? work[x] > work[y] : x < y; });
    d_desc_.reserve(std::max<size_t>(n, 1) * sizeof(PoaWinDev));
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (n)
        check_cuda(cudaMemcpyAsync(d_desc_.ptr, wd, n * sizeof(PoaWinDev), cudaMemcpyHostToDevice, stream_),
                   "H2D desc");
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "stage sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.h2d_ms = ms;
    stats_.h2d_bytes = n * sizeof(PoaWinDev);
    in_bytes_ = 0;
    in_ptr_ = d_in;
    layers_ptr_ = d_layers;
    nwin_ = n;
}

void PoaEngine::forget() {
    nwin_ = 0;
    in_ptr_ = nullptr;
    layers_ptr_ = nullptr;
}

void PoaEngine::prepare_outputs() {
    const size_t n = nwin_;
    stats_.launches = 0;
    stats_.items = n;
    stats_.cells = 0;
    stats_.edge_cells = 0;
    stats_.kernel_ms = 0;
    stats_.top_kernel_ms = 0;
    if (n == 0) return;
    d_out_.reserve(std::max<uint64_t>(out_cap_, 16));
    d_outlen_.reserve(n * 4);
    d_flags_.reserve(n);
    d_misc_.reserve(64);
}

void PoaEngine::run(bool plain) {
    prepare_outputs();
    const size_t n = nwin_;
    if (n == 0) return;
    std::vector<uint32_t> todo(n);
    const uint32_t* h_order = h_order_.as<uint32_t>();
    // batched form: size-sorted queue (heaviest first, or size buckets
    // interleaved by the device's tuning); plain form: input order
    const rb_tuning tune = tuning_get(dev_.device);
    for (size_t i = 0; i < n; ++i) todo[i] = plain ? uint32_t(i) : h_order[i];
    if (!plain && tune.consensus_order == 1)
        for (size_t i = 0, lo = 0, hi = n; i < n; ++i) todo[i] = h_order[(i & 1) ? --hi : lo++];
    // starting graph capacity; windows that outgrow it run again with four
    // times as much. RB_POA_NCAP lowers the start (tests of the retry path);
    // results do not depend on it.
    int ncap = 4096;
    if (const char* e = getenv("RB_POA_NCAP")) ncap = std::max(256, std::min(4096, atoi(e)));
    run_list(std::move(todo), ncap, plain);
}

void PoaEngine::run_list(std::vector<uint32_t> todo, int ncap, bool plain) {
    const size_t n = nwin_;
    std::vector<uint8_t> flags(n);
    float total_ms = 0;
    // DP row width: every layer's columns rounded up to whole warp passes
    const uint32_t* lens_max = &max_len_;
    const int lcap = row_cover(int(*lens_max) + 1);
    while (!todo.empty()) {
        const int ecap = 2 * ncap, acap = ncap;
        const size_t slot = walk_layout(ncap, ecap, acap, lcap, [](int, size_t) {});
        // resident windows (one warp each): enough to fill the SMs, bounded by
        // a scratch budget
        const size_t budget = scratch_budget_;
        // resident windows: the device's tuned CTAs per SM on the context's
        // share of the SMs (all by default)
        const uint32_t cps = std::min<uint32_t>(kCtasPerSm, tuning_get(dev_.device).consensus_ctas_per_sm);
        const size_t resident = std::max<size_t>(
            kWarpsPerCta, size_t(dev_.sm_count) * kWarpsPerCta * cps * sm_share_pct_ / 100);
        size_t slots = std::min<size_t>(todo.size(), plain ? todo.size() : resident);
        // RB_POA_SLOTS caps the resident windows (smaller scratch, e.g. for
        // profiler captures); results do not depend on it
        if (const char* e = getenv("RB_POA_SLOTS"))
            slots = std::max<size_t>(1, std::min<size_t>(slots, strtoull(e, nullptr, 10)));
        while (slots > 1 && slots * slot > budget) slots /= 2;
        if (!plain) slots = (slots + kWarpsPerCta - 1) / kWarpsPerCta * kWarpsPerCta;
        d_graph_.reserve(slots * slot);
        DevBuf& d_todo = d_dp_;
        d_todo.reserve(todo.size() * 4);
        check_cuda(cudaMemcpyAsync(d_todo.ptr, todo.data(), todo.size() * 4, cudaMemcpyHostToDevice, stream_),
                   "H2D todo");
        PoaArgs a;
        memset(&a, 0, sizeof(a));
        a.in = in_ptr_;
        a.wins = d_desc_.as<PoaWinDev>();
        a.layers = layers_ptr_;
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
        check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset counters");
        check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
        if (plain) {
            // one launch per batch of `slots` windows
            check_cuda(cudaFuncSetAttribute(poa_plain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            kRingBytesPerWarp),
                       "cudaFuncSetAttribute");
            for (size_t b0 = 0; b0 < todo.size(); b0 += slots) {
                PoaArgs ab = a;
                ab.order = a.order + b0;
                ab.nwin = uint32_t(std::min(slots, todo.size() - b0));
                poa_plain_kernel<<<int(ab.nwin), 32, kRingBytesPerWarp, stream_>>>(ab);
                ++stats_.launches;
            }
        } else {
            const int smem = kWarpsPerCta * kRingBytesPerWarp;
            check_cuda(cudaFuncSetAttribute(poa_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                       "cudaFuncSetAttribute");
            // persistent by default; with a per-warp cap, enough launches
            // back to back that every window is taken
            size_t launches = 1;
            if (yield_windows_ > 0) {
                a.per_warp_cap = yield_windows_;
                launches = (todo.size() + slots * yield_windows_ - 1) / (slots * yield_windows_);
            }
            for (size_t l = 0; l < launches; ++l) {
                poa_kernel<<<int(slots / kWarpsPerCta), 32 * kWarpsPerCta, smem, stream_>>>(a);
                ++stats_.launches;
            }
        }
        check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
        unsigned long long cells[2] = {0, 0};
        check_cuda(cudaMemcpyAsync(cells, a.cells, 16, cudaMemcpyDeviceToHost, stream_), "D2H cells");
        check_cuda(cudaMemcpyAsync(flags.data(), d_flags_.ptr, n, cudaMemcpyDeviceToHost, stream_), "D2H flags");
        check_cuda(cudaStreamSynchronize(stream_), "poa sync");
        check_cuda(cudaGetLastError(), "poa kernel");
        float ms = 0;
        cudaEventElapsedTime(&ms, ev0_, ev1_);
        total_ms += ms;
        stats_.cells += cells[0];
        stats_.edge_cells += cells[1];
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
    stats_.kernel_ms += total_ms;
    stats_.top_kernel_ms += total_ms;
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

// ---------------------------------------------------------------------------
// Shared window-consensus service (continuous batching for the serving loop)

namespace rb {

struct PoaSvcState {
    explicit PoaSvcState(int device) : ring(device, sizeof(PoaJobDev), "rb_poa service") {}
    RingService ring;
    void* d_scratch = nullptr;  // one graph slot per resident warp
    PoaSvcArgs args{};
    uint32_t slots = 0, grid = 0;
};

namespace {
cudaError_t launch_poa_service(cudaStream_t stream, void* user) {
    const PoaSvcState* S = static_cast<const PoaSvcState*>(user);
    poa_service_kernel<<<S->grid, 32 * kWarpsPerCta, kWarpsPerCta * kRingBytesPerWarp, stream>>>(S->args);
    return cudaGetLastError();
}
}  // namespace

PoaService::PoaService(int device, int8_t m, int8_t x, int8_t g, uint32_t window_length, size_t scratch_budget,
                       uint32_t ctas_per_sm, uint32_t large_first_every)
    : st_(nullptr) {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    int sm_count = 148;
    check_cuda(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device), "sm count");
    std::unique_ptr<PoaSvcState> S(new PoaSvcState(device));
    // slot layout for layers up to three window lengths; longer ones (and
    // graphs over 4096 nodes) overflow and run again in the job's own engine
    const int ncap = 4096, ecap = 2 * ncap, acap = ncap;
    const int lcap = row_cover(int(std::max<uint32_t>(window_length, 1)) * 3 + 1);
    const size_t slot = walk_layout(ncap, ecap, acap, lcap, [](int, size_t) {});
    const uint32_t cps = std::max<uint32_t>(1, std::min<uint32_t>(ctas_per_sm, kSvcCtasPerSm));
    size_t slots = size_t(sm_count) * cps * kWarpsPerCta;
    while (slots > kWarpsPerCta && slots * slot > scratch_budget) slots -= kWarpsPerCta;
    S->slots = uint32_t(slots);
    S->grid = uint32_t(slots / kWarpsPerCta);
    check_cuda(cudaMalloc(&S->d_scratch, slots * slot), "cudaMalloc service scratch");
    PoaSvcArgs& A = S->args;
    memset(&A, 0, sizeof(A));
    A.base.scratch = static_cast<uint8_t*>(S->d_scratch);
    A.base.slot_bytes = slot;
    A.base.ncap = ncap;
    A.base.ecap = ecap;
    A.base.acap = acap;
    A.base.lcap = lcap;
    A.base.match = m;
    A.base.mismatch = x;
    A.base.gap = g;
    S->ring.set_large_first_every(large_first_every);
    A.jobs = static_cast<const PoaJobDev*>(S->ring.records());
    A.q = S->ring.queue();
    check_cuda(cudaFuncSetAttribute(poa_service_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    kWarpsPerCta * kRingBytesPerWarp),
               "cudaFuncSetAttribute");
    prefer_max_shared(reinterpret_cast<const void*>(poa_service_kernel));
    st_ = S.release();
    st_->ring.start(launch_poa_service, st_);
}

PoaService::~PoaService() {
    st_->ring.stop();
    cudaFree(st_->d_scratch);
    delete st_;
}

uint32_t PoaService::slots() const { return st_->slots; }
uint32_t PoaService::launches() const { return st_->ring.launches(); }

void PoaService::run_batch(const PoaJobDev& job, const uint32_t* order, size_t n, int queue) {
    st_->ring.run_batch(&job, order, n, queue);
}

void PoaEngine::run_shared(PoaService& svc, uint32_t priority_windows) {
    prepare_outputs();
    const size_t n = nwin_;
    if (n == 0) return;
    check_cuda(cudaMemsetAsync(d_misc_.ptr, 0, 64, stream_), "memset counters");
    // the batch's inputs and descriptors are complete on this engine's stream
    check_cuda(cudaStreamSynchronize(stream_), "poa stage sync");
    PoaJobDev job;
    memset(&job, 0, sizeof(job));
    job.in = in_ptr_;
    job.wins = d_desc_.as<PoaWinDev>();
    job.layers = layers_ptr_;
    job.out = d_out_.as<char>();
    job.out_len = d_outlen_.as<uint32_t>();
    job.flags = d_flags_.as<uint8_t>();
    job.cells = reinterpret_cast<unsigned long long*>(d_misc_.as<unsigned int>() + 8);
    job.trim = trim_;
    const auto t0 = std::chrono::steady_clock::now();
    // size class: ring 0 up to priority_windows windows, then x4 per ring
    const uint64_t p = std::max<uint32_t>(1, priority_windows);
    const int queue = n <= p ? 0 : n <= 4 * p ? 1 : n <= 16 * p ? 2 : 3;
    svc.run_batch(job, h_order_.as<uint32_t>(), n, queue);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::vector<uint8_t> flags(n);
    unsigned long long cells[2] = {0, 0};
    check_cuda(cudaMemcpyAsync(flags.data(), d_flags_.ptr, n, cudaMemcpyDeviceToHost, stream_), "D2H flags");
    check_cuda(cudaMemcpyAsync(cells, job.cells, 16, cudaMemcpyDeviceToHost, stream_), "D2H cells");
    check_cuda(cudaStreamSynchronize(stream_), "poa sync");
    stats_.cells = cells[0];
    stats_.edge_cells = cells[1];
    stats_.kernel_ms = ms;
    stats_.top_kernel_ms = ms;
    std::vector<uint32_t> again;
    for (uint32_t w = 0; w < n; ++w) {
        if (flags[w] & kFailed) throw Error{RB_ERR_DEVICE, "rb_poa: window consensus failed on the device"};
        if (flags[w] & kOverflow) again.push_back(w);
    }
    // windows that outgrew the shared slots: this engine's own launch with
    // four times the graph capacity (the same path a private run takes)
    if (!again.empty()) run_list(std::move(again), 4 * 4096, false);
}

}  // namespace rb
