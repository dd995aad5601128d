// ORACLE — test infrastructure only. C entry points of the CPU restatement,
// loaded with ctypes by tests/ and bench.py (CPU baseline); never by the
// product library.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "edlib_nw.hpp"
#include "racon_cpu.hpp"

using namespace oracle;

extern "C" {

// NW edit distance only (test/racon_test.cpp:16-25 metric).
int oracle_nw_distance(const char* q, int qlen, const char* t, int tlen) {
    return nw_align(q, qlen, t, tlen, false).edit_distance;
}

// NW with path (src/overlap.cpp:205-224). Writes the standard CIGAR into
// cigar[0..cap) (NUL-terminated when it fits) and its length to *cigar_len.
// Returns the edit distance, or -1 on failure.
int oracle_nw_cigar(const char* q, int qlen, const char* t, int tlen, char* cigar,
                    int cap, int* cigar_len) {
    NwResult r = nw_align(q, qlen, t, tlen, true);
    if (!r.ok) return -1;
    const std::string c = ops_to_cigar(r.ops);
    *cigar_len = int(c.size());
    if (int(c.size()) < cap) memcpy(cigar, c.c_str(), c.size() + 1);
    return r.edit_distance;
}

// Breaking points from a CIGAR (src/overlap.cpp:226-292); writes
// (t,q) pairs as 2*count uint32 values; returns the number of values, or the
// negative required size when cap is too small.
int oracle_breakpoints(const char* cigar, uint32_t q_begin, uint32_t q_end,
                       uint32_t q_length, uint32_t t_begin, uint32_t t_end,
                       uint32_t strand, uint32_t window_length, uint32_t* out, int cap) {
    CpuOverlap o;
    o.cigar = cigar;
    o.q_begin = q_begin;
    o.q_end = q_end;
    o.q_length = q_length;
    o.t_begin = t_begin;
    o.t_end = t_end;
    o.strand = strand;
    std::vector<std::pair<uint32_t, uint32_t>> bp;
    breakpoints_from_cigar(o, window_length, bp);
    const int need = int(bp.size() * 2);
    if (need > cap) return -need;
    for (size_t i = 0; i < bp.size(); ++i) {
        out[2 * i] = bp[i].first;
        out[2 * i + 1] = bp[i].second;
    }
    return need;
}

// Window::generate_consensus (src/window.cpp:65-142) on one window. quals[i]
// may be NULL. Returns 1 when polished, 0 when the backbone was kept, -1 when
// cap is too small (out_len then holds the size needed).
int oracle_window_consensus(const char* backbone, const char* bqual, uint32_t blen,
                            uint32_t nlayers, const char* const* seqs,
                            const char* const* quals, const uint32_t* lens,
                            const uint32_t* begins, const uint32_t* ends, int tgs, int trim,
                            int match, int mismatch, int gap, char* out, int cap,
                            int* out_len, uint64_t* cells_out, uint32_t* nodes_out) {
    CpuWindowInput w;
    w.backbone = backbone;
    w.backbone_len = blen;
    w.backbone_qual = bqual;
    for (uint32_t i = 0; i < nlayers; ++i) {
        w.seqs.push_back(seqs[i]);
        w.quals.push_back(quals ? quals[i] : nullptr);
        w.lens.push_back(lens[i]);
        w.positions.emplace_back(begins[i], ends[i]);
    }
    std::string cons;
    WindowStats st;
    const bool pol = window_consensus(w, tgs != 0, trim != 0, match, mismatch, gap, cons, &st);
    if (cells_out) *cells_out = st.cells;
    if (nodes_out) *nodes_out = st.nodes;
    *out_len = int(cons.size());
    if (int(cons.size()) > cap) return -1;
    memcpy(out, cons.data(), cons.size());
    return pol ? 1 : 0;
}

// Full pipeline; returns a malloc'd FASTA text (free with oracle_free), or
// NULL where racon would exit(1). times[0..4] = load, align, layers,
// consensus seconds; counts[0..2] = overlaps, windows, poa cells.
char* oracle_polish(const char* sequences, const char* overlaps, const char* targets,
                    int fragment, uint32_t window_length, double quality_threshold,
                    double error_threshold, int trim, int match, int mismatch, int gap,
                    uint32_t threads, int drop_unpolished, double* times, uint64_t* counts) {
    PolishOptions opt;
    opt.fragment = fragment != 0;
    opt.window_length = window_length;
    opt.quality_threshold = quality_threshold;
    opt.error_threshold = error_threshold;
    opt.trim = trim != 0;
    opt.match = match;
    opt.mismatch = mismatch;
    opt.gap = gap;
    opt.threads = threads;
    opt.drop_unpolished = drop_unpolished != 0;
    std::vector<std::pair<std::string, std::string>> out;
    PolishTimes tm;
    if (polish_files(sequences, overlaps, targets, opt, out, &tm)) return nullptr;
    if (times) {
        times[0] = tm.load_s;
        times[1] = tm.align_s;
        times[2] = tm.layers_s;
        times[3] = tm.consensus_s;
    }
    if (counts) {
        counts[0] = tm.overlaps;
        counts[1] = tm.windows;
        counts[2] = tm.poa_cells;
    }
    std::string text;
    for (const auto& s : out) {
        text += '>';
        text += s.first;
        text += '\n';
        text += s.second;
        text += '\n';
    }
    char* buf = static_cast<char*>(malloc(text.size() + 1));
    memcpy(buf, text.c_str(), text.size() + 1);
    return buf;
}

void oracle_free(void* p) { free(p); }

}  // extern "C"

extern "C" {

// Every window after initialize() (src/polisher.cpp:192-460) as a binary blob
// (free with oracle_free). Layout, little endian, per window:
//   u64 target_id, u32 rank, u8 tgs, u32 backbone_len, u32 n_layers,
//   backbone bytes, backbone quality bytes,
//   per layer: u32 len, u32 begin, u32 end, u8 has_quality, bytes, [quality]
// preceded by a u64 window count. Returns NULL on error.
char* oracle_dump_windows(const char* sequences, const char* overlaps, const char* targets,
                          int fragment, uint32_t window_length, double quality_threshold,
                          double error_threshold, uint32_t threads, uint64_t* nbytes) {
    PolishOptions opt;
    opt.fragment = fragment != 0;
    opt.window_length = window_length;
    opt.quality_threshold = quality_threshold;
    opt.error_threshold = error_threshold;
    opt.threads = threads;
    std::vector<DumpedWindow> ws;
    if (collect_windows(sequences, overlaps, targets, opt, ws)) return nullptr;
    std::string b;
    auto put = [&](const void* p, size_t n) { b.append(static_cast<const char*>(p), n); };
    const uint64_t nw = ws.size();
    put(&nw, 8);
    for (const auto& w : ws) {
        const uint32_t bl = uint32_t(w.backbone.size()), nl = uint32_t(w.seqs.size());
        const uint8_t tgs = w.tgs ? 1 : 0;
        put(&w.target_id, 8);
        put(&w.rank, 4);
        put(&tgs, 1);
        put(&bl, 4);
        put(&nl, 4);
        put(w.backbone.data(), bl);
        put(w.backbone_qual.data(), bl);
        for (uint32_t i = 0; i < nl; ++i) {
            const uint32_t len = uint32_t(w.seqs[i].size());
            const uint8_t hq = w.quals[i].empty() ? 0 : 1;
            put(&len, 4);
            put(&w.positions[i].first, 4);
            put(&w.positions[i].second, 4);
            put(&hq, 1);
            put(w.seqs[i].data(), len);
            if (hq) put(w.quals[i].data(), len);
        }
    }
    char* out = static_cast<char*>(malloc(b.size()));
    memcpy(out, b.data(), b.size());
    *nbytes = b.size();
    return out;
}

// The inputs of racon's layer loop after initialize()'s breaking points
// (src/polisher.cpp:401-457), as a binary blob (free with oracle_free), for
// checking a restatement of that loop against the windows the oracle builds.
// Layout, little endian: u64 sequences, u64 targets, u8 tgs; per sequence
// four u32-length-prefixed strings (data, quality, reverse complement,
// reversed quality; empty when dropped or absent); u64 overlaps; per overlap
// u32 q_id, u32 t_id, u32 strand, u32 points, then (u32 t, u32 q) per point.
char* oracle_dump_layer_input(const char* sequences, const char* overlaps, const char* targets,
                              int fragment, uint32_t window_length, double quality_threshold,
                              double error_threshold, uint32_t threads, uint64_t* nbytes) {
    PolishOptions opt;
    opt.fragment = fragment != 0;
    opt.window_length = window_length;
    opt.quality_threshold = quality_threshold;
    opt.error_threshold = error_threshold;
    opt.threads = threads;
    std::vector<CpuSequence> seqs;
    std::vector<CpuOverlap> ovl;
    uint64_t targets_n = 0;
    bool tgs = true;
    if (collect_layer_input(sequences, overlaps, targets, opt, seqs, targets_n, tgs, ovl)) return nullptr;
    std::string b;
    auto put = [&](const void* p, size_t n) { b.append(static_cast<const char*>(p), n); };
    auto put_str = [&](const std::string& x) {
        const uint32_t n = uint32_t(x.size());
        put(&n, 4);
        put(x.data(), n);
    };
    const uint64_t ns = seqs.size();
    const uint8_t t8 = tgs ? 1 : 0;
    put(&ns, 8);
    put(&targets_n, 8);
    put(&t8, 1);
    for (const auto& q : seqs) {
        put_str(q.data);
        put_str(q.quality);
        put_str(q.rc);
        put_str(q.rquality);
    }
    const uint64_t no = ovl.size();
    put(&no, 8);
    for (const auto& o : ovl) {
        const uint32_t qid = uint32_t(o.q_id), tid = uint32_t(o.t_id), st = o.strand,
                       np = uint32_t(o.breaking_points.size());
        put(&qid, 4);
        put(&tid, 4);
        put(&st, 4);
        put(&np, 4);
        for (const auto& p : o.breaking_points) {
            put(&p.first, 4);
            put(&p.second, 4);
        }
    }
    char* out = static_cast<char*>(malloc(b.size()));
    memcpy(out, b.data(), b.size());
    *nbytes = b.size();
    return out;
}

}  // extern "C"

#include <atomic>
#include <chrono>
#include <thread>

extern "C" {

// Window consensus of the first max_windows windows of a blob in the
// oracle_dump_windows layout, on `threads` host threads. Returns the number of
// windows done; *seconds = wall time of the consensus loop, *cells = DP cells.
// Used as the CPU baseline (the oracle, not reference racon).
// Window consensus of up to max_windows windows of a blob in the
// oracle_dump_windows layout on `threads` threads. When `out` is given, the
// consensus of window i goes to out[offsets[i], offsets[i + 1]) (offsets has
// room for n + 1 entries, out for out_cap bytes) and polished[i] is its
// generate_consensus result; edge_cells (optional) gets the DP work counted
// as sum |layer| x sum_v (1 + indeg v).
int64_t oracle_consensus_blob_out(const char* blob, uint64_t nbytes, int64_t max_windows, uint32_t threads,
                                  int match, int mismatch, int gap, int trim, double* seconds,
                                  uint64_t* cells, uint64_t* edge_cells, char* out, uint64_t out_cap,
                                  uint64_t* offsets, uint8_t* polished) {
    uint64_t off = 0;
    auto get = [&](void* dst, size_t n) {
        if (off + n > nbytes) return false;
        memcpy(dst, blob + off, n);
        off += n;
        return true;
    };
    uint64_t nw = 0;
    if (!get(&nw, 8)) return -1;
    std::vector<CpuWindowInput> wins;
    std::vector<uint8_t> tgs;
    for (uint64_t i = 0; i < nw && int64_t(wins.size()) < max_windows; ++i) {
        uint64_t tid;
        uint32_t rank, bl, nl;
        uint8_t t;
        if (!get(&tid, 8) || !get(&rank, 4) || !get(&t, 1) || !get(&bl, 4) || !get(&nl, 4)) return -1;
        CpuWindowInput w;
        w.backbone = blob + off;
        w.backbone_len = bl;
        off += bl;
        w.backbone_qual = blob + off;
        off += bl;
        for (uint32_t k = 0; k < nl; ++k) {
            uint32_t len, b, e;
            uint8_t hq;
            if (!get(&len, 4) || !get(&b, 4) || !get(&e, 4) || !get(&hq, 1)) return -1;
            w.seqs.push_back(blob + off);
            off += len;
            w.quals.push_back(hq ? blob + off : nullptr);
            if (hq) off += len;
            w.lens.push_back(len);
            w.positions.emplace_back(b, e);
        }
        if (off > nbytes) return -1;
        wins.push_back(std::move(w));
        tgs.push_back(t);
    }
    std::vector<uint64_t> c(wins.size(), 0), ec(wins.size(), 0);
    std::vector<std::string> cons(out ? wins.size() : 0);
    std::vector<uint8_t> pol(wins.size(), 0);
    std::atomic<size_t> next(0);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (uint32_t k = 0; k < std::max<uint32_t>(1, threads); ++k) {
        pool.emplace_back([&]() {
            for (size_t i = next++; i < wins.size(); i = next++) {
                std::string cs;
                WindowStats st;
                pol[i] = window_consensus(wins[i], tgs[i] != 0, trim != 0, match, mismatch, gap, cs, &st);
                c[i] = st.cells;
                ec[i] = st.edge_cells;
                if (out) cons[i].swap(cs);
            }
        });
    }
    for (auto& th : pool) th.join();
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint64_t total = 0, etotal = 0;
    for (auto x : c) total += x;
    for (auto x : ec) etotal += x;
    *cells = total;
    if (edge_cells) *edge_cells = etotal;
    if (out) {
        uint64_t o = 0;
        for (size_t i = 0; i < wins.size(); ++i) {
            offsets[i] = o;
            if (o + cons[i].size() > out_cap) return -2;
            memcpy(out + o, cons[i].data(), cons[i].size());
            o += cons[i].size();
            polished[i] = pol[i];
        }
        offsets[wins.size()] = o;
    }
    return int64_t(wins.size());
}

int64_t oracle_consensus_blob(const char* blob, uint64_t nbytes, int64_t max_windows, uint32_t threads,
                              int match, int mismatch, int gap, int trim, double* seconds,
                              uint64_t* cells) {
    return oracle_consensus_blob_out(blob, nbytes, max_windows, threads, match, mismatch, gap, trim, seconds,
                                     cells, nullptr, nullptr, 0, nullptr, nullptr);
}

}  // extern "C"
