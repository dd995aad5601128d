// ORACLE — test infrastructure only (see racon_cpu.hpp).
#include "racon_cpu.hpp"

#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <unordered_map>

#include "edlib_nw.hpp"

namespace oracle {
namespace {

double now_s() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

void parallel_for(uint64_t n, uint32_t threads, const std::function<void(uint64_t)>& fn) {
    if (threads <= 1 || n < 2) {
        for (uint64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<uint64_t> next(0);
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t) {
        pool.emplace_back([&]() {
            for (uint64_t i = next++; i < n; i = next++) fn(i);
        });
    }
    for (auto& th : pool) th.join();
}

// Line reader over gzip or plain text.
class LineReader {
public:
    explicit LineReader(const std::string& path) { f_ = gzopen(path.c_str(), "rb"); }
    ~LineReader() {
        if (f_) gzclose(f_);
    }
    bool ok() const { return f_ != nullptr; }
    bool next(std::string& line) {
        line.clear();
        while (true) {
            if (pos_ >= len_) {
                len_ = gzread(f_, buf_, sizeof(buf_));
                pos_ = 0;
                if (len_ <= 0) return !line.empty();
            }
            char* nl = static_cast<char*>(memchr(buf_ + pos_, '\n', size_t(len_ - pos_)));
            if (nl) {
                line.append(buf_ + pos_, size_t(nl - (buf_ + pos_)));
                pos_ = int(nl - buf_) + 1;
                if (!line.empty() && line.back() == '\r') line.pop_back();
                return true;
            }
            line.append(buf_ + pos_, size_t(len_ - pos_));
            pos_ = len_;
        }
    }

private:
    gzFile f_ = nullptr;
    char buf_[1 << 16];
    int pos_ = 0, len_ = 0;
};

std::string first_word(const std::string& s, size_t from) {
    size_t e = from;
    while (e < s.size() && !isspace(uint8_t(s[e]))) ++e;
    return s.substr(from, e - from);
}

void append_bases(std::string& dst, const std::string& line) {
    for (char c : line)
        if (!isspace(uint8_t(c))) dst += c;
}

CpuSequence make_sequence(const std::string& name, const std::string& data,
                          const std::string* qual) {
    CpuSequence s;
    s.name = name;
    s.data.reserve(data.size());
    for (char c : data) s.data += char(toupper(uint8_t(c)));
    if (qual) {
        uint32_t sum = 0;
        for (char c : *qual) sum += uint32_t(c - '!');
        if (sum > 0) s.quality = *qual;
    }
    return s;
}

bool split_fields(const std::string& line, char sep, std::vector<std::string>& f) {
    f.clear();
    size_t b = 0;
    while (b <= line.size()) {
        size_t e = line.find(sep, b);
        if (e == std::string::npos) e = line.size();
        f.push_back(line.substr(b, e - b));
        b = e + 1;
    }
    return true;
}

bool read_overlaps(const std::string& path, int kind, std::vector<CpuOverlap>& out) {
    // kind: 0 mhap, 1 paf, 2 sam
    LineReader r(path);
    if (!r.ok()) return false;
    std::string line;
    std::vector<std::string> f;
    while (r.next(line)) {
        if (line.empty()) continue;
        CpuOverlap o;
        if (kind == 0) {
            // split on runs of whitespace
            f.clear();
            size_t i = 0;
            while (i < line.size()) {
                while (i < line.size() && isspace(uint8_t(line[i]))) ++i;
                size_t j = i;
                while (j < line.size() && !isspace(uint8_t(line[j]))) ++j;
                if (j > i) f.push_back(line.substr(i, j - i));
                i = j;
            }
            if (f.size() < 12) continue;
            const uint64_t a_id = std::strtoull(f[0].c_str(), nullptr, 10);
            const uint64_t b_id = std::strtoull(f[1].c_str(), nullptr, 10);
            o.q_id = a_id - 1;
            o.t_id = b_id - 1;
            const uint32_t a_rc = uint32_t(std::strtoul(f[4].c_str(), nullptr, 10));
            o.q_begin = uint32_t(std::strtoul(f[5].c_str(), nullptr, 10));
            o.q_end = uint32_t(std::strtoul(f[6].c_str(), nullptr, 10));
            o.q_length = uint32_t(std::strtoul(f[7].c_str(), nullptr, 10));
            const uint32_t b_rc = uint32_t(std::strtoul(f[8].c_str(), nullptr, 10));
            o.t_begin = uint32_t(std::strtoul(f[9].c_str(), nullptr, 10));
            o.t_end = uint32_t(std::strtoul(f[10].c_str(), nullptr, 10));
            o.t_length = uint32_t(std::strtoul(f[11].c_str(), nullptr, 10));
            o.strand = a_rc ^ b_rc;
            o.length = std::max(o.q_end - o.q_begin, o.t_end - o.t_begin);
            o.error = 1 - std::min(o.q_end - o.q_begin, o.t_end - o.t_begin) /
                              static_cast<double>(o.length);
        } else if (kind == 1) {
            split_fields(line, '\t', f);
            if (f.size() < 12) continue;
            o.q_name = f[0];
            o.q_length = uint32_t(std::strtoul(f[1].c_str(), nullptr, 10));
            o.q_begin = uint32_t(std::strtoul(f[2].c_str(), nullptr, 10));
            o.q_end = uint32_t(std::strtoul(f[3].c_str(), nullptr, 10));
            o.strand = f[4] == "-";
            o.t_name = f[5];
            o.t_length = uint32_t(std::strtoul(f[6].c_str(), nullptr, 10));
            o.t_begin = uint32_t(std::strtoul(f[7].c_str(), nullptr, 10));
            o.t_end = uint32_t(std::strtoul(f[8].c_str(), nullptr, 10));
            o.length = std::max(o.q_end - o.q_begin, o.t_end - o.t_begin);
            o.error = 1 - std::min(o.q_end - o.q_begin, o.t_end - o.t_begin) /
                              static_cast<double>(o.length);
        } else {
            if (line[0] == '@') continue;
            split_fields(line, '\t', f);
            if (f.size() < 11) continue;
            o.q_name = f[0];
            const uint32_t flag = uint32_t(std::strtoul(f[1].c_str(), nullptr, 10));
            o.t_name = f[2];
            o.t_begin = uint32_t(std::strtoul(f[3].c_str(), nullptr, 10)) - 1;
            o.cigar = f[5];
            o.strand = (flag & 0x10) ? 1 : 0;
            o.valid = !(flag & 0x4);
            o.q_begin = 0;
            o.q_length = 0;
            if (o.cigar.size() < 2 && o.valid) {
                fprintf(stderr, "[Racon::Overlap::Overlap] error: missing alignment from SAM object!\n");
                exit(1);
            }
            const std::string& cg = o.cigar;
            for (size_t i = 0; i < cg.size(); ++i) {
                if (cg[i] == 'S' || cg[i] == 'H') {
                    o.q_begin = uint32_t(atoi(&cg[0]));
                    break;
                } else if (cg[i] == 'M' || cg[i] == '=' || cg[i] == 'I' || cg[i] == 'D' ||
                           cg[i] == 'N' || cg[i] == 'P' || cg[i] == 'X') {
                    break;
                }
            }
            uint32_t qa = 0, qc = 0, ta = 0;
            for (size_t i = 0, j = 0; i < cg.size(); ++i) {
                const char c = cg[i];
                if (c == 'M' || c == '=' || c == 'X') {
                    const uint32_t nb = uint32_t(atoi(&cg[j]));
                    j = i + 1;
                    qa += nb;
                    ta += nb;
                } else if (c == 'I') {
                    qa += uint32_t(atoi(&cg[j]));
                    j = i + 1;
                } else if (c == 'D' || c == 'N') {
                    ta += uint32_t(atoi(&cg[j]));
                    j = i + 1;
                } else if (c == 'S' || c == 'H') {
                    qc += uint32_t(atoi(&cg[j]));
                    j = i + 1;
                } else if (c == 'P') {
                    j = i + 1;
                }
            }
            o.q_end = o.q_begin + qa;
            o.q_length = qc + qa;
            if (o.strand) {
                const uint32_t tmp = o.q_begin;
                o.q_begin = o.q_length - o.q_end;
                o.q_end = o.q_length - tmp;
            }
            o.t_end = o.t_begin + ta;
            o.length = std::max(qa, ta);
            o.error = 1 - std::min(qa, ta) / static_cast<double>(o.length);
        }
        out.push_back(std::move(o));
    }
    return true;
}

bool has_suffix(const std::string& s, const std::string& x) {
    return s.size() >= x.size() && s.compare(s.size() - x.size(), x.size(), x) == 0;
}

int seq_format(const std::string& p) {
    for (const char* x : {".fasta", ".fasta.gz", ".fna", ".fna.gz", ".fa", ".fa.gz"})
        if (has_suffix(p, x)) return 0;
    for (const char* x : {".fastq", ".fastq.gz", ".fq", ".fq.gz"})
        if (has_suffix(p, x)) return 1;
    return -1;
}

int ovl_format(const std::string& p) {
    if (has_suffix(p, ".mhap") || has_suffix(p, ".mhap.gz")) return 0;
    if (has_suffix(p, ".paf") || has_suffix(p, ".paf.gz")) return 1;
    if (has_suffix(p, ".sam") || has_suffix(p, ".sam.gz")) return 2;
    return -1;
}

void align_and_break(CpuOverlap& o, const std::vector<CpuSequence>& seqs, uint32_t w) {
    if (!o.transmuted) {
        fprintf(stderr, "[racon::Overlap::find_breaking_points] error: overlap is not transmuted!\n");
        exit(1);
    }
    if (!o.breaking_points.empty()) return;
    if (o.cigar.empty()) {
        const char* q = !o.strand ? &seqs[o.q_id].data[o.q_begin]
                                  : &seqs[o.q_id].rc[o.q_length - o.q_end];
        const char* t = &seqs[o.t_id].data[o.t_begin];
        NwResult r = nw_align(q, int(o.q_end - o.q_begin), t, int(o.t_end - o.t_begin), true);
        if (!r.ok) {
            fprintf(stderr, "[racon::Overlap::find_breaking_points] error: "
                            "edlib unable to align pair (%zu x %zu)!\n",
                    size_t(o.q_id), size_t(o.t_id));
            exit(1);
        }
        o.cigar = ops_to_cigar(r.ops);
    }
    breakpoints_from_cigar(o, w, o.breaking_points);
    std::string().swap(o.cigar);
}

struct Loaded {
    std::vector<CpuSequence> seqs;
    uint64_t targets = 0;
    bool tgs = true;
    std::vector<CpuOverlap> overlaps;
};

// initialize() up to (not including) breaking points; 0 ok, 1 error.
int load_inputs(const std::string& sp, const std::string& op, const std::string& tp,
                const PolishOptions& opt, Loaded& L) {
    if (opt.window_length == 0) {
        fprintf(stderr, "[racon::createPolisher] error: invalid window length!\n");
        return 1;
    }
    const int sf = seq_format(sp), of = ovl_format(op), tf = seq_format(tp);
    if (sf < 0) {
        fprintf(stderr, "[racon::createPolisher] error: file %s has unsupported format extension "
                        "(valid extensions: .fasta, .fasta.gz, .fna, .fna.gz, .fa, .fa.gz, .fastq, "
                        ".fastq.gz, .fq, .fq.gz)!\n", sp.c_str());
        return 1;
    }
    if (of < 0) {
        fprintf(stderr, "[racon::createPolisher] error: file %s has unsupported format extension "
                        "(valid extensions: .mhap, .mhap.gz, .paf, .paf.gz, .sam, .sam.gz)!\n",
                op.c_str());
        return 1;
    }
    if (tf < 0) {
        fprintf(stderr, "[racon::createPolisher] error: file %s has unsupported format extension "
                        "(valid extensions: .fasta, .fasta.gz, .fna, .fna.gz, .fa, .fa.gz, .fastq, "
                        ".fastq.gz, .fq, .fq.gz)!\n", tp.c_str());
        return 1;
    }
    auto& seqs = L.seqs;
    if (!read_sequences(tp, seqs)) return 1;
    const uint64_t T = seqs.size();
    L.targets = T;
    if (T == 0) {
        fprintf(stderr, "[racon::Polisher::initialize] error: empty target sequences set!\n");
        return 1;
    }
    std::unordered_map<std::string, uint64_t> name_to_id;
    std::unordered_map<uint64_t, uint64_t> id_to_id;
    for (uint64_t i = 0; i < T; ++i) {
        name_to_id[seqs[i].name + "t"] = i;
        id_to_id[i << 1 | 1] = i;
    }
    std::vector<CpuSequence> reads;
    if (!read_sequences(sp, reads)) return 1;
    uint64_t nreads = 0, total_len = 0;
    for (auto& r : reads) {
        total_len += r.data.size();
        auto it = name_to_id.find(r.name + "t");
        if (it != name_to_id.end()) {
            if (r.data.size() != seqs[it->second].data.size() ||
                r.quality.size() != seqs[it->second].quality.size()) {
                fprintf(stderr, "[racon::Polisher::initialize] error: duplicate sequence %s with unequal data\n",
                        r.name.c_str());
                return 1;
            }
            name_to_id[r.name + "q"] = it->second;
            id_to_id[nreads << 1 | 0] = it->second;
        } else {
            name_to_id[r.name + "q"] = seqs.size();
            id_to_id[nreads << 1 | 0] = seqs.size();
            seqs.push_back(std::move(r));
        }
        ++nreads;
    }
    if (nreads == 0) {
        fprintf(stderr, "[racon::Polisher::initialize] error: empty sequences set!\n");
        return 1;
    }
    L.tgs = !(static_cast<double>(total_len) / nreads <= 1000);

    std::vector<CpuOverlap> raw;
    if (!read_overlaps(op, of, raw)) return 1;
    // transmute
    std::vector<bool> alive(raw.size(), true);
    for (size_t i = 0; i < raw.size(); ++i) {
        CpuOverlap& o = raw[i];
        if (!o.valid || o.transmuted) {
            if (!o.valid) alive[i] = false;
            continue;
        }
        if (!o.q_name.empty()) {
            auto it = name_to_id.find(o.q_name + "q");
            if (it == name_to_id.end()) { o.valid = false; alive[i] = false; continue; }
            o.q_id = it->second;
        } else {
            auto it = id_to_id.find(o.q_id << 1 | 0);
            if (it == id_to_id.end()) { o.valid = false; alive[i] = false; continue; }
            o.q_id = it->second;
        }
        if (o.q_length != seqs[o.q_id].data.size()) {
            fprintf(stderr, "[racon::Overlap::transmute] error: unequal lengths in sequence and "
                            "overlap file for sequence %s!\n", seqs[o.q_id].name.c_str());
            return 1;
        }
        if (!o.t_name.empty()) {
            auto it = name_to_id.find(o.t_name + "t");
            if (it == name_to_id.end()) { o.valid = false; alive[i] = false; continue; }
            o.t_id = it->second;
        } else {
            auto it = id_to_id.find(o.t_id << 1 | 1);
            if (it == id_to_id.end()) { o.valid = false; alive[i] = false; continue; }
            o.t_id = it->second;
        }
        if (o.t_length != 0 && o.t_length != seqs[o.t_id].data.size()) {
            fprintf(stderr, "[racon::Overlap::transmute] error: unequal lengths in target and "
                            "overlap file for target %s!\n", seqs[o.t_id].name.c_str());
            return 1;
        }
        o.t_length = uint32_t(seqs[o.t_id].data.size());
        o.transmuted = true;
    }
    // filter per contiguous run of equal q_id (src/polisher.cpp:284-335)
    auto remove_invalid = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            if (!alive[i]) continue;
            if (raw[i].error > opt.error_threshold || raw[i].q_id == raw[i].t_id) {
                alive[i] = false;
                continue;
            }
            if (!opt.fragment) {
                for (size_t j = i + 1; j < e; ++j) {
                    if (!alive[j]) continue;
                    if (raw[i].length > raw[j].length) {
                        alive[j] = false;
                    } else {
                        alive[i] = false;
                        break;
                    }
                }
            }
        }
    };
    size_t c = 0;
    for (size_t i = 0; i < raw.size(); ++i) {
        if (!alive[i]) continue;
        while (!alive[c]) ++c;
        if (raw[c].q_id != raw[i].q_id) {
            remove_invalid(c, i);
            c = i;
        }
    }
    remove_invalid(c, raw.size());

    std::vector<bool> has_name(seqs.size(), false), has_data(seqs.size(), false),
        has_rev(seqs.size(), false);
    for (uint64_t i = 0; i < T; ++i) has_name[i] = has_data[i] = true;
    for (size_t i = 0; i < raw.size(); ++i) {
        if (!alive[i]) continue;
        if (raw[i].strand) has_rev[raw[i].q_id] = true;
        else has_data[raw[i].q_id] = true;
        L.overlaps.push_back(std::move(raw[i]));
    }
    if (L.overlaps.empty()) {
        fprintf(stderr, "[racon::Polisher::initialize] error: empty overlap set!\n");
        return 1;
    }
    for (size_t i = 0; i < seqs.size(); ++i) {
        if (!has_name[i]) std::string().swap(seqs[i].name);
        if (has_rev[i]) seqs[i].build_reverse();
        if (!has_data[i]) {
            std::string().swap(seqs[i].data);
            std::string().swap(seqs[i].quality);
        }
    }
    return 0;
}

struct Layered {
    std::vector<CpuWindowInput> windows;
    std::vector<uint64_t> window_target;
    std::vector<uint32_t> window_rank;
    std::vector<uint32_t> target_coverage;
    std::string dummy_quality;
};

void build_windows(Loaded& L, const PolishOptions& opt, Layered& Y) {
    const uint32_t w = opt.window_length;
    Y.dummy_quality.assign(w, '!');
    std::vector<uint64_t> first_window(L.targets + 1, 0);
    for (uint64_t i = 0; i < L.targets; ++i) {
        const auto& s = L.seqs[i];
        uint32_t k = 0;
        for (uint32_t j = 0; j < s.data.size(); j += w, ++k) {
            const uint32_t len = std::min(j + w, uint32_t(s.data.size())) - j;
            CpuWindowInput win;
            win.backbone = &s.data[j];
            win.backbone_len = len;
            win.backbone_qual = s.quality.empty() ? Y.dummy_quality.data() : &s.quality[j];
            Y.windows.push_back(win);
            Y.window_target.push_back(i);
            Y.window_rank.push_back(k);
        }
        first_window[i + 1] = first_window[i] + k;
    }
    Y.target_coverage.assign(L.targets, 0);
    for (auto& o : L.overlaps) {
        ++Y.target_coverage[o.t_id];
        const auto& sq = L.seqs[o.q_id];
        const auto& bp = o.breaking_points;
        for (size_t j = 0; j < bp.size(); j += 2) {
            if (bp[j + 1].second - bp[j].second < 0.02 * w) continue;
            if (!sq.quality.empty() || !sq.rquality.empty()) {
                const std::string& qual = o.strand ? sq.rquality : sq.quality;
                double avg = 0;
                for (uint32_t k = bp[j].second; k < bp[j + 1].second; ++k)
                    avg += static_cast<uint32_t>(qual[k]) - 33;
                avg /= bp[j + 1].second - bp[j].second;
                if (avg < opt.quality_threshold) continue;
            }
            const uint64_t wid = first_window[o.t_id] + bp[j].first / w;
            const uint32_t wstart = (bp[j].first / w) * w;
            const char* data = o.strand ? &sq.rc[bp[j].second] : &sq.data[bp[j].second];
            const uint32_t dlen = bp[j + 1].second - bp[j].second;
            const char* qual = o.strand ? (sq.rquality.empty() ? nullptr : &sq.rquality[bp[j].second])
                                        : (sq.quality.empty() ? nullptr : &sq.quality[bp[j].second]);
            const uint32_t begin = bp[j].first - wstart;
            const uint32_t end = bp[j + 1].first - wstart - 1;
            // Window::add_layer (src/window.cpp:42-63)
            CpuWindowInput& win = Y.windows[wid];
            if (dlen == 0 || begin == end) continue;
            if (begin >= end || begin > win.backbone_len || end > win.backbone_len) {
                fprintf(stderr, "[racon::Window::add_layer] error: layer begin and end positions are invalid!\n");
                exit(1);
            }
            win.seqs.push_back(data);
            win.quals.push_back(qual);
            win.lens.push_back(dlen);
            win.positions.emplace_back(begin, end);
        }
    }
}

int run_initialize(const std::string& sp, const std::string& op, const std::string& tp,
                   const PolishOptions& opt, Loaded& L, Layered& Y, PolishTimes* times) {
    double t0 = now_s();
    if (load_inputs(sp, op, tp, opt, L)) return 1;
    double t1 = now_s();
    parallel_for(L.overlaps.size(), opt.threads,
                 [&](uint64_t i) { align_and_break(L.overlaps[i], L.seqs, opt.window_length); });
    double t2 = now_s();
    build_windows(L, opt, Y);
    double t3 = now_s();
    if (times) {
        times->load_s = t1 - t0;
        times->align_s = t2 - t1;
        times->layers_s = t3 - t2;
        times->overlaps = L.overlaps.size();
        times->windows = Y.windows.size();
    }
    return 0;
}

}  // namespace

void CpuSequence::build_reverse() {
    if (!rc.empty()) return;
    rc.clear();
    rc.reserve(data.size());
    for (size_t i = data.size(); i-- > 0;) {
        switch (data[i]) {
            case 'A': rc += 'T'; break;
            case 'T': rc += 'A'; break;
            case 'C': rc += 'G'; break;
            case 'G': rc += 'C'; break;
            default: rc += data[i]; break;
        }
    }
    rquality.assign(quality.rbegin(), quality.rend());
}

bool read_sequences(const std::string& path, std::vector<CpuSequence>& out) {
    const int fmt = seq_format(path);
    LineReader r(path);
    if (!r.ok()) {
        fprintf(stderr, "[oracle] error: unable to open %s\n", path.c_str());
        return false;
    }
    std::string line, name, data, qual;
    if (fmt == 0) {
        bool have = false;
        while (r.next(line)) {
            if (!line.empty() && line[0] == '>') {
                if (have) out.push_back(make_sequence(name, data, nullptr));
                name = first_word(line, 1);
                data.clear();
                have = true;
            } else if (have) {
                append_bases(data, line);
            }
        }
        if (have) out.push_back(make_sequence(name, data, nullptr));
    } else {
        while (r.next(line)) {
            if (line.empty()) continue;
            if (line[0] != '@') continue;
            name = first_word(line, 1);
            data.clear();
            qual.clear();
            bool plus = false;
            while (r.next(line)) {
                if (!line.empty() && line[0] == '+') { plus = true; break; }
                append_bases(data, line);
            }
            if (!plus) break;
            while (qual.size() < data.size() && r.next(line)) append_bases(qual, line);
            out.push_back(make_sequence(name, data, &qual));
        }
    }
    return true;
}

void breakpoints_from_cigar(const CpuOverlap& o, uint32_t w,
                            std::vector<std::pair<uint32_t, uint32_t>>& out) {
    std::vector<int32_t> ends;
    for (uint32_t i = 0; i < o.t_end; i += w)
        if (i > o.t_begin) ends.push_back(int32_t(i) - 1);
    ends.push_back(int32_t(o.t_end) - 1);
    uint32_t wi = 0;
    bool found = false;
    std::pair<uint32_t, uint32_t> first = {0, 0}, last = {0, 0};
    int32_t q_ptr = int32_t(o.strand ? (o.q_length - o.q_end) : o.q_begin) - 1;
    int32_t t_ptr = int32_t(o.t_begin) - 1;
    const std::string& cg = o.cigar;
    for (size_t i = 0, j = 0; i < cg.size(); ++i) {
        const char c = cg[i];
        if (c == 'M' || c == '=' || c == 'X') {
            uint32_t nb = uint32_t(atoi(&cg[j]));
            j = i + 1;
            for (uint32_t k = 0; k < nb; ++k) {
                ++q_ptr;
                ++t_ptr;
                if (!found) {
                    found = true;
                    first = {uint32_t(t_ptr), uint32_t(q_ptr)};
                }
                last = {uint32_t(t_ptr + 1), uint32_t(q_ptr + 1)};
                if (t_ptr == ends[wi]) {
                    if (found) {
                        out.push_back(first);
                        out.push_back(last);
                    }
                    found = false;
                    ++wi;
                }
            }
        } else if (c == 'I') {
            q_ptr += atoi(&cg[j]);
            j = i + 1;
        } else if (c == 'D' || c == 'N') {
            uint32_t nb = uint32_t(atoi(&cg[j]));
            j = i + 1;
            for (uint32_t k = 0; k < nb; ++k) {
                ++t_ptr;
                if (t_ptr == ends[wi]) {
                    if (found) {
                        out.push_back(first);
                        out.push_back(last);
                    }
                    found = false;
                    ++wi;
                }
            }
        } else if (c == 'S' || c == 'H' || c == 'P') {
            j = i + 1;
        }
    }
}

bool window_consensus(const CpuWindowInput& w, bool tgs, bool trim, int match,
                      int mismatch, int gap, std::string& consensus,
                      WindowStats* stats, uint64_t window_id, uint32_t rank_id) {
    const uint32_t n = uint32_t(w.seqs.size()) + 1;  // entries incl. backbone
    if (n < 3) {
        consensus.assign(w.backbone, w.backbone_len);
        return false;
    }
    PoaGraph graph;
    graph.add_alignment(PoaAlignment(), w.backbone, w.backbone_len, w.backbone_qual,
                        w.backbone_len);
    std::vector<uint32_t> rank(n);
    for (uint32_t i = 0; i < n; ++i) rank[i] = i;
    auto first_of = [&](uint32_t i) { return i == 0 ? 0u : w.positions[i - 1].first; };
    std::sort(rank.begin() + 1, rank.end(),
              [&](uint32_t a, uint32_t b) { return first_of(a) < first_of(b); });
    const uint32_t offset = 0.01 * w.backbone_len;
    PoaStats ps;
    for (uint32_t j = 1; j < n; ++j) {
        const uint32_t i = rank[j] - 1;
        PoaAlignment aln;
        if (w.positions[i].first < offset && w.positions[i].second > w.backbone_len - offset) {
            aln = poa_align_nw(w.seqs[i], w.lens[i], graph, match, mismatch, gap, &ps);
        } else {
            std::vector<int32_t> mapping;
            auto sub = graph.subgraph(w.positions[i].first, w.positions[i].second, mapping);
            aln = poa_align_nw(w.seqs[i], w.lens[i], *sub, match, mismatch, gap, &ps);
            PoaGraph::update_alignment(aln, mapping);
        }
        if (w.quals[i] == nullptr) graph.add_alignment(aln, w.seqs[i], w.lens[i]);
        else graph.add_alignment(aln, w.seqs[i], w.lens[i], w.quals[i], w.lens[i]);
    }
    std::vector<uint32_t> cov;
    consensus = graph.generate_consensus(cov);
    if (stats) {
        stats->cells += ps.cells;
        stats->edge_cells += ps.edge_cells;
        stats->nodes = uint32_t(graph.nodes().size());
        stats->edges = uint32_t(graph.edges().size());
        stats->layers = n - 1;
    }
    if (tgs && trim) {
        const uint32_t avg = (n - 1) / 2;
        int32_t b = 0, e = int32_t(consensus.size()) - 1;
        for (; b < int32_t(consensus.size()); ++b)
            if (cov[b] >= avg) break;
        for (; e >= 0; --e)
            if (cov[e] >= avg) break;
        if (b >= e) {
            fprintf(stderr, "[racon::Window::generate_consensus] warning: contig %lu might be "
                            "chimeric in window %u!\n", (unsigned long)window_id, rank_id);
        } else {
            consensus = consensus.substr(b, e - b + 1);
        }
    }
    return true;
}

int polish_files(const std::string& sp, const std::string& op, const std::string& tp,
                 const PolishOptions& opt,
                 std::vector<std::pair<std::string, std::string>>& out,
                 PolishTimes* times) {
    Loaded L;
    Layered Y;
    if (run_initialize(sp, op, tp, opt, L, Y, times)) return 1;
    const size_t nw = Y.windows.size();
    std::vector<std::string> cons(nw);
    std::vector<uint8_t> polished(nw, 0);
    std::vector<uint64_t> cells(nw, 0);
    double t0 = now_s();
    parallel_for(nw, opt.threads, [&](uint64_t i) {
        WindowStats st;
        polished[i] = window_consensus(Y.windows[i], L.tgs, opt.trim, opt.match, opt.mismatch,
                                       opt.gap, cons[i], &st, Y.window_target[i],
                                       Y.window_rank[i]) ? 1 : 0;
        cells[i] = st.cells;
    });
    double t1 = now_s();
    if (times) {
        times->consensus_s = t1 - t0;
        for (auto c : cells) times->poa_cells += c;
    }
    std::string data;
    uint32_t npol = 0;
    for (size_t i = 0; i < nw; ++i) {
        npol += polished[i];
        data += cons[i];
        if (i == nw - 1 || Y.window_rank[i + 1] == 0) {
            const double ratio = npol / static_cast<double>(Y.window_rank[i] + 1);
            if (!opt.drop_unpolished || ratio > 0) {
                std::string tags = opt.fragment ? "r" : "";
                tags += " LN:i:" + std::to_string(data.size());
                tags += " RC:i:" + std::to_string(Y.target_coverage[Y.window_target[i]]);
                tags += " XC:f:" + std::to_string(ratio);
                out.emplace_back(L.seqs[Y.window_target[i]].name + tags, data);
            }
            npol = 0;
            data.clear();
        }
    }
    return 0;
}

int collect_layer_input(const std::string& sp, const std::string& op, const std::string& tp,
                        const PolishOptions& opt, std::vector<CpuSequence>& seqs, uint64_t& n_targets,
                        bool& tgs, std::vector<CpuOverlap>& overlaps_out) {
    Loaded L;
    if (load_inputs(sp, op, tp, opt, L)) return 1;
    parallel_for(L.overlaps.size(), opt.threads,
                 [&](uint64_t i) { align_and_break(L.overlaps[i], L.seqs, opt.window_length); });
    seqs = std::move(L.seqs);
    n_targets = L.targets;
    tgs = L.tgs;
    overlaps_out = std::move(L.overlaps);
    return 0;
}

int collect_windows(const std::string& sp, const std::string& op, const std::string& tp,
                    const PolishOptions& opt, std::vector<DumpedWindow>& windows) {
    Loaded L;
    Layered Y;
    if (run_initialize(sp, op, tp, opt, L, Y, nullptr)) return 1;
    for (size_t i = 0; i < Y.windows.size(); ++i) {
        const auto& w = Y.windows[i];
        DumpedWindow d;
        d.target_id = Y.window_target[i];
        d.rank = Y.window_rank[i];
        d.tgs = L.tgs;
        d.backbone.assign(w.backbone, w.backbone_len);
        d.backbone_qual.assign(w.backbone_qual, w.backbone_len);
        for (size_t j = 0; j < w.seqs.size(); ++j) {
            d.seqs.emplace_back(w.seqs[j], w.lens[j]);
            d.quals.push_back(w.quals[j] ? std::string(w.quals[j], w.lens[j]) : std::string());
        }
        d.positions = w.positions;
        windows.push_back(std::move(d));
    }
    return 0;
}

}  // namespace oracle
