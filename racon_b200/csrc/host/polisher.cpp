// racon's polishing pipeline on the host side of the B200 path.
//
// Mirrors, in behaviour, the reference sources:
//   src/sequence.cpp:19-100   Sequence
//   src/overlap.cpp:15-177    Overlap construction (MHAP/PAF/SAM) and transmute
//   src/polisher.cpp:55-460   createPolisher checks, initialize (loading,
//                             filtering, windows, layer assignment)
//   src/polisher.cpp:486-548  polish (stitching, tags, drop rule)
// The two hot calls go to the device through include/racon_b200.h:
//   find_overlap_breaking_points -> rb_align_batch / rb_cigar_breakpoints
//   layer assembly              -> rb_sequences_stage + rb_poa_stage_overlaps
//   polish                      -> rb_poa_run + rb_poa_fetch (window consensus)
// Input readers (the reference uses the absent bioparser library) are
// written here: FASTA/FASTQ (multi-line, gzip or plain), PAF, MHAP, SAM;
// names end at the first whitespace.
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "../../../include/racon_b200.h"
#include "racon.hpp"

namespace racon {

// ---------------------------------------------------------------- errors

struct Fatal : std::runtime_error {
    explicit Fatal(const std::string& m) : std::runtime_error(m) {}
};

namespace {
thread_local bool g_throw_on_error = false;

[[noreturn]] void fail(const std::string& msg) {
    if (g_throw_on_error) throw Fatal(msg);
    fprintf(stderr, "%s\n", msg.c_str());
    exit(1);
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool has_suffix(const std::string& s, const char* x) {
    const size_t n = strlen(x);
    return s.size() >= n && s.compare(s.size() - n, n, x) == 0;
}

// 0 FASTA, 1 FASTQ, -1 unknown
int sequence_format(const std::string& p) {
    for (const char* x : {".fasta", ".fasta.gz", ".fna", ".fna.gz", ".fa", ".fa.gz"})
        if (has_suffix(p, x)) return 0;
    for (const char* x : {".fastq", ".fastq.gz", ".fq", ".fq.gz"})
        if (has_suffix(p, x)) return 1;
    return -1;
}
// 0 MHAP, 1 PAF, 2 SAM, -1 unknown
int overlap_format(const std::string& p) {
    if (has_suffix(p, ".mhap") || has_suffix(p, ".mhap.gz")) return 0;
    if (has_suffix(p, ".paf") || has_suffix(p, ".paf.gz")) return 1;
    if (has_suffix(p, ".sam") || has_suffix(p, ".sam.gz")) return 2;
    return -1;
}

// Buffered line reader over gzip or plain files.
class Lines {
public:
    explicit Lines(const std::string& path) : f_(gzopen(path.c_str(), "rb")) {
        if (f_) gzbuffer(f_, 1 << 20);
    }
    ~Lines() {
        if (f_) gzclose(f_);
    }
    bool ok() const { return f_ != nullptr; }
    // next line without '\n' / '\r'; false at end of file
    bool next(std::string& line) {
        line.clear();
        while (true) {
            if (pos_ >= len_) {
                len_ = gzread(f_, buf_.data(), unsigned(buf_.size()));
                pos_ = 0;
                if (len_ <= 0) {
                    len_ = 0;
                    return !line.empty();
                }
            }
            const char* b = buf_.data() + pos_;
            const char* nl = static_cast<const char*>(memchr(b, '\n', size_t(len_ - pos_)));
            if (nl) {
                line.append(b, size_t(nl - b));
                pos_ += int(nl - b) + 1;
                if (!line.empty() && line.back() == '\r') line.pop_back();
                return true;
            }
            line.append(b, size_t(len_ - pos_));
            pos_ = len_;
        }
    }

private:
    gzFile f_;
    std::vector<char> buf_ = std::vector<char>(1 << 20);
    int pos_ = 0, len_ = 0;
};

// Whole file (gzip or plain) in memory; plain files by one fread.
std::string slurp(const std::string& path, bool& ok) {
    std::string buf;
    if (FILE* pf = fopen(path.c_str(), "rb")) {
        unsigned char magic[2] = {0, 0};
        const size_t got = fread(magic, 1, 2, pf);
        if (!(got == 2 && magic[0] == 0x1f && magic[1] == 0x8b) && fseek(pf, 0, SEEK_END) == 0) {
            const long size = ftell(pf);
            if (size >= 0 && fseek(pf, 0, SEEK_SET) == 0) {
                buf.resize(size_t(size));
                const size_t r = size ? fread(&buf[0], 1, size_t(size), pf) : 0;
                fclose(pf);
                ok = r == size_t(size);
                return buf;
            }
        }
        fclose(pf);
    }
    gzFile f = gzopen(path.c_str(), "rb");
    ok = f != nullptr;
    if (!f) return buf;
    gzbuffer(f, 1 << 20);
    const size_t chunk = size_t(16) << 20;
    size_t len = 0;
    while (true) {
        buf.resize(len + chunk);
        const int r = gzread(f, &buf[len], unsigned(chunk));
        if (r <= 0) break;
        len += size_t(r);
    }
    buf.resize(len);
    gzclose(f);
    return buf;
}

inline bool is_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Appends [b, e) without whitespace; a whole-line append when there is none
// (the check is a branch-free loop the compiler vectorises).
void append_clean(std::string& dst, const char* b, const char* e) {
    bool any = false;
    for (const char* p = b; p < e; ++p) any |= is_space(*p);
    if (!any) {
        dst.append(b, size_t(e - b));
        return;
    }
    for (const char* p = b; p < e; ++p)
        if (!is_space(*p)) dst.push_back(*p);
}

// Line cursor over an in-memory file: [b, e) of the next line without '\n'
// and a trailing '\r'.
struct LineCursor {
    const char* p;
    const char* end;
    bool next(const char*& b, const char*& e) {
        if (p >= end) return false;
        b = p;
        const char* nl = static_cast<const char*>(memchr(p, '\n', size_t(end - p)));
        e = nl ? nl : end;
        p = nl ? nl + 1 : end;
        if (e > b && e[-1] == '\r') --e;
        return true;
    }
};

size_t name_len(const char* b, const char* e) {
    const char* q = b;
    while (q < e && !isspace(uint8_t(*q))) ++q;
    return size_t(q - b);
}

void read_sequences(const std::string& path, int format, std::vector<std::unique_ptr<Sequence>>& dst) {
    bool ok = false;
    const std::string buf = slurp(path, ok);
    if (!ok) fail("[racon::Polisher::initialize] error: unable to open file " + path + "!");
    LineCursor in{buf.data(), buf.data() + buf.size()};
    const char *b, *e;
    std::string data, qual;
    if (format == 0) {
        bool open = false;
        const char* nb = nullptr;
        size_t nl = 0;
        while (in.next(b, e)) {
            if (e > b && *b == '>') {
                if (open) dst.emplace_back(new Sequence(nb, uint32_t(nl), data.data(), uint32_t(data.size())));
                nb = b + 1;
                nl = name_len(b + 1, e);
                data.clear();
                open = true;
            } else if (open) {
                append_clean(data, b, e);
            }
        }
        if (open) dst.emplace_back(new Sequence(nb, uint32_t(nl), data.data(), uint32_t(data.size())));
        return;
    }
    while (in.next(b, e)) {
        if (e == b || *b != '@') continue;
        const char* nb = b + 1;
        const size_t nl = name_len(b + 1, e);
        data.clear();
        qual.clear();
        bool plus = false;
        while (in.next(b, e)) {
            if (e > b && *b == '+') {
                plus = true;
                break;
            }
            append_clean(data, b, e);
        }
        if (!plus) fail("[racon::Polisher::initialize] error: truncated FASTQ record in " + path + "!");
        while (qual.size() < data.size() && in.next(b, e)) append_clean(qual, b, e);
        dst.emplace_back(new Sequence(nb, uint32_t(nl), data.data(), uint32_t(data.size()), qual.data(),
                                      uint32_t(qual.size())));
    }
}

uint32_t to_u32(const std::string& s) { return uint32_t(strtoul(s.c_str(), nullptr, 10)); }

}  // namespace

// ---------------------------------------------------------------- Sequence

Sequence::Sequence(const char* name, uint32_t name_length, const char* data, uint32_t data_length)
    : name_(name, name_length) {
    data_.resize(data_length);
    // toupper in the C locale: only a-z change
    char* d = &data_[0];
    for (uint32_t i = 0; i < data_length; ++i) {
        const char c = data[i];
        d[i] = (c >= 'a' && c <= 'z') ? char(c - 32) : c;
    }
}

Sequence::Sequence(const char* name, uint32_t name_length, const char* data, uint32_t data_length,
                   const char* quality, uint32_t quality_length)
    : Sequence(name, name_length, data, data_length) {
    uint32_t sum = 0;
    for (uint32_t i = 0; i < quality_length; ++i) sum += uint32_t(quality[i] - '!');
    if (sum > 0) quality_.assign(quality, quality_length);
}

Sequence::Sequence(const std::string& name, const std::string& data) : name_(name), data_(data) {}

std::unique_ptr<Sequence> createSequence(const std::string& name, const std::string& data) {
    return std::unique_ptr<Sequence>(new Sequence(name, data));
}

void Sequence::create_reverse_complement() {
    if (!reverse_complement_.empty()) return;
    // A <-> T, C <-> G, every other byte unchanged (src/sequence.cpp:49-84)
    static const struct Table {
        char t[256];
        Table() {
            for (int c = 0; c < 256; ++c) t[c] = char(c);
            t[uint8_t('A')] = 'T';
            t[uint8_t('T')] = 'A';
            t[uint8_t('C')] = 'G';
            t[uint8_t('G')] = 'C';
        }
    } comp;
    reverse_complement_.resize(data_.size());
    char* r = &reverse_complement_[0];
    for (size_t i = 0, n = data_.size(); i < n; ++i) r[i] = comp.t[uint8_t(data_[n - 1 - i])];
    reverse_quality_.assign(quality_.rbegin(), quality_.rend());
}

void Sequence::transmute(bool has_name, bool has_data, bool has_reverse_data) {
    if (!has_name) std::string().swap(name_);
    // the forward strand also stays when only the reverse one is used: the
    // device builds the reverse complement from it (the host one is made
    // only on demand, create_reverse_complement)
    if (!has_data && !has_reverse_data) {
        std::string().swap(data_);
        std::string().swap(quality_);
    }
}

// ---------------------------------------------------------------- Overlap

class Overlap {
public:
    std::string q_name, t_name;
    uint64_t q_id = 0, t_id = 0;
    uint32_t q_begin = 0, q_end = 0, q_length = 0;
    uint32_t t_begin = 0, t_end = 0, t_length = 0;
    uint32_t strand = 0, length = 0;
    double error = 0;
    std::string cigar;
    bool valid = true, transmuted = false;
    std::vector<std::pair<uint32_t, uint32_t>> breaking_points;

    void finish_lengths(uint32_t qspan, uint32_t tspan) {
        length = std::max(qspan, tspan);
        error = 1 - std::min(qspan, tspan) / static_cast<double>(length);
    }

    // src/overlap.cpp:129-177
    void transmute(const std::vector<std::unique_ptr<Sequence>>& seqs,
                   const std::unordered_map<std::string, uint64_t>& name_to_id,
                   const std::unordered_map<uint64_t, uint64_t>& id_to_id) {
        if (!valid || transmuted) return;
        if (!q_name.empty()) {
            auto it = name_to_id.find(q_name + "q");
            if (it == name_to_id.end()) {
                valid = false;
                return;
            }
            q_id = it->second;
            std::string().swap(q_name);
        } else {
            auto it = id_to_id.find(q_id << 1 | 0);
            if (it == id_to_id.end()) {
                valid = false;
                return;
            }
            q_id = it->second;
        }
        if (q_length != seqs[q_id]->data().size())
            fail("[racon::Overlap::transmute] error: unequal lengths in sequence and overlap file for sequence " +
                 seqs[q_id]->name() + "!");
        if (!t_name.empty()) {
            auto it = name_to_id.find(t_name + "t");
            if (it == name_to_id.end()) {
                valid = false;
                return;
            }
            t_id = it->second;
            std::string().swap(t_name);
        } else {
            auto it = id_to_id.find(t_id << 1 | 1);
            if (it == id_to_id.end()) {
                valid = false;
                return;
            }
            t_id = it->second;
        }
        if (t_length != 0 && t_length != seqs[t_id]->data().size())
            fail("[racon::Overlap::transmute] error: unequal lengths in target and overlap file for target " +
                 seqs[t_id]->name() + "!");
        t_length = uint32_t(seqs[t_id]->data().size());
        transmuted = true;
    }
};

namespace {

void split_tabs(const std::string& line, std::vector<std::string>& f) {
    f.clear();
    size_t b = 0;
    while (true) {
        const size_t e = line.find('\t', b);
        f.emplace_back(line, b, e == std::string::npos ? std::string::npos : e - b);
        if (e == std::string::npos) break;
        b = e + 1;
    }
}

void split_spaces(const std::string& line, std::vector<std::string>& f) {
    f.clear();
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && isspace(uint8_t(line[i]))) ++i;
        size_t j = i;
        while (j < line.size() && !isspace(uint8_t(line[j]))) ++j;
        if (j > i) f.emplace_back(line, i, j - i);
        i = j;
    }
}

// SAM record -> overlap (src/overlap.cpp:44-108)
void sam_overlap(Overlap& o, const std::vector<std::string>& f) {
    o.q_name = f[0];
    const uint32_t flag = to_u32(f[1]);
    o.t_name = f[2];
    o.t_begin = to_u32(f[3]) - 1;
    o.cigar = f[5];
    o.strand = (flag & 0x10) ? 1 : 0;
    o.valid = !(flag & 0x4);
    if (o.cigar.size() < 2 && o.valid) fail("[Racon::Overlap::Overlap] error: missing alignment from SAM object!");
    const std::string& c = o.cigar;
    for (size_t i = 0; i < c.size(); ++i) {
        if (c[i] == 'S' || c[i] == 'H') {
            o.q_begin = uint32_t(atoi(&c[0]));
            break;
        }
        if (strchr("M=IDNPX", c[i]) && c[i] != 0) break;
    }
    uint32_t qa = 0, qc = 0, ta = 0;
    for (size_t i = 0, j = 0; i < c.size(); ++i) {
        const char ch = c[i];
        if (ch == 'M' || ch == '=' || ch == 'X') {
            const uint32_t n = uint32_t(atoi(&c[j]));
            j = i + 1;
            qa += n;
            ta += n;
        } else if (ch == 'I') {
            qa += uint32_t(atoi(&c[j]));
            j = i + 1;
        } else if (ch == 'D' || ch == 'N') {
            ta += uint32_t(atoi(&c[j]));
            j = i + 1;
        } else if (ch == 'S' || ch == 'H') {
            qc += uint32_t(atoi(&c[j]));
            j = i + 1;
        } else if (ch == 'P') {
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
    o.finish_lengths(qa, ta);
}

void read_overlaps(const std::string& path, int format, std::vector<std::unique_ptr<Overlap>>& dst) {
    Lines in(path);
    if (!in.ok()) fail("[racon::Polisher::initialize] error: unable to open file " + path + "!");
    std::string line;
    std::vector<std::string> f;
    while (in.next(line)) {
        if (line.empty()) continue;
        std::unique_ptr<Overlap> o(new Overlap());
        if (format == 0) {  // MHAP (src/overlap.cpp:15-27)
            split_spaces(line, f);
            if (f.size() < 12) continue;
            o->q_id = strtoull(f[0].c_str(), nullptr, 10) - 1;
            o->t_id = strtoull(f[1].c_str(), nullptr, 10) - 1;
            o->strand = to_u32(f[4]) ^ to_u32(f[8]);
            o->q_begin = to_u32(f[5]);
            o->q_end = to_u32(f[6]);
            o->q_length = to_u32(f[7]);
            o->t_begin = to_u32(f[9]);
            o->t_end = to_u32(f[10]);
            o->t_length = to_u32(f[11]);
            o->finish_lengths(o->q_end - o->q_begin, o->t_end - o->t_begin);
        } else if (format == 1) {  // PAF (src/overlap.cpp:29-42)
            split_tabs(line, f);
            if (f.size() < 12) continue;
            o->q_name = f[0];
            o->q_length = to_u32(f[1]);
            o->q_begin = to_u32(f[2]);
            o->q_end = to_u32(f[3]);
            o->strand = f[4] == "-" ? 1 : 0;
            o->t_name = f[5];
            o->t_length = to_u32(f[6]);
            o->t_begin = to_u32(f[7]);
            o->t_end = to_u32(f[8]);
            o->finish_lengths(o->q_end - o->q_begin, o->t_end - o->t_begin);
        } else {  // SAM
            if (line[0] == '@') continue;
            split_tabs(line, f);
            if (f.size() < 11) continue;
            sam_overlap(*o, f);
        }
        dst.push_back(std::move(o));
    }
}

}  // namespace

// ---------------------------------------------------------------- Window

class Window {
public:
    uint64_t id;
    uint32_t rank;
    const char* backbone;
    uint32_t backbone_length;
    const char* quality;  // nullptr: racon's dummy '!' quality
    std::vector<const char*> seqs, quals;
    std::vector<uint32_t> lens, begins, ends;
    std::string consensus;

    // src/window.cpp:42-63
    void add_layer(const char* s, uint32_t len, const char* q, uint32_t qlen, uint32_t b, uint32_t e) {
        if (len == 0 || b == e) return;
        if (q != nullptr && len != qlen) fail("[racon::Window::add_layer] error: unequal quality size!");
        if (b >= e || b > backbone_length || e > backbone_length)
            fail("[racon::Window::add_layer] error: layer begin and end positions are invalid!");
        seqs.push_back(s);
        quals.push_back(q);
        lens.push_back(len);
        begins.push_back(b);
        ends.push_back(e);
    }
};

// ---------------------------------------------------------------- Polisher

// Argument checks of createPolisher (src/polisher.cpp:135-159): polisher
// type, window length and the three file extensions.
static void check_polisher_args(const std::string& sequences_path, const std::string& overlaps_path,
                         const std::string& target_path, PolisherType type, uint32_t window_length, int& sf,
                         int& of, int& tf) {
    if (type != PolisherType::kC && type != PolisherType::kF)
        fail("[racon::createPolisher] error: invalid polisher type!");
    if (window_length == 0) fail("[racon::createPolisher] error: invalid window length!");
    sf = sequence_format(sequences_path);
    if (sf < 0)
        fail("[racon::createPolisher] error: file " + sequences_path +
             " has unsupported format extension (valid extensions: .fasta, .fasta.gz, .fna, .fna.gz, "
             ".fa, .fa.gz, .fastq, .fastq.gz, .fq, .fq.gz)!");
    of = overlap_format(overlaps_path);
    if (of < 0)
        fail("[racon::createPolisher] error: file " + overlaps_path +
             " has unsupported format extension (valid extensions: .mhap, .mhap.gz, .paf, .paf.gz, "
             ".sam, .sam.gz)!");
    tf = sequence_format(target_path);
    if (tf < 0)
        fail("[racon::createPolisher] error: file " + target_path +
             " has unsupported format extension (valid extensions: .fasta, .fasta.gz, .fna, .fna.gz, "
             ".fa, .fa.gz, .fastq, .fastq.gz, .fq, .fq.gz)!");
}

std::unique_ptr<Polisher> createPolisher(const std::string& sequences_path,
    const std::string& overlaps_path, const std::string& target_path,
    PolisherType type, uint32_t window_length, double quality_threshold,
    double error_threshold, bool trim, int8_t match, int8_t mismatch, int8_t gap,
    uint32_t num_threads, uint32_t cuda_batches, bool cuda_banded_alignment,
    uint32_t cudaaligner_batches, uint32_t cudaaligner_band_width) {
    (void)cuda_batches;
    (void)cuda_banded_alignment;
    (void)cudaaligner_batches;
    (void)cudaaligner_band_width;
    int sf, of, tf;
    check_polisher_args(sequences_path, overlaps_path, target_path, type, window_length, sf, of, tf);
    return std::unique_ptr<Polisher>(new Polisher(sequences_path, overlaps_path, target_path, sf, of, tf, type,
                                                  window_length, quality_threshold, error_threshold, trim,
                                                  match, mismatch, gap, num_threads));
}

std::unique_ptr<Polisher> createPolisherOnContext(rb_ctx* ctx, int device, const std::string& sequences_path,
    const std::string& overlaps_path, const std::string& target_path, PolisherType type, uint32_t window_length,
    double quality_threshold, double error_threshold, bool trim, int8_t match, int8_t mismatch, int8_t gap) {
    if (!ctx) fail("[racon::createPolisher] error: no device context!");
    int sf, of, tf;
    check_polisher_args(sequences_path, overlaps_path, target_path, type, window_length, sf, of, tf);
    return std::unique_ptr<Polisher>(new Polisher(sequences_path, overlaps_path, target_path, sf, of, tf, type,
                                                  window_length, quality_threshold, error_threshold, trim,
                                                  match, mismatch, gap, 1, ctx, device));
}

Polisher::Polisher(const std::string& sp, const std::string& op, const std::string& tp, int sf, int of,
                   int tf, PolisherType type, uint32_t window_length, double quality_threshold,
                   double error_threshold, bool trim, int8_t match, int8_t mismatch, int8_t gap,
                   uint32_t num_threads, rb_ctx* borrowed_ctx, int device)
    : sequences_path_(sp), overlaps_path_(op), target_path_(tp), sequences_format_(sf),
      overlaps_format_(of), target_format_(tf), type_(type), quality_threshold_(quality_threshold),
      error_threshold_(error_threshold), trim_(trim), match_(match), mismatch_(mismatch), gap_(gap),
      dummy_quality_(window_length, '!'), window_length_(window_length), num_threads_(num_threads) {
    if (borrowed_ctx) {
        ctx_ = borrowed_ctx;
        owns_ctx_ = false;
        device_ = device;
        return;
    }
    const char* dev = getenv("RACON_B200_DEVICE");
    device_ = dev ? atoi(dev) : 0;
    rb_params p;
    p.match = match;
    p.mismatch = mismatch;
    p.gap = gap;
    p.window_length = window_length;
    ctx_ = rb_create(device_, &p);
    if (!ctx_) fail(std::string("[racon::Polisher] error: ") + rb_create_error());
}

Polisher::~Polisher() {
    if (ctx_ && owns_ctx_) rb_destroy(ctx_);
}

void Polisher::initialize() {
    if (!windows_.empty()) {
        fprintf(stderr, "[racon::Polisher::initialize] warning: object already initialized!\n");
        return;
    }
    const double t0 = now_s();
    read_sequences(target_path_, target_format_, sequences_);
    const uint64_t targets_size = sequences_.size();
    if (targets_size == 0) fail("[racon::Polisher::initialize] error: empty target sequences set!");
    std::unordered_map<std::string, uint64_t> name_to_id;
    std::unordered_map<uint64_t, uint64_t> id_to_id;
    for (uint64_t i = 0; i < targets_size; ++i) {
        name_to_id[sequences_[i]->name() + "t"] = i;
        id_to_id[i << 1 | 1] = i;
    }
    std::vector<std::unique_ptr<Sequence>> reads;
    read_sequences(sequences_path_, sequences_format_, reads);
    uint64_t sequences_size = 0, total_length = 0;
    for (auto& r : reads) {
        total_length += r->data().size();
        auto it = name_to_id.find(r->name() + "t");
        if (it != name_to_id.end()) {
            if (r->data().size() != sequences_[it->second]->data().size() ||
                r->quality().size() != sequences_[it->second]->quality().size())
                fail("[racon::Polisher::initialize] error: duplicate sequence " + r->name() + " with unequal data");
            name_to_id[r->name() + "q"] = it->second;
            id_to_id[sequences_size << 1 | 0] = it->second;
        } else {
            name_to_id[r->name() + "q"] = sequences_.size();
            id_to_id[sequences_size << 1 | 0] = sequences_.size();
            sequences_.push_back(std::move(r));
        }
        ++sequences_size;
    }
    reads.clear();
    if (sequences_size == 0) fail("[racon::Polisher::initialize] error: empty sequences set!");
    tgs_ = !(static_cast<double>(total_length) / sequences_size <= 1000);

    std::vector<std::unique_ptr<Overlap>> all;
    read_overlaps(overlaps_path_, overlaps_format_, all);
    for (auto& o : all) {
        o->transmute(sequences_, name_to_id, id_to_id);
        if (!o->valid) o.reset();
    }
    // per contiguous run of equal query id (src/polisher.cpp:284-335)
    auto remove_invalid = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            if (!all[i]) continue;
            if (all[i]->error > error_threshold_ || all[i]->q_id == all[i]->t_id) {
                all[i].reset();
                continue;
            }
            if (type_ == PolisherType::kC) {
                for (size_t j = i + 1; j < e; ++j) {
                    if (!all[j]) continue;
                    if (all[i]->length > all[j]->length) {
                        all[j].reset();
                    } else {
                        all[i].reset();
                        break;
                    }
                }
            }
        }
    };
    size_t c = 0;
    for (size_t i = 0; i < all.size(); ++i) {
        if (!all[i]) continue;
        while (!all[c]) ++c;
        if (all[c]->q_id != all[i]->q_id) {
            remove_invalid(c, i);
            c = i;
        }
    }
    remove_invalid(c, all.size());
    std::vector<std::unique_ptr<Overlap>> overlaps;
    std::vector<bool> has_name(sequences_.size(), false), has_data(sequences_.size(), false),
        has_reverse(sequences_.size(), false);
    for (uint64_t i = 0; i < targets_size; ++i) has_name[i] = has_data[i] = true;
    for (auto& o : all) {
        if (!o) continue;
        if (o->strand) has_reverse[o->q_id] = true;
        else has_data[o->q_id] = true;
        overlaps.push_back(std::move(o));
    }
    all.clear();
    if (overlaps.empty()) fail("[racon::Polisher::initialize] error: empty overlap set!");
    for (size_t i = 0; i < sequences_.size(); ++i) sequences_[i]->transmute(has_name[i], has_data[i], has_reverse[i]);
    const double t1 = now_s();

    // the sequence table in device memory: the aligner and the layer
    // assembly read the reads from there
    sequence_table_.resize(sequences_.size());
    for (size_t i = 0; i < sequences_.size(); ++i) {
        const Sequence& q = *sequences_[i];
        rb_sequence& e = sequence_table_[i];
        e.data = q.data().data();
        e.quality = q.quality().empty() ? nullptr : q.quality().data();
        e.length = uint32_t(q.data().size());
        e.forward = has_data[i] ? 1 : 0;
        e.reverse = has_reverse[i] ? 1 : 0;
    }
    if (rb_sequences_stage(ctx_, sequence_table_.data(), sequence_table_.size()) != RB_OK)
        fail(std::string("[racon::Polisher::initialize] error: ") + rb_last_error(ctx_));
    staged_ = false;
    targets_size_ = targets_size;
    find_overlap_breaking_points(overlaps);
    const double t2 = now_s();

    // windows (src/polisher.cpp:384-399)
    std::vector<uint64_t> first_window(targets_size + 1, 0);
    for (uint64_t i = 0; i < targets_size; ++i) {
        const std::string& d = sequences_[i]->data();
        uint32_t k = 0;
        for (uint32_t j = 0; j < d.size(); j += window_length_, ++k) {
            const uint32_t len = std::min(j + window_length_, uint32_t(d.size())) - j;
            if (len == 0) fail("[racon::createWindow] error: empty backbone sequence/unequal quality length!");
            std::shared_ptr<Window> w(new Window());
            w->id = i;
            w->rank = k;
            w->backbone = &d[j];
            w->backbone_length = len;
            w->quality = sequences_[i]->quality().empty() ? nullptr : &sequences_[i]->quality()[j];
            windows_.push_back(w);
        }
        first_window[i + 1] = first_window[i] + k;
    }
    // layers (src/polisher.cpp:401-457), assembled on the device from the
    // overlaps' ids, strands and breaking points
    targets_coverages_.assign(targets_size, 0);
    layer_overlaps_.clear();
    breakpoints_.clear();
    bp_offsets_.assign(1, 0);
    for (auto& o : overlaps) {
        ++targets_coverages_[o->t_id];
        layer_overlaps_.push_back(rb_layer_overlap{uint32_t(o->q_id), uint32_t(o->t_id), o->strand ? 1u : 0u});
        for (const auto& p : o->breaking_points) {
            breakpoints_.push_back(p.first);
            breakpoints_.push_back(p.second);
        }
        bp_offsets_.push_back(breakpoints_.size());
        o.reset();
    }
    // the aligner already staged the layers when every overlap was aligned
    // on the device; otherwise (SAM CIGARs) they come from these points
    if (!staged_) {
        if (rb_poa_stage_overlaps(ctx_, targets_size, layer_overlaps_.data(), layer_overlaps_.size(),
                                  breakpoints_.data(), bp_offsets_.data(), quality_threshold_, tgs_ ? 1 : 0,
                                  trim_ ? 1 : 0) != RB_OK)
            fail(std::string("[racon::Polisher::initialize] error: ") + rb_last_error(ctx_));
        staged_ = true;
    }
    const double t3 = now_s();
    stage_s_[0] = t1 - t0;
    stage_s_[1] = t2 - t1;
    stage_s_[2] = t3 - t2;
}

void Polisher::assemble_host_layers() {
    const size_t targets_size = targets_coverages_.size();
    std::vector<uint64_t> first_window(targets_size + 1, 0);
    for (const auto& w : windows_) ++first_window[w->id + 1];
    for (size_t i = 0; i < targets_size; ++i) first_window[i + 1] += first_window[i];
    for (size_t i = 0; i < layer_overlaps_.size(); ++i) {
        const rb_layer_overlap& o = layer_overlaps_[i];
        Sequence& s = *sequences_[o.q_id];
        if (o.strand) s.create_reverse_complement();
        std::vector<std::pair<uint32_t, uint32_t>> bp;
        for (uint64_t x = bp_offsets_[i]; x < bp_offsets_[i + 1]; x += 2)
            bp.emplace_back(breakpoints_[x], breakpoints_[x + 1]);
        for (size_t j = 0; j + 1 < bp.size(); j += 2) {
            if (bp[j + 1].second - bp[j].second < 0.02 * window_length_) continue;
            if (!s.quality().empty() || !s.reverse_quality().empty()) {
                const std::string& q = o.strand ? s.reverse_quality() : s.quality();
                double avg = 0;
                for (uint32_t k = bp[j].second; k < bp[j + 1].second; ++k) avg += static_cast<uint32_t>(q[k]) - 33;
                avg /= bp[j + 1].second - bp[j].second;
                if (avg < quality_threshold_) continue;
            }
            const uint64_t wid = first_window[o.t_id] + bp[j].first / window_length_;
            const uint32_t wstart = (bp[j].first / window_length_) * window_length_;
            const char* data = o.strand ? &s.reverse_complement()[bp[j].second] : &s.data()[bp[j].second];
            const uint32_t dlen = bp[j + 1].second - bp[j].second;
            const char* qual = o.strand
                                   ? (s.reverse_quality().empty() ? nullptr : &s.reverse_quality()[bp[j].second])
                                   : (s.quality().empty() ? nullptr : &s.quality()[bp[j].second]);
            windows_[wid]->add_layer(data, dlen, qual, qual ? dlen : 0, bp[j].first - wstart,
                                     bp[j + 1].first - wstart - 1);
        }
    }
}

// Device alignment of every overlap without a CIGAR, from the sequence
// table in device memory; device CIGAR walk for the others
// (src/polisher.cpp:462-484 -> src/overlap.cpp:179-203). When every overlap
// is aligned, the breaking points also become window layers on the device
// in the same call, and only a copy comes back to the host overlaps.
void Polisher::find_overlap_breaking_points(std::vector<std::unique_ptr<Overlap>>& overlaps) {
    std::vector<rb_store_pair> pairs;
    std::vector<size_t> pair_of;
    std::vector<rb_cigar_overlap> cig;
    std::vector<size_t> cig_of;
    for (size_t i = 0; i < overlaps.size(); ++i) {
        Overlap& o = *overlaps[i];
        if (!o.transmuted) fail("[racon::Overlap::find_breaking_points] error: overlap is not transmuted!");
        if (!o.breaking_points.empty()) continue;
        const uint32_t q_offset = o.strand ? o.q_length - o.q_end : o.q_begin;
        if (o.cigar.empty()) {
            rb_store_pair p;
            p.q_id = uint32_t(o.q_id);
            p.q_begin = o.q_begin;
            p.q_end = o.q_end;
            p.t_id = uint32_t(o.t_id);
            p.t_begin = o.t_begin;
            p.t_end = o.t_end;
            p.strand = o.strand ? 1u : 0u;
            pairs.push_back(p);
            pair_of.push_back(i);
        } else {
            rb_cigar_overlap c;
            c.cigar = o.cigar.data();
            c.cigar_length = uint32_t(o.cigar.size());
            c.q_offset = q_offset;
            c.t_begin = o.t_begin;
            c.t_end = o.t_end;
            cig.push_back(c);
            cig_of.push_back(i);
        }
    }
    if (cig.empty() && pairs.size() == overlaps.size()) {
        // every overlap aligned here: layers staged on the device as well
        rb_aln_result r;
        if (rb_poa_stage_alignments(ctx_, targets_size_, pairs.data(), pairs.size(), quality_threshold_,
                                    tgs_ ? 1 : 0, trim_ ? 1 : 0, &r) != RB_OK)
            fail(std::string("[racon::Overlap::find_breaking_points] error: ") + rb_last_error(ctx_));
        for (size_t k = 0; k < pairs.size(); ++k) {
            Overlap& o = *overlaps[pair_of[k]];
            for (uint64_t x = r.bp_offsets[k]; x < r.bp_offsets[k + 1]; x += 2)
                o.breaking_points.emplace_back(r.breakpoints[x], r.breakpoints[x + 1]);
        }
        staged_ = true;
        for (auto& o : overlaps) std::string().swap(o->cigar);
        return;
    }
    // batches bounded by bases so device buffers stay modest
    const uint64_t kBatchBases = uint64_t(1) << 31;
    size_t b = 0;
    while (b < pairs.size()) {
        size_t e = b;
        uint64_t bases = 0;
        while (e < pairs.size()) {
            const uint64_t pb = uint64_t(pairs[e].q_end - pairs[e].q_begin) + (pairs[e].t_end - pairs[e].t_begin);
            if (e > b && bases + pb > kBatchBases) break;
            bases += pb;
            ++e;
        }
        rb_aln_result r;
        if (rb_align_stage_overlaps(ctx_, pairs.data() + b, e - b, 0) != RB_OK || rb_align_run(ctx_) != RB_OK ||
            rb_align_fetch(ctx_, &r) != RB_OK)
            fail(std::string("[racon::Overlap::find_breaking_points] error: ") + rb_last_error(ctx_));
        for (size_t k = b; k < e; ++k) {
            Overlap& o = *overlaps[pair_of[k]];
            for (uint64_t x = r.bp_offsets[k - b]; x < r.bp_offsets[k - b + 1]; x += 2)
                o.breaking_points.emplace_back(r.breakpoints[x], r.breakpoints[x + 1]);
        }
        b = e;
    }
    if (!cig.empty()) {
        rb_aln_result r;
        if (rb_cigar_breakpoints(ctx_, cig.data(), cig.size(), &r) != RB_OK)
            fail(std::string("[racon::Overlap::find_breaking_points] error: ") + rb_last_error(ctx_));
        for (size_t k = 0; k < cig.size(); ++k) {
            Overlap& o = *overlaps[cig_of[k]];
            for (uint64_t x = r.bp_offsets[k]; x < r.bp_offsets[k + 1]; x += 2)
                o.breaking_points.emplace_back(r.breakpoints[x], r.breakpoints[x + 1]);
        }
    }
    for (auto& o : overlaps) std::string().swap(o->cigar);
}

void Polisher::polish(std::vector<std::unique_ptr<Sequence>>& dst, bool drop_unpolished_sequences) {
    const double t0 = now_s();
    const size_t nw = windows_.size();
    std::vector<uint8_t> polished(nw, 0);
    // device consensus of the windows initialize() staged
    if (!staged_) fail("[racon::Polisher::polish] error: windows are not staged (initialize first)");
    rb_poa_result r;
    if (rb_poa_run(ctx_) != RB_OK || rb_poa_fetch(ctx_, &r) != RB_OK)
        fail(std::string("[racon::Polisher::polish] error: ") + rb_last_error(ctx_));
    staged_ = false;
    for (size_t i = 0; i < nw; ++i) {
        windows_[i]->consensus.assign(r.consensus + r.offsets[i], r.consensus + r.offsets[i + 1]);
        polished[i] = r.polished[i];
    }
    // stitching (src/polisher.cpp:506-533)
    std::string data;
    uint32_t npol = 0;
    for (size_t i = 0; i < nw; ++i) {
        npol += polished[i];
        data += windows_[i]->consensus;
        if (i == nw - 1 || windows_[i + 1]->rank == 0) {
            const double ratio = npol / static_cast<double>(windows_[i]->rank + 1);
            if (!drop_unpolished_sequences || ratio > 0) {
                std::string tags = type_ == PolisherType::kF ? "r" : "";
                tags += " LN:i:" + std::to_string(data.size());
                tags += " RC:i:" + std::to_string(targets_coverages_[windows_[i]->id]);
                tags += " XC:f:" + std::to_string(ratio);
                dst.emplace_back(createSequence(sequences_[windows_[i]->id]->name() + tags, data));
            }
            npol = 0;
            data.clear();
        }
        windows_[i].reset();
    }
    std::vector<std::shared_ptr<Window>>().swap(windows_);
    std::vector<std::unique_ptr<Sequence>>().swap(sequences_);
    stage_s_[3] = now_s() - t0;
}

std::vector<std::unique_ptr<Sequence>> polish_files(const std::string& sp, const std::string& op,
    const std::string& tp, PolisherType type, uint32_t w, double q, double e, bool trim, int8_t m,
    int8_t x, int8_t g, uint32_t threads, bool drop, double* stage_seconds) {
    auto p = createPolisher(sp, op, tp, type, w, q, e, trim, m, x, g, threads);
    p->initialize();
    std::vector<std::unique_ptr<Sequence>> out;
    p->polish(out, drop);
    if (stage_seconds)
        for (int i = 0; i < 4; ++i) stage_seconds[i] = p->stage_seconds()[i];
    return out;
}

int polish_job_on_context(rb_ctx* ctx, int device, const std::string& sp, const std::string& op,
                          const std::string& tp, bool fragment, uint32_t w, double q, double e, bool trim,
                          int8_t m, int8_t x, int8_t g, bool drop, std::string* fasta, std::string* error,
                          double* stage_seconds) {
    const bool was = g_throw_on_error;
    g_throw_on_error = true;
    try {
        auto p = createPolisherOnContext(ctx, device, sp, op, tp, fragment ? PolisherType::kF : PolisherType::kC, w,
                                         q, e, trim, m, x, g);
        p->initialize();
        std::vector<std::unique_ptr<Sequence>> out;
        p->polish(out, drop);
        if (stage_seconds)
            for (int i = 0; i < 4; ++i) stage_seconds[i] = p->stage_seconds()[i];
        fasta->clear();
        for (const auto& r : out) {
            *fasta += '>';
            *fasta += r->name();
            *fasta += '\n';
            *fasta += r->data();
            *fasta += '\n';
        }
        g_throw_on_error = was;
        return RB_OK;
    } catch (const Fatal& ex) {
        g_throw_on_error = was;
        *error = ex.what();
        return RB_ERR_ARG;
    } catch (const std::bad_alloc&) {
        g_throw_on_error = was;
        *error = "host allocation failed";
        return RB_ERR_NOMEM;
    }
}

}  // namespace racon

// ---------------------------------------------------------------- C entry

extern "C" int rb_polish_files(const char* sequences_path, const char* overlaps_path, const char* target_path,
                               int fragment, uint32_t window_length, double quality_threshold,
                               double error_threshold, int trim, int8_t match, int8_t mismatch, int8_t gap,
                               uint32_t threads, int drop_unpolished, int device, char** fasta,
                               double* stage_seconds);

namespace {
std::string g_pipeline_error;
}

extern "C" const char* rb_pipeline_error(void) { return g_pipeline_error.c_str(); }

extern "C" int rb_polish_files(const char* sequences_path, const char* overlaps_path, const char* target_path,
                               int fragment, uint32_t window_length, double quality_threshold,
                               double error_threshold, int trim, int8_t match, int8_t mismatch, int8_t gap,
                               uint32_t threads, int drop_unpolished, int device, char** fasta,
                               double* stage_seconds) {
    if (!sequences_path || !overlaps_path || !target_path || !fasta) return RB_ERR_ARG;
    racon::g_throw_on_error = true;
    std::string dev = std::to_string(device);
    setenv("RACON_B200_DEVICE", dev.c_str(), 1);
    try {
        auto out = racon::polish_files(sequences_path, overlaps_path, target_path,
                                       fragment ? racon::PolisherType::kF : racon::PolisherType::kC, window_length,
                                       quality_threshold, error_threshold, trim != 0, match, mismatch, gap,
                                       threads, drop_unpolished != 0, stage_seconds);
        std::string text;
        for (const auto& s : out) {
            text += '>';
            text += s->name();
            text += '\n';
            text += s->data();
            text += '\n';
        }
        char* buf = static_cast<char*>(malloc(text.size() + 1));
        if (!buf) return RB_ERR_NOMEM;
        memcpy(buf, text.c_str(), text.size() + 1);
        *fasta = buf;
        racon::g_throw_on_error = false;
        g_pipeline_error.clear();
        return RB_OK;
    } catch (const racon::Fatal& e) {
        racon::g_throw_on_error = false;
        g_pipeline_error = e.what();
        *fasta = nullptr;
        return RB_ERR_ARG;
    }
}

// ---------------------------------------------------------------- jobs

struct rb_job {
    std::unique_ptr<racon::Polisher> polisher;
    std::vector<rb_window> views;
    double stage_s[3] = {0, 0, 0};

    // window views after initialize() (friend of racon::Polisher); the
    // layers are assembled on the host for them
    void collect() {
        polisher->assemble_host_layers();
        const racon::Polisher& p = *polisher;
        views.resize(p.windows_.size());
        for (size_t i = 0; i < p.windows_.size(); ++i) {
            const racon::Window& w = *p.windows_[i];
            rb_window& r = views[i];
            r.backbone = w.backbone;
            r.backbone_quality = w.quality;
            r.backbone_length = w.backbone_length;
            r.n_layers = uint32_t(w.seqs.size());
            r.layers = w.seqs.data();
            r.layer_qualities = w.quals.data();
            r.layer_lengths = w.lens.data();
            r.begins = w.begins.data();
            r.ends = w.ends.data();
            r.tgs = p.tgs_ ? 1 : 0;
            r.id = w.id;
            r.rank = w.rank;
        }
        for (int i = 0; i < 3; ++i) stage_s[i] = p.stage_s_[i];
    }
};

extern "C" rb_job* rb_job_prepare(const char* sequences_path, const char* overlaps_path, const char* target_path,
                                  int fragment, uint32_t window_length, double quality_threshold,
                                  double error_threshold, int8_t match, int8_t mismatch, int8_t gap, int device,
                                  double* stage_seconds) {
    if (!sequences_path || !overlaps_path || !target_path) return nullptr;
    racon::g_throw_on_error = true;
    std::string dev = std::to_string(device);
    setenv("RACON_B200_DEVICE", dev.c_str(), 1);
    try {
        std::unique_ptr<rb_job> job(new rb_job());
        job->polisher = racon::createPolisher(sequences_path, overlaps_path, target_path,
                                              fragment ? racon::PolisherType::kF : racon::PolisherType::kC,
                                              window_length, quality_threshold, error_threshold, true, match,
                                              mismatch, gap, 1);
        job->polisher->initialize();
        job->collect();
        if (stage_seconds)
            for (int i = 0; i < 3; ++i) stage_seconds[i] = job->stage_s[i];
        racon::g_throw_on_error = false;
        return job.release();
    } catch (const racon::Fatal& e) {
        racon::g_throw_on_error = false;
        g_pipeline_error = e.what();
        return nullptr;
    }
}

extern "C" size_t rb_job_windows(const rb_job* job, const rb_window** windows) {
    if (!job || !windows) return 0;
    *windows = job->views.data();
    return job->views.size();
}

extern "C" int rb_job_layer_input(const rb_job* job, const rb_sequence** sequences, size_t* n_sequences,
                                  size_t* n_targets, const rb_layer_overlap** overlaps, size_t* n_overlaps,
                                  const uint32_t** breakpoints, const uint64_t** bp_offsets, int* tgs) {
    if (!job || !sequences || !n_sequences || !n_targets || !overlaps || !n_overlaps || !breakpoints ||
        !bp_offsets || !tgs)
        return RB_ERR_ARG;
    const racon::Polisher& p = *job->polisher;
    *sequences = p.sequence_table_.data();
    *n_sequences = p.sequence_table_.size();
    *n_targets = p.targets_coverages_.size();
    *overlaps = p.layer_overlaps_.data();
    *n_overlaps = p.layer_overlaps_.size();
    *breakpoints = p.breakpoints_.data();
    *bp_offsets = p.bp_offsets_.data();
    *tgs = p.tgs_ ? 1 : 0;
    return RB_OK;
}

extern "C" rb_ctx* rb_job_context(const rb_job* job) { return job ? job->polisher->ctx_ : nullptr; }

extern "C" void rb_job_free(rb_job* job) { delete job; }
