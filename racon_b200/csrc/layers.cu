// Device-side layer assembly with the semantics of racon's
//   src/polisher.cpp:384-399  windows over the targets
//   src/polisher.cpp:401-457  breaking points -> window layers
//   src/sequence.cpp:49-84    reverse complement and reversed quality
//   src/window.cpp:42-63      Window::add_layer (skips and position checks)
//   src/window.cpp:78-85      layer order inside a window (std::sort by begin)
//
// Design (B200, sm_100a). The sequence table (targets, then reads) lives in
// one device byte store: forward bases and qualities are copied once, the
// reverse complement and the reversed quality of every sequence an overlap
// uses on the '-' strand are built on the device. Layers are never copied:
// a layer record is an (offset, length) view into the store, as racon's
// Window keeps (const char*, uint32_t) views into its Sequence strings.
//
//   candidates  one warp per overlap walks its breaking-point pairs; for each
//               pair it applies racon's two filters (query span below
//               0.02 * w; mean Phred-33 quality below -q, summed by the warp
//               in exact integer arithmetic and divided once in fp64, which
//               gives racon's double accumulate bit for bit because every
//               partial sum is an integer below 2^53), then add_layer's skip
//               (begin == end), and counts the window's layers.
//   scan        exclusive sum of the per-window counts (one CTA).
//   place       each kept candidate takes a slot in its window's range.
//   order       one warp per window restores overlap order inside the range
//               (the order racon's add_layer calls append in) by ranking the
//               candidate indices, and gathers the begin positions.
//   host sort   racon's std::sort of the window's layers by begin is not
//               stable, so the order of equal begins is libstdc++'s: the host
//               runs that same call on the 2-byte begin keys (nothing else
//               leaves the device) and sends back the permutation.
//   gather      one warp per window writes its layer records in that order.
// The window records then go to PoaEngine::stage_device, whose kernels read
// the bases and qualities straight from the store.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "rb_internal.hpp"

namespace rb {
namespace {

constexpr uint64_t kNone = kNotStaged;
constexpr uint32_t kDropped = ~0u;

// Errors found by the kernels; the first one is kept with its overlap index.
enum LayerStatus : uint32_t {
    kLsOk = 0,
    kLsBadIds = 1,         // q_id / t_id out of range, or the strand was not staged
    kLsBadPoints = 2,      // breaking points outside their read or target, or not increasing
    kLsBadPositions = 3,   // add_layer's position check (src/window.cpp:54-58)
    kLsEndOnLast = 4,      // layer end on the backbone's last base + 1
    kLsLongLayer = 5,      // layer longer than 65535 bases
    kLsManyPoints = 6,     // more breaking-point pairs than candidate slots
    kLsBadQuality = 7,     // a quality byte outside '!'..'~' in a kept layer or a backbone
};

struct OvlDev {
    uint64_t bp_off;   // first uint32 of the overlap's breaking points
    uint64_t cand;     // first candidate slot
    uint32_t q_id, t_id;
    uint32_t strand;
    uint32_t cnt;      // uint32 values of breaking points (when no count array is given)
    uint32_t cnt_idx;  // index into the count array
    uint32_t cap;      // candidate slots
};

struct CandArgs {
    const uint8_t* store;
    const SeqDev* seqs;
    uint32_t nseq;
    uint32_t n_targets;
    const uint64_t* first_window;  // per target, n_targets + 1
    uint32_t w;
    double min_span;               // 0.02 * w
    double q_threshold;
    const OvlDev* ovl;
    uint32_t novl;
    const uint32_t* bp;
    const uint32_t* bpcnt;         // nullptr: OvlDev::cnt
    PoaLayerDev* cand;
    uint32_t* cand_win;
    uint32_t* win_cnt;
    uint32_t* status;              // [0] LayerStatus, [1] overlap index
};

__device__ __forceinline__ void report(uint32_t* status, uint32_t code, uint32_t ovl) {
    if (atomicCAS(status, 0u, code) == 0u) status[1] = ovl;
}

__device__ __forceinline__ uint8_t complement(uint8_t c) {
    // A <-> T, C <-> G, every other byte unchanged (src/sequence.cpp:58-75)
    return c == 'A' ? 'T' : c == 'T' ? 'A' : c == 'C' ? 'G' : c == 'G' ? 'C' : c;
}

// Reverse complement and reversed quality of the listed sequences, one block
// per sequence at a time.
__global__ void __launch_bounds__(256) revcomp_kernel(uint8_t* store, const SeqDev* seqs, const uint32_t* list,
                                                     uint32_t n) {
    for (uint32_t b = blockIdx.x; b < n; b += gridDim.x) {
        const SeqDev s = seqs[list[b]];
        const uint8_t* f = store + s.fwd;
        uint8_t* r = store + s.rev;
        for (uint32_t k = threadIdx.x; k < s.len; k += blockDim.x) r[k] = complement(f[s.len - 1 - k]);
        if (s.rq != kNone) {
            const uint8_t* fq = store + s.fq;
            uint8_t* rq = store + s.rq;
            for (uint32_t k = threadIdx.x; k < s.len; k += blockDim.x) rq[k] = fq[s.len - 1 - k];
        }
    }
}

// One warp per overlap: racon's loop over breaking-point pairs
// (src/polisher.cpp:410-456).
__global__ void __launch_bounds__(256) layer_candidates_kernel(CandArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; o < a.novl; o += nwarps) {
        const OvlDev ov = a.ovl[o];
        const uint32_t cnt = a.bpcnt ? a.bpcnt[ov.cnt_idx] : ov.cnt;
        const uint32_t npair = cnt / 4;
        for (uint32_t p = lane; p < ov.cap; p += 32) a.cand_win[ov.cand + p] = kDropped;
        __syncwarp();
        if (ov.q_id >= a.nseq || ov.t_id >= a.n_targets) {
            if (lane == 0) report(a.status, kLsBadIds, o);
            continue;
        }
        if (npair > ov.cap || (cnt & 3u)) {
            if (lane == 0) report(a.status, kLsManyPoints, o);
            continue;
        }
        const SeqDev q = a.seqs[ov.q_id];
        const SeqDev t = a.seqs[ov.t_id];
        const uint64_t data = ov.strand ? q.rev : q.fwd;
        const uint64_t qual = q.fq == kNone ? kNone : (ov.strand ? q.rq : q.fq);
        if ((npair > 0 && data == kNone) || t.fwd == kNone) {
            if (lane == 0) report(a.status, kLsBadIds, o);
            continue;
        }
        const uint64_t fw = a.first_window[ov.t_id];
        for (uint32_t p = 0; p < npair; ++p) {
            const uint32_t* b = a.bp + ov.bp_off + 4ull * p;
            const uint32_t t0 = b[0], q0 = b[1], t1 = b[2], q1 = b[3];
            if (!(t0 < t1 && t1 <= t.len && q0 < q1 && q1 <= q.len)) {
                if (lane == 0) report(a.status, kLsBadPoints, o);
                break;
            }
            const uint32_t span = q1 - q0;
            bool keep = !(double(span) < a.min_span);
            bool bad_quality = false;
            if (keep && qual != kNone) {
                // sum of (uint32)quality - 33 over the span (racon's loop adds
                // each term to a double; all partial sums are exact integers)
                const uint8_t* qs = a.store + qual + q0;
                unsigned long long s = 0;
                bool bad = false;
                for (uint32_t k = lane; k < span; k += 32) {
                    s += uint32_t(int32_t(int8_t(qs[k]))) - 33u;
                    bad |= uint32_t(qs[k]) - 33u > 93u;
                }
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
                bad_quality = __any_sync(0xffffffffu, bad);
                const double avg = double(s) / double(span);
                keep = !(avg < a.q_threshold);
            }
            if (!keep || lane != 0) continue;
            const uint32_t rank = t0 / a.w;
            const uint32_t ws = rank * a.w;
            const uint32_t bb_len = min(a.w, t.len - ws);
            const uint32_t begin = t0 - ws, end = t1 - ws - 1;
            if (begin == end) continue;  // add_layer ignores it (src/window.cpp:45-47)
            if (begin >= end || begin > bb_len || end > bb_len) {
                report(a.status, kLsBadPositions, o);
                continue;
            }
            if (end == bb_len) {
                report(a.status, kLsEndOnLast, o);
                continue;
            }
            if (span > 65535u) {
                report(a.status, kLsLongLayer, o);
                continue;
            }
            if (bad_quality) {
                report(a.status, kLsBadQuality, o);
                continue;
            }
            const uint64_t c = ov.cand + p;
            PoaLayerDev L;
            L.seq_off = data + q0;
            L.qual_off = qual == kNone ? kNoQual : qual + q0;
            L.len = span;
            L.begin = begin;
            L.end = end;
            L.pad = 0;
            a.cand[c] = L;
            const uint32_t win = uint32_t(fw + rank);
            a.cand_win[c] = win;
            atomicAdd(a.win_cnt + win, 1u);
        }
    }
}

// Backbone qualities: every quality byte of targets 0 .. n-1 within '!'..'~'
// (the window consensus weights are Phred values 0..93), one block per
// target at a time.
__global__ void __launch_bounds__(256) quality_check_kernel(const uint8_t* store, const SeqDev* seqs, uint32_t n,
                                                            uint32_t* status) {
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const SeqDev s = seqs[t];
        if (s.fq == kNone) continue;
        const uint8_t* q = store + s.fq;
        bool bad = false;
        for (uint32_t k = threadIdx.x; k < s.len; k += blockDim.x) bad |= uint32_t(q[k]) - 33u > 93u;
        if (__syncthreads_or(bad) && threadIdx.x == 0) report(status, kLsBadQuality, t);
    }
}

// Exclusive prefix sum of n counts into base (one CTA of 1024 threads, tiles
// of 4096 with a running carry); base[n] = total.
// One small block: a kernel of this context must fit beside the persistent
// kernels that other contexts (the serving loop's shared consensus kernel)
// keep resident, or it would wait for them to drain.
constexpr int kScanThreads = 256;
constexpr int kScanWarps = kScanThreads / 32;

__global__ void __launch_bounds__(kScanThreads) scan_kernel(const uint32_t* cnt, uint64_t* base, uint32_t n) {
    __shared__ unsigned long long warp_sum[32];
    __shared__ unsigned long long carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t t0 = 0; t0 < n; t0 += kScanThreads * 4) {
        uint32_t v[4];
        unsigned long long s = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t i = t0 + threadIdx.x * 4 + u;
            v[u] = i < n ? cnt[i] : 0u;
            s += v[u];
        }
        // inclusive scan of the thread sums
        unsigned long long x = s;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warp_sum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            unsigned long long z = lane < kScanWarps ? warp_sum[lane] : 0ull;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, z, d);
                if (lane >= d) z += y;
            }
            warp_sum[lane] = z;
        }
        __syncthreads();
        unsigned long long run = carry + (wid > 0 ? warp_sum[wid - 1] : 0ull) + x - s;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t i = t0 + threadIdx.x * 4 + u;
            if (i < n) base[i] = run;
            run += v[u];
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sum[kScanWarps - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) base[n] = carry;
}

__global__ void __launch_bounds__(256) place_kernel(const uint32_t* cand_win, uint64_t ncand, const uint64_t* base,
                                                    uint32_t* fill, uint32_t* placed) {
    for (uint64_t c = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; c < ncand;
         c += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t w = cand_win[c];
        if (w == kDropped) continue;
        const uint32_t p = atomicAdd(fill + w, 1u);
        placed[base[w] + p] = uint32_t(c);
    }
}

// One warp per window: candidate indices of the window in increasing order
// (overlap order, then pair order), their begins, the layers' total and
// largest length.
__global__ void __launch_bounds__(256) order_kernel(const uint32_t* placed, const uint64_t* base, uint32_t nwin,
                                                    const PoaLayerDev* cand, uint32_t* ordered, uint16_t* begins,
                                                    unsigned long long* sum_len, uint32_t* max_len) {
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwin; w += nwarps) {
        const uint64_t b = base[w];
        const uint32_t n = uint32_t(base[w + 1] - b);
        unsigned long long s = 0;
        uint32_t mx = 0;
        for (uint32_t i = lane; i < n; i += 32) {
            const uint32_t c = placed[b + i];
            uint32_t r = 0;
            for (uint32_t k = 0; k < n; ++k) r += placed[b + k] < c ? 1u : 0u;
            const PoaLayerDev L = cand[c];
            ordered[b + r] = c;
            begins[b + r] = uint16_t(L.begin);
            s += L.len;
            mx = max(mx, L.len);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, d);
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        }
        if (lane == 0) {
            sum_len[w] = s;
            if (mx) atomicMax(max_len, mx);
        }
    }
}

__global__ void __launch_bounds__(256) gather_kernel(const uint32_t* ordered, const uint16_t* perm,
                                                     const uint64_t* base, uint32_t nwin, const PoaLayerDev* cand,
                                                     PoaLayerDev* out) {
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nwin; w += nwarps) {
        const uint64_t b = base[w];
        const uint32_t n = uint32_t(base[w + 1] - b);
        for (uint32_t j = lane; j < n; j += 32) out[b + j] = cand[ordered[b + perm[b + j]]];
    }
}

int grid_for(const DeviceInfo& dev, uint64_t warps_needed, int warps_per_block) {
    const uint64_t blocks = (warps_needed + warps_per_block - 1) / warps_per_block;
    return int(std::max<uint64_t>(1, std::min<uint64_t>(blocks, uint64_t(dev.sm_count) * 16)));
}

uint64_t align16(uint64_t x) { return (x + 15) & ~uint64_t(15); }

}  // namespace

LayerEngine::LayerEngine(const DeviceInfo& dev, cudaStream_t stream) : dev_(dev), stream_(stream) {
    check_cuda(cudaEventCreate(&ev0_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1_), "cudaEventCreate");
    const void* kernels[] = {reinterpret_cast<const void*>(revcomp_kernel),
                             reinterpret_cast<const void*>(layer_candidates_kernel),
                             reinterpret_cast<const void*>(quality_check_kernel),
                             reinterpret_cast<const void*>(scan_kernel), reinterpret_cast<const void*>(place_kernel),
                             reinterpret_cast<const void*>(order_kernel), reinterpret_cast<const void*>(gather_kernel)};
    for (const void* k : kernels) prefer_max_shared(k);
}

LayerEngine::~LayerEngine() {
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
}

void LayerEngine::stage_sequences(const rb_sequence* seqs, size_t n, PoaEngine& poa) {
    if (n > 0 && !seqs) throw Error{RB_ERR_ARG, "rb_sequences_stage: sequences is NULL"};
    if (n >= kDropped) throw Error{RB_ERR_ARG, "rb_sequences_stage: too many sequences"};
    // the staged windows read the store that is about to change
    poa.forget();
    nseq_ = 0;
    std::vector<SeqDev> tab(n);
    std::vector<uint32_t> rev_list;
    uint64_t up = 0;
    for (size_t i = 0; i < n; ++i) {
        const rb_sequence& s = seqs[i];
        SeqDev& d = tab[i];
        d.fwd = d.fq = d.rev = d.rq = kNone;
        d.len = s.length;
        d.pad = 0;
        if (!s.forward && !s.reverse) continue;
        if (s.length > 0 && !s.data) throw Error{RB_ERR_ARG, "rb_sequences_stage: NULL data with nonzero length"};
        d.fwd = up;
        up += align16(s.length);
        if (s.quality) {
            d.fq = up;
            up += align16(s.length);
        }
    }
    uint64_t dev_bytes = up;
    for (size_t i = 0; i < n; ++i) {
        if (!seqs[i].reverse) continue;
        SeqDev& d = tab[i];
        d.rev = dev_bytes;
        dev_bytes += align16(d.len);
        if (d.fq != kNone) {
            d.rq = dev_bytes;
            dev_bytes += align16(d.len);
        }
        if (d.len) rev_list.push_back(uint32_t(i));
    }
    h_store_.reserve(std::max<uint64_t>(up, 16));
    uint8_t* h = h_store_.as<uint8_t>();
    auto copy_range = [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            const SeqDev& d = tab[i];
            if (d.fwd == kNone || d.len == 0) continue;
            memcpy(h + d.fwd, seqs[i].data, d.len);
            if (d.fq != kNone) memcpy(h + d.fq, seqs[i].quality, d.len);
        }
    };
    const unsigned nth = up > (uint64_t(32) << 20) ? std::max(1u, std::min(8u, std::thread::hardware_concurrency())) : 1u;
    if (nth == 1) {
        copy_range(0, n);
    } else {
        // ranges of about equal bytes
        std::vector<std::thread> pool;
        size_t b = 0;
        for (unsigned k = 0; k < nth && b < n; ++k) {
            const uint64_t goal = up * (k + 1) / nth;
            size_t e = b;
            while (e < n && (k + 1 == nth || tab[e].fwd == kNone || tab[e].fwd < goal)) ++e;
            pool.emplace_back(copy_range, b, e);
            b = e;
        }
        if (b < n) copy_range(b, n);
        for (auto& th : pool) th.join();
    }
    d_store_.reserve(std::max<uint64_t>(dev_bytes, 16));
    d_seqs_.reserve(std::max<size_t>(n, 1) * sizeof(SeqDev));
    d_list_.reserve(std::max<size_t>(rev_list.size(), 1) * 4);
    h_misc_.reserve(std::max<size_t>(n, 1) * sizeof(SeqDev) + std::max<size_t>(rev_list.size(), 1) * 4);
    memcpy(h_misc_.ptr, tab.data(), n * sizeof(SeqDev));
    uint32_t* hl = reinterpret_cast<uint32_t*>(h_misc_.as<uint8_t>() + n * sizeof(SeqDev));
    if (!rev_list.empty()) memcpy(hl, rev_list.data(), rev_list.size() * 4);
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (up) check_cuda(cudaMemcpyAsync(d_store_.ptr, h, up, cudaMemcpyHostToDevice, stream_), "H2D sequences");
    if (n)
        check_cuda(cudaMemcpyAsync(d_seqs_.ptr, h_misc_.ptr, n * sizeof(SeqDev), cudaMemcpyHostToDevice, stream_),
                   "H2D sequence table");
    if (!rev_list.empty()) {
        check_cuda(cudaMemcpyAsync(d_list_.ptr, hl, rev_list.size() * 4, cudaMemcpyHostToDevice, stream_),
                   "H2D reverse list");
        const int grid = int(std::min<size_t>(rev_list.size(), size_t(dev_.sm_count) * 8));
        revcomp_kernel<<<grid, 256, 0, stream_>>>(d_store_.as<uint8_t>(), d_seqs_.as<SeqDev>(),
                                                  d_list_.as<uint32_t>(), uint32_t(rev_list.size()));
        check_cuda(cudaGetLastError(), "revcomp_kernel");
    }
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaStreamSynchronize(stream_), "sequences sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    seq_stats_ = rb_stats{};
    seq_stats_.h2d_ms = ms;
    seq_stats_.h2d_bytes = up + n * sizeof(SeqDev) + rev_list.size() * 4;
    seq_stats_.launches = rev_list.empty() ? 0 : 1;
    seq_stats_.items = n;
    lens_.resize(n);
    fwd_.resize(n);
    fq_.resize(n);
    for (size_t i = 0; i < n; ++i) {
        lens_[i] = tab[i].len;
        fwd_[i] = tab[i].fwd;
        fq_[i] = tab[i].fq;
    }
    store_bytes_ = dev_bytes;
    host_tab_ = std::move(tab);
    nseq_ = n;
}

SeqStore LayerEngine::store() const {
    SeqStore st;
    st.bytes = d_store_.as<uint8_t>();
    st.seqs = d_seqs_.as<SeqDev>();
    st.host = host_tab_.data();
    st.n = nseq_;
    return st;
}

void LayerEngine::assemble_aligned(size_t n_targets, const rb_store_pair* pairs, size_t n, uint32_t window_length,
                                   double quality_threshold, int tgs, int trim, NwEngine& nw, PoaEngine& poa,
                                   rb_aln_result* out) {
    poa.forget();
    if (n > 0 && !pairs) throw Error{RB_ERR_ARG, "rb_poa_stage_alignments: pairs is NULL"};
    if (n_targets > nseq_) throw Error{RB_ERR_ARG, "rb_poa_stage_alignments: more targets than staged sequences"};
    if (window_length == 0) throw Error{RB_ERR_ARG, "rb_poa_stage_alignments: window length is 0"};
    // candidate slots in overlap order: one per window the target span
    // touches (the aligner's breaking-point slots)
    std::vector<uint64_t> cand(n + 1, 0);
    for (size_t i = 0; i < n; ++i) {
        const uint32_t tb = pairs[i].t_begin, te = pairs[i].t_end;
        const uint64_t segs = te > tb ? (uint64_t(te) - 1) / window_length - tb / window_length + 1 : 0;
        cand[i + 1] = cand[i] + segs;
    }
    if (cand[n] >= kDropped) throw Error{RB_ERR_ARG, "rb_poa_stage_alignments: more than 2^32 - 1 layer candidates"};
    begin(n_targets, window_length, quality_threshold, cand[n]);
    if (out) {
        out_dist_.clear();
        out_bp_.clear();
        out_bp_off_.assign(1, 0);
    }
    const SeqStore st = store();
    // batches bounded by bases so the aligner's buffers stay modest;
    // RB_ALIGN_BATCH_BASES lowers the bound (tests of the multi-batch path);
    // results do not depend on it
    uint64_t kBatchBases = uint64_t(1) << 31;
    if (const char* e = getenv("RB_ALIGN_BATCH_BASES")) kBatchBases = std::max<uint64_t>(1, strtoull(e, nullptr, 10));
    std::vector<OvlDev> od;
    size_t b = 0;
    while (b < n) {
        size_t e = b;
        uint64_t bases = 0;
        while (e < n) {
            const uint64_t pb = uint64_t(pairs[e].q_end - pairs[e].q_begin) + (pairs[e].t_end - pairs[e].t_begin);
            if (e > b && bases + pb > kBatchBases) break;
            bases += pb;
            ++e;
        }
        nw.stage_store(pairs + b, e - b, 0, window_length, st);
        nw.run();
        const NwPairDev* pd = nw.pairs();
        od.resize(e - b);
        for (size_t k = 0; k < e - b; ++k) {
            const rb_store_pair& p = pairs[b + k];
            OvlDev& d = od[k];
            d.bp_off = pd[k].bp_off;
            d.cand = cand[b + k];
            d.q_id = p.q_id;
            d.t_id = p.t_id;
            d.strand = p.strand ? 1u : 0u;
            d.cnt = 0;
            d.cnt_idx = uint32_t(k);
            d.cap = uint32_t(cand[b + k + 1] - cand[b + k]);
        }
        h_bp_.reserve(od.size() * sizeof(OvlDev));
        memcpy(h_bp_.ptr, od.data(), od.size() * sizeof(OvlDev));
        d_ovl_.reserve(od.size() * sizeof(OvlDev));
        check_cuda(cudaMemcpyAsync(d_ovl_.ptr, h_bp_.ptr, od.size() * sizeof(OvlDev), cudaMemcpyHostToDevice,
                                   stream_),
                   "H2D overlaps");
        stats_.h2d_bytes += od.size() * sizeof(OvlDev);
        add_candidates(nw.bp_slots(), nw.bp_counts(), d_ovl_.ptr, e - b);
        if (out) {
            rb_aln_result r;
            nw.fetch(&r);
            for (size_t k = 0; k < e - b; ++k) {
                out_dist_.push_back(r.edit_distance[k]);
                out_bp_.insert(out_bp_.end(), r.breakpoints + r.bp_offsets[k], r.breakpoints + r.bp_offsets[k + 1]);
                out_bp_off_.push_back(out_bp_.size());
            }
        }
        b = e;
    }
    finish(tgs, trim, poa);
    if (out) {
        out->edit_distance = out_dist_.data();
        out->breakpoints = out_bp_.data();
        out->bp_offsets = out_bp_off_.data();
        out->cigars = nullptr;
        out->cigar_offsets = nullptr;
    }
}

void LayerEngine::assemble(size_t n_targets, const rb_layer_overlap* ovl, size_t n, const uint32_t* bps,
                           const uint64_t* bp_offsets, uint32_t window_length, double quality_threshold, int tgs,
                           int trim, PoaEngine& poa) {
    poa.forget();
    if (n > 0 && (!ovl || !bp_offsets)) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: NULL overlap arrays"};
    if (n_targets > nseq_) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: more targets than staged sequences"};
    if (window_length == 0) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: window length is 0"};
    // overlap records and breaking points
    uint64_t nbp = n ? bp_offsets[n] - bp_offsets[0] : 0;
    if (nbp > 0 && !bps) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: breakpoints is NULL"};
    std::vector<OvlDev> od(n);
    uint64_t cand = 0;
    for (size_t i = 0; i < n; ++i) {
        if (bp_offsets[i + 1] < bp_offsets[i])
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: breakpoint offsets decrease"};
        const uint64_t cnt = bp_offsets[i + 1] - bp_offsets[i];
        if (cnt % 4 != 0 || cnt > 0xFFFFFFFCull)
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: breakpoints must come as (first, last) pairs"};
        OvlDev& d = od[i];
        d.bp_off = bp_offsets[i] - bp_offsets[0];
        d.cand = cand;
        d.q_id = ovl[i].q_id;
        d.t_id = ovl[i].t_id;
        d.strand = ovl[i].strand ? 1u : 0u;
        d.cnt = uint32_t(cnt);
        d.cnt_idx = uint32_t(i);
        d.cap = uint32_t(cnt / 4);
        cand += d.cap;
    }
    if (cand >= kDropped) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: more than 2^32 - 1 layer candidates"};
    begin(n_targets, window_length, quality_threshold, cand);
    d_bp_.reserve(std::max<uint64_t>(nbp, 1) * 4);
    h_bp_.reserve(std::max<uint64_t>(nbp, 1) * 4 + std::max<size_t>(n, 1) * sizeof(OvlDev));
    if (nbp) memcpy(h_bp_.ptr, bps + bp_offsets[0], nbp * 4);
    uint8_t* ho = h_bp_.as<uint8_t>() + nbp * 4;
    if (n) memcpy(ho, od.data(), n * sizeof(OvlDev));
    d_ovl_.reserve(std::max<size_t>(n, 1) * sizeof(OvlDev));
    if (nbp)
        check_cuda(cudaMemcpyAsync(d_bp_.ptr, h_bp_.ptr, nbp * 4, cudaMemcpyHostToDevice, stream_), "H2D breakpoints");
    if (n)
        check_cuda(cudaMemcpyAsync(d_ovl_.ptr, ho, n * sizeof(OvlDev), cudaMemcpyHostToDevice, stream_),
                   "H2D overlaps");
    stats_.h2d_bytes += nbp * 4 + n * sizeof(OvlDev);
    add_candidates(d_bp_.as<uint32_t>(), nullptr, d_ovl_.ptr, n);
    finish(tgs, trim, poa);
}

void LayerEngine::begin(size_t n_targets, uint32_t window_length, double quality_threshold, uint64_t cand_cap) {
    stats_ = rb_stats{};
    n_targets_ = n_targets;
    w_ = window_length;
    q_threshold_ = quality_threshold;
    // windows over the targets (src/polisher.cpp:384-399)
    first_window_.assign(n_targets + 1, 0);
    for (size_t t = 0; t < n_targets; ++t) {
        if (lens_[t] > 0 && fwd_[t] == kNone)
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: target sequence not staged"};
        first_window_[t + 1] = first_window_[t] + (uint64_t(lens_[t]) + w_ - 1) / w_;
    }
    nwin_ = first_window_[n_targets];
    if (nwin_ >= kDropped) throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: more than 2^32 - 1 windows"};
    cand_cap_ = cand_cap;
    d_cand_.reserve(std::max<uint64_t>(cand_cap, 1) * sizeof(PoaLayerDev));
    d_cand_win_.reserve(std::max<uint64_t>(cand_cap, 1) * 4);
    d_win_.reserve((nwin_ + 1) * (4 + 4 + 8 + 8) + 64);
    d_fw_.reserve((n_targets + 1) * 8);
    h_fw_.reserve((n_targets + 1) * 8);
    memcpy(h_fw_.ptr, first_window_.data(), (n_targets + 1) * 8);
    check_cuda(cudaMemcpyAsync(d_fw_.ptr, h_fw_.ptr, (n_targets + 1) * 8, cudaMemcpyHostToDevice, stream_),
               "H2D first windows");
    batches_ = 0;
    cand_ms_ = 0;
    // counts, fill, base, sums, and the status words in one zeroed range
    check_cuda(cudaMemsetAsync(d_win_.ptr, 0, d_win_.bytes, stream_), "memset windows");
    stats_.h2d_bytes += (n_targets + 1) * 8;
}

uint32_t* LayerEngine::win_cnt() const { return d_win_.as<uint32_t>(); }
uint32_t* LayerEngine::win_fill() const { return d_win_.as<uint32_t>() + (nwin_ + 1); }
uint64_t* LayerEngine::win_base() const {
    return reinterpret_cast<uint64_t*>(d_win_.as<uint8_t>() + ((nwin_ + 1) * 8 + 7) / 8 * 8);
}
unsigned long long* LayerEngine::win_sum() const {
    return reinterpret_cast<unsigned long long*>(win_base() + (nwin_ + 1));
}
uint32_t* LayerEngine::status() const { return reinterpret_cast<uint32_t*>(win_sum() + (nwin_ + 1)); }

void LayerEngine::add_candidates(const uint32_t* d_bp, const uint32_t* d_bpcnt, const void* d_ovl, size_t n) {
    if (n == 0) return;
    CandArgs a;
    a.store = d_store_.as<uint8_t>();
    a.seqs = d_seqs_.as<SeqDev>();
    a.nseq = uint32_t(nseq_);
    a.n_targets = uint32_t(n_targets_);
    a.first_window = d_fw_.as<uint64_t>();
    a.w = w_;
    a.min_span = 0.02 * w_;
    a.q_threshold = q_threshold_;
    a.ovl = static_cast<const OvlDev*>(d_ovl);
    a.novl = uint32_t(n);
    a.bp = d_bp;
    a.bpcnt = d_bpcnt;
    a.cand = d_cand_.as<PoaLayerDev>();
    a.cand_win = d_cand_win_.as<uint32_t>();
    a.win_cnt = win_cnt();
    a.status = status();
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    layer_candidates_kernel<<<grid_for(dev_, n, 8), 256, 0, stream_>>>(a);
    check_cuda(cudaGetLastError(), "layer_candidates_kernel");
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(ev1_), "candidates sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    cand_ms_ += ms;
    ++batches_;
    ++stats_.launches;
}

void LayerEngine::finish(int tgs, int trim, PoaEngine& poa) {
    const uint32_t nw = uint32_t(nwin_);
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    if (n_targets_) {
        const int grid = int(std::min<size_t>(n_targets_, size_t(dev_.sm_count) * 8));
        quality_check_kernel<<<grid, 256, 0, stream_>>>(d_store_.as<uint8_t>(), d_seqs_.as<SeqDev>(),
                                                         uint32_t(n_targets_), status());
        check_cuda(cudaGetLastError(), "quality_check_kernel");
        ++stats_.launches;
    }
    scan_kernel<<<1, kScanThreads, 0, stream_>>>(win_cnt(), win_base(), nw);
    check_cuda(cudaGetLastError(), "scan_kernel");
    ++stats_.launches;
    // totals and status before the layer-sized buffers
    h_misc_.reserve(64);
    uint64_t* hm = h_misc_.as<uint64_t>();
    check_cuda(cudaMemcpyAsync(hm, win_base() + nw, 8, cudaMemcpyDeviceToHost, stream_), "D2H layer total");
    check_cuda(cudaMemcpyAsync(hm + 1, status(), 16, cudaMemcpyDeviceToHost, stream_), "D2H status");
    check_cuda(cudaStreamSynchronize(stream_), "layers sync");
    const uint64_t nlayers = hm[0];
    const uint32_t* st = reinterpret_cast<const uint32_t*>(hm + 1);
    if (st[0] != kLsOk) {
        const uint32_t code = st[0], o = st[1];
        const std::string at = " (overlap " + std::to_string(o) + ")";
        switch (code) {
        case kLsBadPositions:
            throw Error{RB_ERR_ARG, "[racon::Window::add_layer] error: layer begin and end positions are invalid!" + at};
        case kLsEndOnLast:
            throw Error{RB_ERR_ARG, "rb_poa: layer begin and end positions are invalid" + at};
        case kLsLongLayer:
            throw Error{RB_ERR_ARG, "rb_poa: empty, NULL or over-long layer" + at};
        case kLsBadPoints:
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: breaking points outside their read or target" + at};
        case kLsBadQuality:
            throw Error{RB_ERR_ARG, "rb_poa: quality values outside '!'..'~' (Phred+33 0..93)" + at};
        case kLsManyPoints:
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: more breaking-point pairs than candidate slots" + at};
        default:
            throw Error{RB_ERR_ARG, "rb_poa_stage_overlaps: read or target id out of range, or strand not staged" + at};
        }
    }
    d_lay_.reserve(std::max<uint64_t>(nlayers, 1) * (4 + 4 + 2 + 2) + 64);
    d_final_.reserve(std::max<uint64_t>(nlayers, 1) * sizeof(PoaLayerDev));
    uint32_t* placed = d_lay_.as<uint32_t>();
    uint32_t* ordered = placed + nlayers;
    uint16_t* begins = reinterpret_cast<uint16_t*>(ordered + nlayers);
    uint16_t* perm = begins + nlayers;
    uint32_t* max_len = status() + 2;
    place_kernel<<<grid_for(dev_, (cand_cap_ + 31) / 32, 8), 256, 0, stream_>>>(d_cand_win_.as<uint32_t>(), cand_cap_,
                                                                             win_base(), win_fill(), placed);
    check_cuda(cudaGetLastError(), "place_kernel");
    order_kernel<<<grid_for(dev_, nw, 8), 256, 0, stream_>>>(placed, win_base(), nw, d_cand_.as<PoaLayerDev>(),
                                                            ordered, begins, win_sum(), max_len);
    check_cuda(cudaGetLastError(), "order_kernel");
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    stats_.launches += 2;
    // begins, counts and sums to the host
    const size_t hb = nlayers * 2 + (nw + 1) * 8 + nw * 8 + 64;
    h_lay_.reserve(hb);
    uint16_t* h_begin = h_lay_.as<uint16_t>();
    uint64_t* h_base = reinterpret_cast<uint64_t*>(h_lay_.as<uint8_t>() + (nlayers * 2 + 7) / 8 * 8);
    uint64_t* h_sum = h_base + (nw + 1);
    uint32_t* h_max = reinterpret_cast<uint32_t*>(h_sum + nw);
    if (nlayers)
        check_cuda(cudaMemcpyAsync(h_begin, begins, nlayers * 2, cudaMemcpyDeviceToHost, stream_), "D2H begins");
    check_cuda(cudaMemcpyAsync(h_base, win_base(), (nw + 1) * 8, cudaMemcpyDeviceToHost, stream_), "D2H bases");
    if (nw) check_cuda(cudaMemcpyAsync(h_sum, win_sum(), nw * 8, cudaMemcpyDeviceToHost, stream_), "D2H sums");
    check_cuda(cudaMemcpyAsync(h_max, max_len, 4, cudaMemcpyDeviceToHost, stream_), "D2H max length");
    check_cuda(cudaStreamSynchronize(stream_), "layers sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    float total_ms = cand_ms_ + ms;
    stats_.d2h_bytes += nlayers * 2 + (nw + 1) * 8 + nw * 8 + 4 + 24;
    // racon's per-window std::sort by begin (src/window.cpp:78-85) on the
    // host, on the begin keys in overlap order
    h_perm_.reserve(std::max<uint64_t>(nlayers, 1) * 2);
    uint16_t* h_perm = h_perm_.as<uint16_t>();
    for (uint32_t w = 0; w < nw; ++w)
        if (h_base[w + 1] - h_base[w] > 65535) throw Error{RB_ERR_ARG, "rb_poa: more than 65535 layers"};
    auto sort_range = [&](uint32_t w0, uint32_t w1) {
        std::vector<uint32_t> rank;
        for (uint32_t w = w0; w < w1; ++w) {
            const uint64_t b = h_base[w];
            const uint32_t m = uint32_t(h_base[w + 1] - b);
            const uint16_t* key = h_begin + b;
            rank.resize(size_t(m) + 1);
            for (uint32_t j = 0; j <= m; ++j) rank[j] = j;
            std::sort(rank.begin() + 1, rank.end(), [&](uint32_t lhs, uint32_t rhs) {
                const uint32_t x = lhs == 0 ? 0u : key[lhs - 1];
                const uint32_t y = rhs == 0 ? 0u : key[rhs - 1];
                return x < y;
            });
            for (uint32_t j = 1; j <= m; ++j) h_perm[b + j - 1] = uint16_t(rank[j] - 1);
        }
    };
    unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (nlayers < 200000) nth = 1;
    if (nth == 1) {
        sort_range(0, nw);
    } else {
        // ranges of about equal layer counts
        std::vector<std::thread> pool;
        uint32_t w0 = 0;
        for (unsigned k = 0; k < nth; ++k) {
            const uint64_t goal = h_base[0] + nlayers * (k + 1) / nth;
            // windows [w0, w1) start at or below goal
            const uint32_t idx = uint32_t(std::upper_bound(h_base, h_base + nw + 1, goal) - h_base) - 1;
            const uint32_t w1 = k + 1 == nth ? nw : std::max(w0, std::min(idx, nw));
            if (w1 > w0) pool.emplace_back(sort_range, w0, w1);
            w0 = w1;
        }
        for (auto& th : pool) th.join();
    }
    if (nlayers)
        check_cuda(cudaMemcpyAsync(perm, h_perm, nlayers * 2, cudaMemcpyHostToDevice, stream_), "H2D permutation");
    check_cuda(cudaEventRecord(ev0_, stream_), "cudaEventRecord");
    gather_kernel<<<grid_for(dev_, nw, 8), 256, 0, stream_>>>(ordered, perm, win_base(), nw, d_cand_.as<PoaLayerDev>(),
                                                             d_final_.as<PoaLayerDev>());
    check_cuda(cudaGetLastError(), "gather_kernel");
    ++stats_.launches;
    check_cuda(cudaEventRecord(ev1_, stream_), "cudaEventRecord");
    stats_.h2d_bytes += nlayers * 2;
    // window records (src/polisher.cpp:384-399; rb_poa_stage's layout)
    std::vector<PoaWinDev> wins(nw);
    std::vector<std::pair<uint64_t, uint32_t>> labels(nw);
    uint64_t oo = 0;
    for (size_t t = 0; t < n_targets_; ++t) {
        for (uint64_t wi = first_window_[t]; wi < first_window_[t + 1]; ++wi) {
            const uint32_t r = uint32_t(wi - first_window_[t]);
            const uint64_t ws = uint64_t(r) * w_;
            PoaWinDev& d = wins[wi];
            d.bb_len = uint32_t(std::min<uint64_t>(w_, lens_[t] - ws));
            if (d.bb_len > 65535) throw Error{RB_ERR_ARG, "rb_poa: backbone empty, NULL or longer than 65535"};
            d.bb_off = fwd_[t] + ws;
            d.bq_off = fq_[t] == kNone ? kNoQual : fq_[t] + ws;
            d.layer_base = h_base[wi];
            d.n_layers = uint32_t(h_base[wi + 1] - h_base[wi]);
            d.out_off = oo;
            d.out_cap = 3u * d.bb_len + 1024;
            oo += d.out_cap;
            d.offset = uint32_t(0.01 * d.bb_len);
            d.tgs = tgs ? 1u : 0u;
            d.pad = 0;
            labels[wi] = {uint64_t(t), r};
        }
    }
    check_cuda(cudaStreamSynchronize(stream_), "layers sync");
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    total_ms += ms;
    stats_.kernel_ms = total_ms;
    stats_.items = nlayers;
    stats_.top_kernel_ms = cand_ms_;
    stats_.cells = cand_cap_;
    poa.stage_device(d_store_.as<uint8_t>(), wins.data(), nw, d_final_.as<PoaLayerDev>(), h_sum, labels, *h_max,
                     trim);
}

}  // namespace rb
