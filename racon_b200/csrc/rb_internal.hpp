// Internal host-side interfaces shared by the C ABI (rb_capi.cpp) and the
// device engines (nw_align.cu, poa_consensus.cu). Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/racon_b200.h"

namespace rb {

// Error with an RB_ERR_* code; thrown inside the library, turned into a
// return code at the C ABI boundary.
struct Error {
    int code;
    std::string msg;
};

void check_cuda(cudaError_t e, const char* what);

// Growable device buffer, reused across calls. Inside a C ABI call it grows
// in the calling context's stream order (cudaMallocAsync / cudaFreeAsync), so
// growing never waits for other contexts' work on the device.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;  // stream of the allocation when stream-ordered
    bool stream_ordered = false;
    void reserve(size_t need);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
    ~DevBuf() { release(); }
};

// Growable pinned host buffer (outgrown buffers are freed with it).
struct HostBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    std::vector<void*> retired;
    void reserve(size_t need);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
    ~HostBuf() { release(); }
};

// Binds the calling thread's device-buffer growth to a context's stream for
// the duration of one C ABI call (rb_capi.cpp).
struct AllocStreamScope {
    explicit AllocStreamScope(cudaStream_t s);
    ~AllocStreamScope();
    cudaStream_t prev;
    bool prev_bound;
};

struct DeviceInfo {
    int device = 0;
    int sm_count = 148;
    size_t smem_optin = 0;
};

// Every kernel of the library asks for the largest shared-memory carveout, so
// an SM never has to change its L1/shared split between kernels. A change
// can only happen on an idle SM, so kernels of one context would otherwise
// wait for another context's resident persistent kernel (the serving loop's
// shared consensus kernel) to drain.
void prefer_max_shared(const void* kernel);
// The device's default memory pool keeps what it has reserved: trimming it
// at synchronisation points can wait for the device (and so for a resident
// persistent kernel). Called once per device when a context is created.
void keep_pool_reserve(int device);

// Launch choices of a device (rb_tuning), read by the engines at every run.
rb_tuning tuning_get(int device);
void tuning_set(int device, const rb_tuning& t);

// ----- shared work queue of a persistent kernel (ring_service.cpp) -----
// Continuous batching for the serving loop. Batches (one job's windows, or
// one pass of one job's alignments) are appended as (batch slot, index)
// items to size-class rings in device memory; a persistent kernel's warps
// claim items from the rings (ring 0 first) and report each one done; the
// last item of a batch raises the batch's flag in mapped host memory. The
// kernel leaves, as a whole, after a bounded idle time, and a dispatcher
// thread relaunches it while items are pending.
constexpr int kSvcQueues = 4;

// Every batch record starts with this header (filled in by run_batch).
struct SvcJobHead {
    uint32_t total;       // items in the batch
    uint32_t generation;  // value the last item writes to the batch's flag
};

// What the persistent kernel reads and writes (device pointers).
struct SvcQueueDev {
    const uint2* items;              // kSvcQueues rings of ring_mask + 1 items, ring 0 first
    const unsigned long long* tail;  // [kSvcQueues] items published
    unsigned long long* head;        // [kSvcQueues] items claimed
    unsigned int* live;              // [0] warps working on an item, [1] closing (per launch)
    unsigned long long ring_mask;
    unsigned int* done;              // items finished per batch slot
    volatile unsigned int* finished; // mapped host: generation of the last finished batch per slot
    const unsigned int* stop;        // leave now
    unsigned long long idle_ns;      // the kernel leaves after this long without work
    uint32_t large_first_every;      // 0: every warp drains ring 0 first; k: warps k-1, 2k-1, ... drain the last ring first
    uint32_t pad;
};

struct RingState;

class RingService {
public:
    // record_bytes: sizeof the batch record type (starting with
    // SvcJobHead); the device table records() is an array of that type.
    // name prefixes error messages.
    RingService(int device, size_t record_bytes, const char* name);
    ~RingService();
    RingService(const RingService&) = delete;
    RingService& operator=(const RingService&) = delete;
    // Every k-th warp drains the rings largest first (0: none), so the
    // largest jobs keep a share of the warps under a stream of small ones.
    // Set before start().
    void set_large_first_every(uint32_t k);
    // Starts the dispatcher; launch(stream) enqueues one persistent launch.
    void start(cudaError_t (*launch)(cudaStream_t, void*), void* user);
    // Ends a running kernel (stop word) and the dispatcher; idempotent.
    void stop();
    const SvcQueueDev& queue() const;
    void* records() const;  // device: one record per batch slot
    // Appends index[0..n) of the batch described by `record` to ring
    // `queue` and waits until every item is done. At most max_batch() items.
    // Throws rb::Error on device failure.
    void run_batch(const void* record, const uint32_t* index, size_t n, int queue);
    size_t max_batch() const;
    uint32_t launches() const;

private:
    void dispatcher();
    RingState* st_;
};

// ----- device sequence store (layers.cu) -----
// One entry of the staged sequence table: offsets of the forward bases and
// quality and of the reverse complement and reversed quality in the store.
constexpr uint64_t kNotStaged = ~0ull;

struct SeqDev {
    uint64_t fwd, fq, rev, rq;  // store offsets, kNotStaged when absent
    uint32_t len;
    uint32_t pad;
};

// The staged table as the aligner and the layer assembly read it.
struct SeqStore {
    const uint8_t* bytes = nullptr;   // device
    const SeqDev* seqs = nullptr;     // device
    const SeqDev* host = nullptr;     // host copy of seqs
    size_t n = 0;
};

// ----- overlap alignment engine (nw_align.cu) -----
struct NwPairDev {
    uint64_t q_off, t_off;  // offsets of the encoded query / target in the code buffer
    uint64_t mq_off;        // offset of the per-target-position match array
    uint64_t bp_off;        // offset (uint32 units) of the breakpoint slots
    uint32_t m, n;          // query / target span lengths
    uint32_t nsym;          // symbol codes are < nsym
    uint32_t q_offset, t_begin;
};

class NwService;

class NwEngine {
public:
    explicit NwEngine(const DeviceInfo& dev, cudaStream_t stream);
    ~NwEngine();
    void stage(const rb_pair* pairs, size_t n, int want_cigar, uint32_t window_length);
    // Pairs cut from the staged sequence table and encoded on the device.
    void stage_store(const rb_store_pair* pairs, size_t n, int want_cigar, uint32_t window_length,
                     const SeqStore& st);
    // Aligns the staged pairs: through the shared service when one is set
    // and the pairs fit its scratch, else on this engine's own kernels.
    void run();
    // Routes run() through a shared alignment service (nullptr: own
    // kernels). Batches of at most priority_pairs pairs use the first ring,
    // larger ones later rings (x4 per ring).
    void set_service(NwService* svc, uint32_t priority_pairs) {
        svc_ = svc;
        svc_priority_ = priority_pairs;
    }
    void fetch(rb_aln_result* out);
    // Breaking points of the last run on the device: pair i's (t, q) values
    // at bp_slots()[pairs()[i].bp_off ...], bp_counts()[i] of them.
    // scheduling (results do not depend on them): the stream the engine
    // enqueues on, and pairs or tasks a warp takes per launch (0: the
    // kernels are persistent until their queue is empty)
    void set_stream(cudaStream_t s) { stream_ = s; }
    void set_yield(uint32_t items) { yield_items_ = items; }
    // percent of the SMs the persistent kernels fill (100: all)
    void set_sm_share(uint32_t pct) { sm_share_pct_ = pct ? pct : 100; }
    const uint32_t* bp_slots() const { return d_bp_.as<uint32_t>(); }
    const uint32_t* bp_counts() const { return d_bpcnt_.as<uint32_t>(); }
    const NwPairDev* pairs() const { return h_pairs_.as<NwPairDev>(); }
    // breaking points straight from SAM CIGARs (no alignment)
    void cigar_breakpoints(const rb_cigar_overlap* ovl, size_t n, uint32_t window_length,
                           rb_aln_result* out);
    const rb_stats& stats() const { return stats_; }
    size_t staged() const { return npairs_; }

private:
    void reserve_scratch(uint32_t max_m, uint32_t max_n);
    void run_own();
    void run_shared();
    void finish_outputs(const void* args);
    NwService* svc_ = nullptr;
    uint32_t svc_priority_ = 0;
    DeviceInfo dev_;
    cudaStream_t stream_;
    cudaEvent_t ev0_, ev1_, ev2_, ev3_;
    size_t npairs_ = 0;
    uint32_t yield_items_ = 0;
    uint32_t sm_share_pct_ = 100;
    int want_cigar_ = 0;
    uint32_t window_length_ = 500;
    uint32_t max_m_ = 0, max_n_ = 0;
    uint64_t code_bytes_ = 0, mq_len_ = 0, bp_slots_ = 0;
    HostBuf h_codes_, h_pairs_, h_order_, h_src_;
    HostBuf h_dist_, h_bp_, h_bpcnt_, h_cig_, h_cigoff_, h_misc_;
    DevBuf d_codes_, d_pairs_, d_src_, d_order_, d_dist_, d_mq_, d_bp_, d_bpcnt_;
    DevBuf d_tasks_[2], d_misc_, d_scratch_, d_ciglen_, d_cigoff_, d_cig_;
    size_t scratch_warps_ = 0, scratch_stride_ = 0;
    std::vector<int32_t> dist_;
    std::vector<uint64_t> bp_offsets_, cig_offsets_;
    std::vector<uint32_t> bp_;
    rb_stats stats_{};
};

// ----- window consensus engine (poa_consensus.cu) -----
// Device records of a staged batch: windows and their layers, byte offsets
// into one input buffer (packed by PoaEngine::stage, or the resident
// sequence store of LayerEngine).
constexpr uint64_t kNoQual = ~0ull;

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

class PoaService;

class PoaEngine {
public:
    PoaEngine(const DeviceInfo& dev, cudaStream_t stream, int8_t m, int8_t x, int8_t g);
    ~PoaEngine();
    void stage(const rb_window* wins, size_t n, int trim);
    // Windows whose bytes and layer records already sit in device memory
    // (device layer assembly): d_in holds every offset of wins and of the
    // d_layers records; sum_len[i] is the total layer length of window i and
    // labels[i] its (target id, rank). The device buffers must stay
    // unchanged until the next stage call or forget().
    void stage_device(const uint8_t* d_in, const PoaWinDev* wins, size_t n, const PoaLayerDev* d_layers,
                      const uint64_t* sum_len, const std::vector<std::pair<uint64_t, uint32_t>>& labels,
                      uint32_t max_len, int trim);
    // Drops a device stage whose buffers are about to change.
    void forget();
    // scheduling (results do not depend on them): the stream the engine
    // enqueues on, and windows a warp takes per launch (0: persistent)
    void set_stream(cudaStream_t s) { stream_ = s; }
    void set_yield(uint32_t windows) { yield_windows_ = windows; }
    // percent of the SMs the persistent kernel fills (100: all)
    void set_sm_share(uint32_t pct) { sm_share_pct_ = pct ? pct : 100; }
    void run(bool plain = false);
    // The staged windows through a device-wide shared queue (serving):
    // returns when every window of this batch is done; windows that outgrow
    // the shared slots run again here with larger graph capacity. Batches
    // of at most priority_windows windows use the first ring, larger ones
    // later rings (x4 per ring).
    void run_shared(PoaService& svc, uint32_t priority_windows);
    size_t staged() const { return nwin_; }
    void fetch(rb_poa_result* out);
    const rb_stats& stats() const { return stats_; }
    // device bytes the per-window scratch slots may take (resident windows
    // are halved until they fit)
    void set_scratch_budget(size_t bytes) { scratch_budget_ = bytes; }
    // scratch bytes of one resident window at the starting graph capacity
    static size_t slot_bytes_for(uint32_t max_layer_length);

private:
    friend class PoaService;
    void prepare_outputs();
    void run_list(std::vector<uint32_t> todo, int ncap, bool plain);
    DeviceInfo dev_;
    cudaStream_t stream_;
    cudaEvent_t ev0_, ev1_, ev2_, ev3_;
    int8_t match_, mismatch_, gap_;
    int trim_ = 1;
    uint32_t yield_windows_ = 0;
    uint32_t sm_share_pct_ = 100;
    size_t nwin_ = 0;
    uint64_t in_bytes_ = 0, out_cap_ = 0;
    uint32_t max_len_ = 0, max_nodes_cap_ = 0;
    const uint8_t* in_ptr_ = nullptr;          // input bytes of the staged windows
    const PoaLayerDev* layers_ptr_ = nullptr;  // their layer records
    HostBuf h_in_, h_desc_, h_layers_, h_order_, h_out_, h_outlen_, h_flags_;
    DevBuf d_in_, d_desc_, d_layers_, d_order_, d_out_, d_outlen_, d_flags_, d_misc_;
    DevBuf d_graph_, d_dp_;
    size_t slots_ = 0, graph_stride_ = 0, dp_stride_ = 0;
    std::vector<uint64_t> offsets_;
    std::vector<char> cons_;
    std::vector<uint8_t> polished_;
    std::vector<std::pair<uint64_t, uint32_t>> labels_;  // (id, rank) per window
    size_t scratch_budget_ = size_t(48) << 30;
    rb_stats stats_{};
};

// ----- shared window-consensus service (poa_consensus.cu) -----
// One persistent consensus kernel per device on a RingService: its warps
// take (job, window) items of every job in flight, smallest jobs' ring
// first, so windows of jobs admitted while others run start as soon as any
// warp frees up. Thread-safe.
struct PoaJobDev;
struct PoaSvcState;

class PoaService {
public:
    // ctas_per_sm: resident consensus CTAs (4 warps each) per SM, 1..3; the
    // rest of the SM stays free for other kernels.
    // large_first_every: RingService::set_large_first_every.
    PoaService(int device, int8_t m, int8_t x, int8_t g, uint32_t window_length, size_t scratch_budget,
               uint32_t ctas_per_sm, uint32_t large_first_every = 0);
    ~PoaService();
    PoaService(const PoaService&) = delete;
    PoaService& operator=(const PoaService&) = delete;
    // Enqueues windows order[0..n) of the batch described by `job` on ring
    // `queue` (0 is drained first) and waits until all of them are done.
    // Throws rb::Error on device failure.
    void run_batch(const PoaJobDev& job, const uint32_t* order, size_t n, int queue);
    uint32_t slots() const;
    uint32_t launches() const;

private:
    PoaSvcState* st_;
};

// ----- shared overlap-alignment service (nw_align.cu) -----
// One persistent alignment kernel per device on a RingService: its warps
// take the distance passes and the path-recursion tasks of every job in
// flight, smallest jobs' ring first, so a small job's alignments do not wait
// for a large job's persistent grid to drain. Thread-safe.
struct NwJobDev;
struct NwSvcState;

class NwService {
public:
    // max_span: longest query and target span a batch may hold (the warps'
    // scratch is sized for it; longer batches run on the engine's own
    // kernels); ctas_per_sm: resident alignment CTAs (4 warps each) per SM.
    NwService(int device, uint32_t max_span, size_t scratch_budget, uint32_t ctas_per_sm,
              uint32_t large_first_every = 0);
    ~NwService();
    NwService(const NwService&) = delete;
    NwService& operator=(const NwService&) = delete;
    bool fits(uint32_t max_m, uint32_t max_n) const;
    // Enqueues items index[0..n) of `job` (pairs of a distance pass, or
    // tasks of one recursion level) on ring `queue` and waits for them;
    // batches above the ring's limit go in parts.
    void run_batch(const NwJobDev& job, const uint32_t* index, size_t n, int queue);
    uint32_t slots() const;
    uint32_t launches() const;

private:
    NwSvcState* st_;
};

// ----- device layer assembly (layers.cu) -----

class LayerEngine {
public:
    LayerEngine(const DeviceInfo& dev, cudaStream_t stream);
    ~LayerEngine();
    // Copies the sequence table to the device store and builds the reverse
    // complements there; drops any window stage of poa that reads the store.
    void stage_sequences(const rb_sequence* seqs, size_t n, PoaEngine& poa);
    // Layers of every window over targets 0 .. n_targets-1 from host
    // breaking points, then poa.stage_device.
    void assemble(size_t n_targets, const rb_layer_overlap* ovl, size_t n, const uint32_t* bps,
                  const uint64_t* bp_offsets, uint32_t window_length, double quality_threshold, int tgs, int trim,
                  PoaEngine& poa);
    // The same from alignments of pairs cut from the store: each batch's
    // breaking points go from the aligner's device buffers straight to the
    // layer candidates. out (may be NULL) receives edit distances and
    // breaking points on the host.
    void assemble_aligned(size_t n_targets, const rb_store_pair* pairs, size_t n, uint32_t window_length,
                          double quality_threshold, int tgs, int trim, NwEngine& nw, PoaEngine& poa,
                          rb_aln_result* out);
    SeqStore store() const;
    const rb_stats& stats() const { return stats_; }
    const rb_stats& sequence_stats() const { return seq_stats_; }
    void set_stream(cudaStream_t s) { stream_ = s; }

private:
    void begin(size_t n_targets, uint32_t window_length, double quality_threshold, uint64_t cand_cap);
    void add_candidates(const uint32_t* d_bp, const uint32_t* d_bpcnt, const void* d_ovl, size_t n);
    void finish(int tgs, int trim, PoaEngine& poa);
    uint32_t* win_cnt() const;
    uint32_t* win_fill() const;
    uint64_t* win_base() const;
    unsigned long long* win_sum() const;
    uint32_t* status() const;

    DeviceInfo dev_;
    cudaStream_t stream_;
    cudaEvent_t ev0_, ev1_;
    size_t nseq_ = 0, n_targets_ = 0;
    uint64_t nwin_ = 0, cand_cap_ = 0, store_bytes_ = 0;
    uint32_t w_ = 500;
    double q_threshold_ = 10.0;
    int batches_ = 0;
    float cand_ms_ = 0;
    std::vector<uint32_t> lens_;
    std::vector<uint64_t> fwd_, fq_, first_window_;
    std::vector<SeqDev> host_tab_;
    std::vector<int32_t> out_dist_;
    std::vector<uint32_t> out_bp_;
    std::vector<uint64_t> out_bp_off_;
    HostBuf h_store_, h_misc_, h_bp_, h_fw_, h_lay_, h_perm_;
    DevBuf d_store_, d_seqs_, d_list_, d_bp_, d_ovl_, d_fw_, d_cand_, d_cand_win_, d_win_, d_lay_, d_final_;
    rb_stats stats_{}, seq_stats_{};
};

// Caps the window-consensus scratch of a context (server workers share one
// device); defined in rb_capi.cpp.
void ctx_set_poa_budget(rb_ctx* ctx, size_t bytes);
// Routes the context's rb_poa_run through a shared consensus service
// (nullptr: its own kernel); batches of at most priority_windows windows use
// the high-priority queue. Defined in rb_capi.cpp.
void ctx_set_poa_service(rb_ctx* ctx, PoaService* svc, uint32_t priority_windows);
// Routes the context's alignments through a shared alignment service
// (nullptr: its own kernels). Defined in rb_capi.cpp.
void ctx_set_nw_service(rb_ctx* ctx, NwService* svc, uint32_t priority_pairs);

}  // namespace rb
