// Shared work queue of a persistent kernel (RingService, declared in
// rb_internal.hpp): the host half of the serving loop's continuous batching,
// used by the consensus service (poa_consensus.cu) and the alignment service
// (nw_align.cu). The device half (claiming an item, reporting it done) is
// ring_queue.cuh.
//
// Publishing: a batch takes a free slot, then, in one stream, its done
// counter is zeroed, its record written, its items appended to a ring and
// the ring's tail advanced. Copies in one stream start after the previous
// one completes, so a warp that sees the new tail in L2 finds the items and
// the record there too.
//
// Waiting: the batch's last item writes the batch's generation to a flag in
// mapped host memory; run_batch polls it (100 us) and checks the service's
// error state meanwhile.
//
// Relaunching: the kernel leaves as a whole after a bounded idle time (no
// warp working, no item for idle_ns). A dispatcher thread polls the kernel's
// completion event; once it has ended, it reads the ring heads and launches
// again if items are still unclaimed.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rb_internal.hpp"

namespace rb {

namespace {
constexpr uint32_t kSvcJobs = 256;                  // concurrent batches
constexpr unsigned long long kSvcRing = 1ull << 21; // items per ring
// control words (8-byte units): tails, heads, stop, live/closing
constexpr int kCtlTail = 0, kCtlHead = kSvcQueues, kCtlStop = 2 * kSvcQueues, kCtlLive = 2 * kSvcQueues + 1;
constexpr size_t kCtlBytes = 128;
}  // namespace

struct RingState {
    int device = 0;
    size_t rec_bytes = 0;  // one record; also the stride of the device table, which the kernel indexes as an array
    std::string name;
    cudaStream_t stream = nullptr;  // the persistent kernel's stream
    cudaStream_t ctl = nullptr;     // queue writes and head reads (ordered copies)
    cudaEvent_t done_ev = nullptr;
    cudaError_t (*launch)(cudaStream_t, void*) = nullptr;
    void* user = nullptr;
    SvcQueueDev q{};
    // device: rings, control words, batch records, per-slot done counters
    uint2* d_items = nullptr;
    unsigned long long* d_ctl = nullptr;
    uint8_t* d_recs = nullptr;
    unsigned int* d_done = nullptr;
    // host: pinned staging for the copies, mapped finished flags
    uint2* h_stage = nullptr;             // kSvcRing / 2 items
    uint8_t* h_rec = nullptr;             // one record
    unsigned long long* h_val = nullptr;  // tail / stop values
    unsigned int* h_finished = nullptr;   // [kSvcJobs], mapped
    std::mutex mu;      // queue state, dispatcher
    std::mutex pub_mu;  // publishing (staging buffers and the control stream)
    std::condition_variable cv, cv_slot;
    std::vector<uint32_t> free_slots;
    std::vector<uint32_t> generation;
    unsigned long long published[kSvcQueues] = {0, 0, 0, 0};
    unsigned long long active_items = 0;
    bool running = false, stopping = false, stopped = false;
    std::string error;
    std::atomic<uint32_t> launches{0};  // read by other threads (stats)
    std::thread thread;
};

RingService::RingService(int device, size_t record_bytes, const char* name) : st_(new RingState()) {
    RingState& S = *st_;
    S.device = device;
    S.rec_bytes = record_bytes;
    S.name = name;
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaStreamCreateWithFlags(&S.ctl, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreateWithFlags(&S.done_ev, cudaEventDisableTiming), "cudaEventCreate");
    check_cuda(cudaMalloc(&S.d_items, sizeof(uint2) * kSvcRing * kSvcQueues), "cudaMalloc service queue");
    check_cuda(cudaMalloc(&S.d_ctl, kCtlBytes), "cudaMalloc");
    check_cuda(cudaMalloc(&S.d_recs, S.rec_bytes * kSvcJobs), "cudaMalloc");
    check_cuda(cudaMalloc(&S.d_done, kSvcJobs * 4), "cudaMalloc");
    check_cuda(cudaMemset(S.d_ctl, 0, kCtlBytes), "cudaMemset");
    check_cuda(cudaMemset(S.d_done, 0, kSvcJobs * 4), "cudaMemset");
    check_cuda(cudaMemset(S.d_recs, 0, S.rec_bytes * kSvcJobs), "cudaMemset");
    check_cuda(cudaMallocHost(&S.h_stage, sizeof(uint2) * (kSvcRing / 2)), "cudaMallocHost");
    check_cuda(cudaMallocHost(&S.h_rec, S.rec_bytes), "cudaMallocHost");
    memset(S.h_rec, 0, S.rec_bytes);
    check_cuda(cudaMallocHost(&S.h_val, kCtlBytes), "cudaMallocHost");
    check_cuda(cudaHostAlloc(&S.h_finished, 4 * kSvcJobs, cudaHostAllocMapped | cudaHostAllocPortable),
               "cudaHostAlloc mapped");
    memset(S.h_finished, 0, 4 * kSvcJobs);
    void* d_fin = nullptr;
    check_cuda(cudaHostGetDevicePointer(&d_fin, S.h_finished, 0), "cudaHostGetDevicePointer");
    SvcQueueDev& Q = S.q;
    Q.items = S.d_items;
    Q.tail = S.d_ctl + kCtlTail;
    Q.head = S.d_ctl + kCtlHead;
    Q.stop = reinterpret_cast<const unsigned int*>(S.d_ctl + kCtlStop);
    Q.live = reinterpret_cast<unsigned int*>(S.d_ctl + kCtlLive);
    Q.ring_mask = kSvcRing - 1;
    Q.done = S.d_done;
    Q.finished = static_cast<unsigned int*>(d_fin);
    Q.idle_ns = 3000000ull;  // 3 ms
    for (uint32_t j = kSvcJobs; j-- > 0;) S.free_slots.push_back(j);
    S.generation.assign(kSvcJobs, 0);
    keep_pool_reserve(device);
}

void RingService::set_large_first_every(uint32_t k) { st_->q.large_first_every = k; }

void RingService::start(cudaError_t (*launch)(cudaStream_t, void*), void* user) {
    RingState& S = *st_;
    S.launch = launch;
    S.user = user;
    S.thread = std::thread([this] { dispatcher(); });
}

void RingService::stop() {
    RingState& S = *st_;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        if (S.stopped) return;
        S.stopping = true;
        S.stopped = true;
    }
    S.cv.notify_all();
    S.cv_slot.notify_all();
    if (S.thread.joinable()) S.thread.join();
    cudaSetDevice(S.device);
    {
        // the stop word ends a running kernel within its idle bound
        std::lock_guard<std::mutex> lk(S.pub_mu);
        S.h_val[kCtlStop] = 1;
        cudaMemcpyAsync(S.d_ctl + kCtlStop, S.h_val + kCtlStop, 8, cudaMemcpyHostToDevice, S.ctl);
        cudaStreamSynchronize(S.ctl);
    }
    cudaStreamSynchronize(S.stream);
}

RingService::~RingService() {
    stop();
    RingState& S = *st_;
    cudaFree(S.d_items);
    cudaFree(S.d_ctl);
    cudaFree(S.d_recs);
    cudaFree(S.d_done);
    cudaFreeHost(S.h_stage);
    cudaFreeHost(S.h_rec);
    cudaFreeHost(S.h_val);
    cudaFreeHost(S.h_finished);
    cudaEventDestroy(S.done_ev);
    cudaStreamDestroy(S.stream);
    cudaStreamDestroy(S.ctl);
    delete st_;
}

const SvcQueueDev& RingService::queue() const { return st_->q; }
void* RingService::records() const { return st_->d_recs; }
size_t RingService::max_batch() const { return size_t(kSvcRing / 2); }
uint32_t RingService::launches() const { return st_->launches.load(); }

// Keeps the persistent kernel running while items are pending: after the
// kernel leaves (idle, or racing a publish), items still unclaimed start a
// new launch.
void RingService::dispatcher() {
    RingState& S = *st_;
    cudaSetDevice(S.device);
    std::unique_lock<std::mutex> lk(S.mu);
    while (!S.stopping) {
        S.cv.wait_for(lk, std::chrono::microseconds(500));
        if (S.stopping) break;
        if (S.running) {
            const cudaError_t q = cudaEventQuery(S.done_ev);
            if (q == cudaErrorNotReady) continue;
            S.running = false;
            if (q != cudaSuccess) {
                S.error = S.name + " kernel: " + cudaGetErrorString(q);
                S.cv_slot.notify_all();
                continue;
            }
        }
        if (!S.error.empty()) continue;
        bool pending = false;
        {
            // lock order: mu, then pub_mu (publishers take pub_mu alone)
            std::lock_guard<std::mutex> plk(S.pub_mu);
            unsigned long long any = 0;
            for (int q = 0; q < kSvcQueues; ++q) any += S.published[q];
            if (any == 0) continue;
            if (cudaMemcpyAsync(S.h_val + kCtlHead, S.d_ctl + kCtlHead, 8 * kSvcQueues, cudaMemcpyDeviceToHost,
                                S.ctl) != cudaSuccess ||
                cudaStreamSynchronize(S.ctl) != cudaSuccess) {
                S.error = S.name + ": head read failed";
                S.cv_slot.notify_all();
                continue;
            }
            for (int q = 0; q < kSvcQueues; ++q) pending |= S.h_val[kCtlHead + q] < S.published[q];
        }
        if (!pending) continue;
        // a launch starts with no warp working and not closing
        cudaError_t e = cudaMemsetAsync(S.d_ctl + kCtlLive, 0, 8, S.stream);
        if (e == cudaSuccess) e = S.launch(S.stream, S.user);
        if (e == cudaSuccess) e = cudaEventRecord(S.done_ev, S.stream);
        if (e != cudaSuccess) {
            S.error = S.name + " launch: " + cudaGetErrorString(e);
            S.cv_slot.notify_all();
            continue;
        }
        S.running = true;
        ++S.launches;
    }
}

void RingService::run_batch(const void* record, const uint32_t* index, size_t n, int queue) {
    RingState& S = *st_;
    if (n == 0) return;
    if (n > kSvcRing / 2) throw Error{RB_ERR_ARG, S.name + ": batch larger than the shared queue"};
    if (queue < 0 || queue >= kSvcQueues) throw Error{RB_ERR_ARG, S.name + ": bad queue"};
    uint32_t slot = 0, gen = 0;
    {
        std::unique_lock<std::mutex> lk(S.mu);
        // a batch slot, and room in the rings for every item not yet finished
        S.cv_slot.wait(lk, [&] {
            return !S.error.empty() || S.stopping ||
                   (!S.free_slots.empty() && S.active_items + n <= kSvcRing / 2);
        });
        if (!S.error.empty()) throw Error{RB_ERR_DEVICE, S.error};
        if (S.stopping) throw Error{RB_ERR_ARG, S.name + ": shutting down"};
        slot = S.free_slots.back();
        S.free_slots.pop_back();
        S.active_items += n;
        gen = ++S.generation[slot];
    }
    {
        // done counter, record, items, then tail, in one stream
        std::lock_guard<std::mutex> plk(S.pub_mu);
        const int q = queue;
        const unsigned long long t = S.published[q];
        memcpy(S.h_rec, record, S.rec_bytes);
        SvcJobHead head{uint32_t(n), gen};
        memcpy(S.h_rec, &head, sizeof(head));
        check_cuda(cudaMemsetAsync(S.d_done + slot, 0, 4, S.ctl), "memset done");
        check_cuda(cudaMemcpyAsync(S.d_recs + size_t(slot) * S.rec_bytes, S.h_rec, S.rec_bytes,
                                   cudaMemcpyHostToDevice, S.ctl),
                   "H2D batch record");
        for (size_t i = 0; i < n; ++i) S.h_stage[i] = make_uint2(slot, index[i]);
        const size_t at = size_t(t & (kSvcRing - 1));
        const size_t first = std::min(n, size_t(kSvcRing) - at);
        uint2* ring = S.d_items + size_t(q) * kSvcRing;
        check_cuda(cudaMemcpyAsync(ring + at, S.h_stage, first * sizeof(uint2), cudaMemcpyHostToDevice, S.ctl),
                   "H2D items");
        if (first < n)
            check_cuda(cudaMemcpyAsync(ring, S.h_stage + first, (n - first) * sizeof(uint2),
                                       cudaMemcpyHostToDevice, S.ctl),
                       "H2D items");
        S.h_val[kCtlTail + q] = t + n;
        check_cuda(cudaMemcpyAsync(S.d_ctl + kCtlTail + q, S.h_val + kCtlTail + q, 8, cudaMemcpyHostToDevice, S.ctl),
                   "H2D tail");
        check_cuda(cudaStreamSynchronize(S.ctl), "service publish");
        S.published[q] = t + n;
    }
    S.cv.notify_all();
    // wait for the batch; the dispatcher keeps a kernel running meanwhile
    volatile unsigned int* fin = S.h_finished + slot;
    std::string err;
    for (;;) {
        if (*fin == gen) break;
        {
            std::lock_guard<std::mutex> lk(S.mu);
            if (!S.error.empty()) {
                err = S.error;
                break;
            }
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    {
        std::lock_guard<std::mutex> lk(S.mu);
        if (err.empty()) {
            S.free_slots.push_back(slot);
            S.active_items -= n;
        }
    }
    S.cv_slot.notify_all();
    if (!err.empty()) throw Error{RB_ERR_DEVICE, err};
}

}  // namespace rb
