// Serving loop over the B200 polishing path (include/racon_b200.h,
// rb_server_*). racon itself polishes one job per process; this keeps a pool
// of device contexts alive and runs jobs as they arrive.
//
// Design:
//   - `workers` threads, each owning one rb_ctx (own CUDA streams, own device
//     buffers). Buffers grow to the largest job a worker has run and stay
//     allocated; growth is stream-ordered, so it does not synchronise the
//     device under the other workers.
//   - Continuous batching of the window consensus: one PoaService per server
//     (a persistent consensus kernel on part of every SM, fed by size-class
//     rings in device memory). A worker runs its job's parsing, alignment and
//     layer assembly on its own context, then its rb_poa_run appends the
//     job's windows to the shared queue and waits; windows of jobs admitted
//     while others run start on the next free warp.
//   - Continuous batching of the overlap alignment (shared_alignment): one
//     NwService per server, a persistent alignment kernel on one CTA per SM
//     by default, fed by its own size-class rings. A job's distance pass and
//     each level of its path recursion are batches of that queue, so a small
//     job's pairs start on the next free warp instead of waiting for a large
//     job's persistent alignment grid to drain. Jobs whose spans exceed the
//     kernel's scratch align on their own context.
//   - Optional, for jobs aligned on their own context (alignment_yield):
//     small jobs on the high-priority stream and large jobs' alignment in
//     bounded launches, so a small job's alignment kernels find SMs between
//     a large job's launches.
//   - Admission is first in first out by estimated device footprint: the
//     head of the queue starts when a worker is idle and its estimate fits
//     beside the jobs in flight within hbm_budget (a job alone always
//     starts).
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/racon_b200.h"
#include "../rb_internal.hpp"
#include "racon.hpp"

namespace {

thread_local std::string t_server_error;

struct Request {
    uint64_t ticket = 0;
    std::string sp, op, tp;
    rb_server_job spec{};
    uint64_t footprint = 0;
    uint64_t windows = 0;  // estimated from the target file size
    double t_submit = 0, t_admit = 0, t_done = 0;
    double stage[4] = {0, 0, 0, 0};
    uint32_t worker = 0;
    bool done = false;
    bool claimed = false;  // a thread is waiting on (or has taken) this ticket
    int status = RB_OK;
    std::string fasta, error;
};

uint64_t file_bytes(const std::string& p) {
    struct stat st;
    if (stat(p.c_str(), &st) != 0) return 0;
    const uint64_t b = uint64_t(st.st_size);
    const size_t n = p.size();
    // gzip'd inputs expand roughly fourfold
    return (n > 3 && p.compare(n - 3, 3, ".gz") == 0) ? 4 * b : b;
}

}  // namespace

struct rb_server {
    rb_server_params params{};
    int sm_count = 148;
    uint64_t poa_cap = 0;
    std::unique_ptr<rb::PoaService> svc;    // shared consensus kernel (continuous batching)
    std::unique_ptr<rb::NwService> nw_svc;  // shared alignment kernel
    std::vector<rb_ctx*> ctxs;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::map<uint64_t, std::shared_ptr<Request>> jobs;
    uint64_t next_ticket = 1;
    uint64_t inflight_bytes = 0;
    uint32_t inflight = 0;
    bool closing = false;  // rb_server_destroy has begun: submissions are refused
    bool stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // Device bytes a job is expected to hold: its inputs on the device, the
    // alignment scratch and (without the shared consensus kernel, whose
    // scratch is allocated once) one consensus slot per resident window.
    uint64_t estimate(const Request& r) const {
        const uint64_t reads = file_bytes(r.sp), targets = file_bytes(r.tp);
        const uint64_t w = std::max<uint32_t>(1, params.window_length);
        const uint64_t windows = targets / w + 1;
        const uint64_t resident = std::min<uint64_t>(windows, uint64_t(sm_count) * 12);
        const uint64_t slot = rb::PoaEngine::slot_bytes_for(uint32_t(std::min<uint64_t>(3 * w, 65535)));
        const uint64_t poa = svc ? 0 : std::min<uint64_t>(resident * slot, poa_cap);
        const uint64_t align = std::min<uint64_t>(uint64_t(4) << 30, (reads + targets) * 8 + (uint64_t(256) << 20));
        return poa + align + 3 * (reads + targets);
    }

    bool admissible(const Request& r) const {
        return inflight == 0 || inflight_bytes + r.footprint <= params.hbm_budget;
    }

    void worker(uint32_t w) {
        cudaSetDevice(params.device);
        while (true) {
            std::shared_ptr<Request> r;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || (!queue.empty() && admissible(*queue.front())); });
                if (stop) return;
                r = queue.front();
                queue.pop_front();
                inflight_bytes += r->footprint;
                ++inflight;
                r->t_admit = now();
                r->worker = w;
            }
            cv_work.notify_all();
            std::string fasta, error;
            double stage[4] = {0, 0, 0, 0};
            const rb_server_job& j = r->spec;
            const bool small = r->windows <= params.priority_windows;
            // small jobs on the high-priority stream; large jobs give SMs
            // back between bounded alignment launches, or keep their
            // persistent alignment grids to part of the SMs
            if (params.alignment_yield || params.alignment_share) rb_set_priority(ctxs[w], small ? 1 : 0);
            if (params.alignment_yield) rb_set_yield(ctxs[w], 0, small ? 0u : params.alignment_yield);
            if (params.alignment_share) rb_set_sm_share(ctxs[w], small ? 100u : params.alignment_share);
            const int rc = racon::polish_job_on_context(
                ctxs[w], params.device, r->sp, r->op, r->tp, j.fragment != 0, params.window_length,
                j.quality_threshold, j.error_threshold, j.trim != 0, params.match, params.mismatch, params.gap,
                j.drop_unpolished != 0, &fasta, &error, stage);
            {
                std::lock_guard<std::mutex> lk(mu);
                inflight_bytes -= r->footprint;
                --inflight;
                r->status = rc;
                r->fasta.swap(fasta);
                r->error.swap(error);
                for (int i = 0; i < 4; ++i) r->stage[i] = stage[i];
                r->t_done = now();
                r->done = true;
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

rb_server* rb_server_create(const rb_server_params* params) {
    if (!params) return nullptr;
    std::unique_ptr<rb_server> s(new rb_server());
    s->params = *params;
    if (s->params.workers == 0) s->params.workers = 4;
    rb_params p;
    p.match = params->match;
    p.mismatch = params->mismatch;
    p.gap = params->gap;
    p.window_length = params->window_length;
    for (uint32_t i = 0; i < s->params.workers; ++i) {
        rb_ctx* c = rb_create(params->device, &p);
        if (!c) {
            for (rb_ctx* x : s->ctxs) rb_destroy(x);
            return nullptr;  // rb_create_error() holds the reason
        }
        s->ctxs.push_back(c);
    }
    cudaSetDevice(params->device);
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, params->device);
    if (s->params.hbm_budget == 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        s->params.hbm_budget = uint64_t(total_b) / 4 * 3;
    }
    s->poa_cap = s->params.hbm_budget / s->params.workers;
    for (rb_ctx* c : s->ctxs) rb::ctx_set_poa_budget(c, s->poa_cap);
    if (s->params.priority_windows == 0) s->params.priority_windows = uint32_t(s->sm_count) * 4;
    if (s->params.shared_consensus) {
        // the shared kernel's scratch comes out of the budget once; each
        // worker keeps a small private budget for windows that outgrow it
        const uint32_t cps = s->params.consensus_ctas_per_sm ? s->params.consensus_ctas_per_sm : 2;
        try {
            s->svc.reset(new rb::PoaService(params->device, params->match, params->mismatch, params->gap,
                                            params->window_length, s->params.hbm_budget / 2, cps,
                                            s->params.large_first_every));
        } catch (const rb::Error& e) {
            for (rb_ctx* x : s->ctxs) rb_destroy(x);
            t_server_error = e.msg;
            return nullptr;
        }
        const uint32_t prio = params->priority_windows ? params->priority_windows : s->svc->slots() / 4;
        s->params.priority_windows = prio;
        for (rb_ctx* c : s->ctxs) {
            rb::ctx_set_poa_budget(c, s->params.hbm_budget / 2 / s->params.workers);
            rb::ctx_set_poa_service(c, s->svc.get(), prio);
        }
    }
    if (s->params.shared_alignment) {
        const uint32_t cps = s->params.alignment_ctas_per_sm ? s->params.alignment_ctas_per_sm : 1;
        const uint32_t span = s->params.alignment_max_span ? s->params.alignment_max_span : 131072;
        try {
            s->nw_svc.reset(new rb::NwService(params->device, span, size_t(4) << 30, cps,
                                              s->params.large_first_every));
        } catch (const rb::Error& e) {
            s->svc.reset();
            for (rb_ctx* x : s->ctxs) rb_destroy(x);
            t_server_error = e.msg;
            return nullptr;
        }
        if (s->params.priority_pairs == 0) s->params.priority_pairs = s->nw_svc->slots();
        for (rb_ctx* c : s->ctxs) rb::ctx_set_nw_service(c, s->nw_svc.get(), s->params.priority_pairs);
    }
    for (uint32_t i = 0; i < s->params.workers; ++i) s->threads.emplace_back([srv = s.get(), i] { srv->worker(i); });
    return s.release();
}

int rb_server_submit(rb_server* s, const rb_server_job* job, uint64_t* ticket) {
    if (!s || !job || !ticket || !job->sequences_path || !job->overlaps_path || !job->target_path) {
        t_server_error = "rb_server_submit: NULL argument";
        return RB_ERR_ARG;
    }
    auto r = std::make_shared<Request>();
    r->sp = job->sequences_path;
    r->op = job->overlaps_path;
    r->tp = job->target_path;
    r->spec = *job;
    r->spec.sequences_path = r->sp.c_str();
    r->spec.overlaps_path = r->op.c_str();
    r->spec.target_path = r->tp.c_str();
    r->footprint = s->estimate(*r);
    r->windows = file_bytes(r->tp) / std::max<uint32_t>(1, s->params.window_length) + 1;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->closing || s->stop) {
            t_server_error = "rb_server_submit: server is stopping";
            return RB_ERR_ARG;
        }
        r->ticket = s->next_ticket++;
        r->t_submit = s->now();
        s->jobs[r->ticket] = r;
        s->queue.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_all();
    return RB_OK;
}

int rb_server_wait(rb_server* s, uint64_t ticket, char** fasta, rb_server_times* times) {
    if (!s || !fasta) {
        t_server_error = "rb_server_wait: NULL argument";
        return RB_ERR_ARG;
    }
    *fasta = nullptr;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) {
            t_server_error = "rb_server_wait: unknown ticket";
            return RB_ERR_ARG;
        }
        r = it->second;
        if (r->claimed) {
            t_server_error = "rb_server_wait: ticket already waited for";
            return RB_ERR_ARG;
        }
        r->claimed = true;
        s->cv_done.wait(lk, [&] { return r->done; });
        s->jobs.erase(ticket);
    }
    if (times) {
        times->submitted = r->t_submit;
        times->admitted = r->t_admit;
        times->finished = r->t_done;
        for (int i = 0; i < 4; ++i) times->stage_seconds[i] = r->stage[i];
        times->footprint = r->footprint;
        times->worker = r->worker;
    }
    if (r->status != RB_OK) {
        t_server_error = r->error;
        return r->status;
    }
    char* buf = static_cast<char*>(malloc(r->fasta.size() + 1));
    if (!buf) {
        t_server_error = "host allocation failed";
        return RB_ERR_NOMEM;
    }
    memcpy(buf, r->fasta.c_str(), r->fasta.size() + 1);
    *fasta = buf;
    return RB_OK;
}

const char* rb_server_error(void) { return t_server_error.c_str(); }

int rb_server_load(rb_server* s, uint32_t* queued, uint32_t* in_flight, uint64_t* in_flight_bytes) {
    if (!s) return RB_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (queued) *queued = uint32_t(s->queue.size());
    if (in_flight) *in_flight = s->inflight;
    if (in_flight_bytes) *in_flight_bytes = s->inflight_bytes;
    return RB_OK;
}

void rb_server_destroy(rb_server* s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // refuse new submissions, cancel what has not started, let the jobs
        // in flight finish
        s->closing = true;
        for (auto& r : s->queue) {
            r->status = RB_ERR_ARG;
            r->error = "rb_server: job cancelled (server destroyed)";
            r->t_done = s->now();
            r->done = true;
        }
        s->queue.clear();
        s->cv_done.notify_all();
        s->cv_done.wait(lk, [&] { return s->inflight == 0; });
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->threads) t.join();
    for (rb_ctx* c : s->ctxs) rb_destroy(c);
    s->svc.reset();
    s->nw_svc.reset();
    delete s;
}

}  // extern "C"
