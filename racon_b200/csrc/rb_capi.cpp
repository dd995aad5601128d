// C ABI of racon_b200 (declared in include/racon_b200.h). Thin layer over the
// device engines: argument checks, device selection, error codes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/racon_b200.h"
#include "rb_internal.hpp"

namespace rb {

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? RB_ERR_NOMEM : RB_ERR_CUDA;
        throw Error{code, std::string(what) + ": " + cudaGetErrorString(e)};
    }
}

namespace {
thread_local cudaStream_t t_alloc_stream = nullptr;
thread_local bool t_alloc_bound = false;
}  // namespace

AllocStreamScope::AllocStreamScope(cudaStream_t s) : prev(t_alloc_stream), prev_bound(t_alloc_bound) {
    t_alloc_stream = s;
    t_alloc_bound = true;
}
AllocStreamScope::~AllocStreamScope() {
    t_alloc_stream = prev;
    t_alloc_bound = prev_bound;
}

void DevBuf::reserve(size_t need) {
    if (need <= bytes && ptr) return;
    release();
    size_t b = need < 256 ? 256 : need;
    if (t_alloc_bound) {
        check_cuda(cudaMallocAsync(&ptr, b, t_alloc_stream), "cudaMallocAsync");
        stream = t_alloc_stream;
        stream_ordered = true;
    } else {
        check_cuda(cudaMalloc(&ptr, b), "cudaMalloc");
        stream_ordered = false;
    }
    bytes = b;
}
void DevBuf::release() {
    if (ptr) {
        if (stream_ordered)
            cudaFreeAsync(ptr, stream);
        else
            cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}
void HostBuf::reserve(size_t need) {
    if (need <= bytes && ptr) return;
    // the outgrown buffer is kept until the owner is destroyed: cudaFreeHost
    // synchronises the whole device, which with a resident persistent kernel
    // of another context (the serving loop) would wait for that kernel
    if (ptr) retired.push_back(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t b = need < 256 ? 256 : need;
    b = b + b / 2;  // headroom for growing batches (few growth steps)
    check_cuda(cudaMallocHost(&ptr, b), "cudaMallocHost");
    bytes = b;
}
void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    for (void* r : retired) cudaFreeHost(r);
    retired.clear();
    ptr = nullptr;
    bytes = 0;
}

void prefer_max_shared(const void* kernel) {
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    int(cudaSharedmemCarveoutMaxShared)),
               "cudaFuncSetAttribute carveout");
}

void keep_pool_reserve(int device) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return;
    uint64_t keep = ~uint64_t(0);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
}

namespace {
constexpr int kTuneDevices = 64;
std::mutex g_tune_mu;
rb_tuning g_tune[kTuneDevices];
bool g_tune_init[kTuneDevices] = {false};

rb_tuning tuning_default() {
    rb_tuning t;
    memset(&t, 0, sizeof(t));
    t.consensus_ctas_per_sm = 3;
    t.consensus_order = 0;
    t.alignment_warps_per_sm = 16;
    return t;
}

rb_tuning tuning_clamp(rb_tuning t) {
    t.consensus_ctas_per_sm = std::max<uint32_t>(1, std::min<uint32_t>(3, t.consensus_ctas_per_sm));
    t.consensus_order = t.consensus_order ? 1 : 0;
    t.alignment_warps_per_sm = std::max<uint32_t>(4, std::min<uint32_t>(32, t.alignment_warps_per_sm & ~3u));
    return t;
}
}  // namespace

rb_tuning tuning_get(int device) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (device < 0 || device >= kTuneDevices) return tuning_default();
    if (!g_tune_init[device]) {
        g_tune[device] = tuning_default();
        g_tune_init[device] = true;
    }
    return g_tune[device];
}

void tuning_set(int device, const rb_tuning& t) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (device < 0 || device >= kTuneDevices) return;
    g_tune[device] = tuning_clamp(t);
    g_tune_init[device] = true;
}

}  // namespace rb

struct rb_ctx {
    rb::DeviceInfo dev;
    cudaStream_t stream = nullptr;     // the one the engines use now
    cudaStream_t stream_lo = nullptr;  // normal priority
    cudaStream_t stream_hi = nullptr;  // highest priority
    rb_params params{};
    std::unique_ptr<rb::NwEngine> nw;
    std::unique_ptr<rb::PoaEngine> poa;
    std::unique_ptr<rb::LayerEngine> layers;
    rb::PoaService* svc = nullptr;       // shared consensus kernel (serving), not owned
    uint32_t svc_priority_windows = 0;
    std::string err;
};

namespace rb {
void ctx_set_poa_budget(rb_ctx* ctx, size_t bytes) {
    if (ctx && ctx->poa) ctx->poa->set_scratch_budget(bytes);
}
void ctx_set_poa_service(rb_ctx* ctx, PoaService* svc, uint32_t priority_windows) {
    if (!ctx) return;
    ctx->svc = svc;
    ctx->svc_priority_windows = priority_windows;
}
void ctx_set_nw_service(rb_ctx* ctx, NwService* svc, uint32_t priority_pairs) {
    if (ctx && ctx->nw) ctx->nw->set_service(svc, priority_pairs);
}
}  // namespace rb

namespace {
std::mutex g_err_mu;
std::string g_create_err;

void set_create_error(const std::string& s) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_create_err = s;
}

template <class F>
int guarded(rb_ctx* ctx, F&& f) {
    if (!ctx) return RB_ERR_ARG;
    try {
        cudaSetDevice(ctx->dev.device);
        rb::AllocStreamScope scope(ctx->stream);
        f();
        ctx->err.clear();
        return RB_OK;
    } catch (const rb::Error& e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->err = "host allocation failed";
        return RB_ERR_NOMEM;
    }
}
}  // namespace

extern "C" {

rb_ctx* rb_create(int device, const rb_params* params) {
    if (!params) {
        set_create_error("rb_create: params is NULL");
        return nullptr;
    }
    if (params->window_length == 0) {
        set_create_error("rb_create: invalid window length");
        return nullptr;
    }
    if (params->gap > 0) {
        set_create_error("rb_create: gap penalty must be non-positive");
        return nullptr;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        set_create_error("rb_create: no CUDA device");
        return nullptr;
    }
    if (device < 0 || device >= count) {
        set_create_error("rb_create: device index out of range");
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        set_create_error("rb_create: cudaGetDeviceProperties failed");
        return nullptr;
    }
    if (prop.major != 10) {
        set_create_error("rb_create: device is not sm_100 (B200); this build carries sm_100a code only");
        return nullptr;
    }
    auto ctx = std::unique_ptr<rb_ctx>(new rb_ctx());
    ctx->dev.device = device;
    ctx->dev.sm_count = prop.multiProcessorCount;
    ctx->dev.smem_optin = prop.sharedMemPerBlockOptin;
    ctx->params = *params;
    try {
        rb::check_cuda(cudaSetDevice(device), "cudaSetDevice");
        rb::check_cuda(cudaStreamCreateWithFlags(&ctx->stream_lo, cudaStreamNonBlocking), "cudaStreamCreate");
        int least = 0, greatest = 0;
        rb::check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
        rb::check_cuda(cudaStreamCreateWithPriority(&ctx->stream_hi, cudaStreamNonBlocking, greatest),
                       "cudaStreamCreateWithPriority");
        ctx->stream = ctx->stream_lo;
        rb::keep_pool_reserve(device);
        ctx->nw.reset(new rb::NwEngine(ctx->dev, ctx->stream));
        ctx->poa.reset(new rb::PoaEngine(ctx->dev, ctx->stream, params->match, params->mismatch, params->gap));
        ctx->layers.reset(new rb::LayerEngine(ctx->dev, ctx->stream));
    } catch (const rb::Error& e) {
        set_create_error(e.msg);
        return nullptr;
    }
    return ctx.release();
}

const char* rb_create_error(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_create_err.c_str();
}

void rb_destroy(rb_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->dev.device);
    ctx->nw.reset();
    ctx->layers.reset();
    ctx->poa.reset();
    if (ctx->stream_lo) cudaStreamDestroy(ctx->stream_lo);
    if (ctx->stream_hi) cudaStreamDestroy(ctx->stream_hi);
    delete ctx;
}

const char* rb_last_error(const rb_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

int rb_align_stage(rb_ctx* ctx, const rb_pair* pairs, size_t n, int want_cigar) {
    return guarded(ctx, [&]() { ctx->nw->stage(pairs, n, want_cigar, ctx->params.window_length); });
}
int rb_align_run(rb_ctx* ctx) {
    return guarded(ctx, [&]() { ctx->nw->run(); });
}
int rb_align_fetch(rb_ctx* ctx, rb_aln_result* out) {
    if (!out) return RB_ERR_ARG;
    return guarded(ctx, [&]() { ctx->nw->fetch(out); });
}
int rb_align_batch(rb_ctx* ctx, const rb_pair* pairs, size_t n, int want_cigar, rb_aln_result* out) {
    if (!out) return RB_ERR_ARG;
    return guarded(ctx, [&]() {
        ctx->nw->stage(pairs, n, want_cigar, ctx->params.window_length);
        ctx->nw->run();
        ctx->nw->fetch(out);
    });
}

int rb_cigar_breakpoints(rb_ctx* ctx, const rb_cigar_overlap* overlaps, size_t n, rb_aln_result* out) {
    if (!out) return RB_ERR_ARG;
    return guarded(ctx, [&]() { ctx->nw->cigar_breakpoints(overlaps, n, ctx->params.window_length, out); });
}

int rb_poa_stage(rb_ctx* ctx, const rb_window* windows, size_t n, int trim) {
    return guarded(ctx, [&]() { ctx->poa->stage(windows, n, trim); });
}
int rb_poa_run(rb_ctx* ctx) {
    return guarded(ctx, [&]() {
        if (ctx->svc)
            ctx->poa->run_shared(*ctx->svc, ctx->svc_priority_windows);
        else
            ctx->poa->run();
    });
}

int rb_poa_run_plain(rb_ctx* ctx) {
    return guarded(ctx, [&]() { ctx->poa->run(true); });
}
int rb_poa_fetch(rb_ctx* ctx, rb_poa_result* out) {
    if (!out) return RB_ERR_ARG;
    return guarded(ctx, [&]() { ctx->poa->fetch(out); });
}
int rb_poa_batch(rb_ctx* ctx, const rb_window* windows, size_t n, int trim, rb_poa_result* out) {
    if (!out) return RB_ERR_ARG;
    return guarded(ctx, [&]() {
        ctx->poa->stage(windows, n, trim);
        ctx->poa->run();
        ctx->poa->fetch(out);
    });
}

int rb_sequences_stage(rb_ctx* ctx, const rb_sequence* sequences, size_t n) {
    return guarded(ctx, [&]() { ctx->layers->stage_sequences(sequences, n, *ctx->poa); });
}
int rb_align_stage_overlaps(rb_ctx* ctx, const rb_store_pair* pairs, size_t n, int want_cigar) {
    return guarded(ctx, [&]() {
        ctx->nw->stage_store(pairs, n, want_cigar, ctx->params.window_length, ctx->layers->store());
    });
}
int rb_poa_stage_alignments(rb_ctx* ctx, size_t n_targets, const rb_store_pair* pairs, size_t n,
                            double quality_threshold, int tgs, int trim, rb_aln_result* breakpoints) {
    return guarded(ctx, [&]() {
        ctx->layers->assemble_aligned(n_targets, pairs, n, ctx->params.window_length, quality_threshold, tgs, trim,
                                      *ctx->nw, *ctx->poa, breakpoints);
    });
}
int rb_poa_stage_overlaps(rb_ctx* ctx, size_t n_targets, const rb_layer_overlap* overlaps, size_t n,
                          const uint32_t* breakpoints, const uint64_t* bp_offsets, double quality_threshold,
                          int tgs, int trim) {
    return guarded(ctx, [&]() {
        ctx->layers->assemble(n_targets, overlaps, n, breakpoints, bp_offsets, ctx->params.window_length,
                              quality_threshold, tgs, trim, *ctx->poa);
    });
}
int rb_layer_stats(const rb_ctx* ctx, rb_stats* out) {
    if (!ctx || !out) return RB_ERR_ARG;
    *out = ctx->layers->stats();
    return RB_OK;
}
int rb_sequence_stats(const rb_ctx* ctx, rb_stats* out) {
    if (!ctx || !out) return RB_ERR_ARG;
    *out = ctx->layers->sequence_stats();
    return RB_OK;
}

int rb_set_yield(rb_ctx* ctx, uint32_t consensus_windows, uint32_t alignment_items) {
    if (!ctx) return RB_ERR_ARG;
    ctx->poa->set_yield(consensus_windows);
    ctx->nw->set_yield(alignment_items);
    return RB_OK;
}
int rb_set_sm_share(rb_ctx* ctx, uint32_t percent) {
    if (!ctx || percent > 100) return RB_ERR_ARG;
    ctx->poa->set_sm_share(percent);
    ctx->nw->set_sm_share(percent);
    return RB_OK;
}
int rb_set_priority(rb_ctx* ctx, int high) {
    return guarded(ctx, [&]() {
        cudaStream_t s = high ? ctx->stream_hi : ctx->stream_lo;
        if (s == ctx->stream) return;
        // every call leaves its stream idle; wait anyway before switching
        rb::check_cuda(cudaStreamSynchronize(ctx->stream), "stream sync");
        ctx->stream = s;
        ctx->nw->set_stream(s);
        ctx->poa->set_stream(s);
        ctx->layers->set_stream(s);
    });
}

int rb_poa_stats(const rb_ctx* ctx, rb_stats* out) {
    if (!ctx || !out) return RB_ERR_ARG;
    *out = ctx->poa->stats();
    return RB_OK;
}
int rb_align_stats(const rb_ctx* ctx, rb_stats* out) {
    if (!ctx || !out) return RB_ERR_ARG;
    *out = ctx->nw->stats();
    return RB_OK;
}

void rb_free(void* p) { free(p); }

}  // extern "C"

// ---------------------------------------------------------------- autotuner

extern "C" {

int rb_tuning_get(int device, rb_tuning* out) {
    if (!out) return RB_ERR_ARG;
    *out = rb::tuning_get(device);
    return RB_OK;
}

int rb_tuning_set(int device, const rb_tuning* in) {
    if (!in) return RB_ERR_ARG;
    rb::tuning_set(device, *in);
    return RB_OK;
}

int rb_autotune(rb_ctx* ctx, int what) {
    return guarded(ctx, [&]() {
        const int dev = ctx->dev.device;
        rb_tuning best = rb::tuning_get(dev);
        if (what & 1) {
            if (ctx->poa->staged() == 0) throw rb::Error{RB_ERR_ARG, "rb_autotune: no windows staged"};
            double best_ms = 1e300;
            std::string ref;
            std::vector<uint8_t> ref_pol;
            for (uint32_t cps = 3; cps >= 1; --cps) {
                for (uint32_t order = 0; order <= 1; ++order) {
                    rb_tuning t = best;
                    t.consensus_ctas_per_sm = cps;
                    t.consensus_order = order;
                    rb::tuning_set(dev, t);
                    ctx->poa->run();
                    const double ms = ctx->poa->stats().kernel_ms;
                    rb_poa_result r;
                    ctx->poa->fetch(&r);
                    const size_t n = ctx->poa->staged();
                    std::string cons(r.consensus, r.consensus + r.offsets[n]);
                    std::vector<uint8_t> pol(r.polished, r.polished + n);
                    if (ref_pol.empty() && ref.empty()) {
                        ref.swap(cons);
                        ref_pol.swap(pol);
                    } else if (cons != ref || pol != ref_pol) {
                        rb::tuning_set(dev, best);
                        throw rb::Error{RB_ERR_DEVICE, "rb_autotune: consensus differs between launch settings"};
                    }
                    if (ms < best_ms) {
                        best_ms = ms;
                        best.consensus_ctas_per_sm = cps;
                        best.consensus_order = order;
                    }
                }
            }
            best.consensus_ms = best_ms;
            best.tuned |= 1u;
        }
        if (what & 2) {
            if (ctx->nw->staged() == 0) throw rb::Error{RB_ERR_ARG, "rb_autotune: no pairs staged"};
            double best_ms = 1e300;
            std::vector<int32_t> ref_d;
            std::vector<uint32_t> ref_bp;
            const uint32_t cand[] = {8, 12, 16, 24, 32};
            for (uint32_t w : cand) {
                rb_tuning t = best;
                t.alignment_warps_per_sm = w;
                rb::tuning_set(dev, t);
                ctx->nw->run();
                const double ms = ctx->nw->stats().kernel_ms;
                rb_aln_result r;
                ctx->nw->fetch(&r);
                const size_t n = ctx->nw->staged();
                std::vector<int32_t> d(r.edit_distance, r.edit_distance + n);
                std::vector<uint32_t> bp(r.breakpoints, r.breakpoints + r.bp_offsets[n]);
                if (ref_d.empty()) {
                    ref_d.swap(d);
                    ref_bp.swap(bp);
                } else if (d != ref_d || bp != ref_bp) {
                    rb::tuning_set(dev, best);
                    throw rb::Error{RB_ERR_DEVICE, "rb_autotune: alignments differ between launch settings"};
                }
                if (ms < best_ms) {
                    best_ms = ms;
                    best.alignment_warps_per_sm = w;
                }
            }
            best.alignment_ms = best_ms;
            best.tuned |= 2u;
        }
        rb::tuning_set(dev, best);
    });
}

}  // extern "C"
