/*
 * racon_b200 — C ABI of the B200 polishing hot path.
 *
 * The library replaces the two third-party calls on racon's polishing path:
 *   - per-overlap global alignment + window breaking points
 *       racon src/overlap.cpp:179-203 (Overlap::find_breaking_points),
 *       :205-224 (Overlap::align_overlaps: edlibAlign NW + standard CIGAR),
 *       :226-292 (Overlap::find_breaking_points_from_cigar),
 *     driven from src/polisher.cpp:462-484 (Polisher::find_overlap_breaking_points);
 *   - per-window partial-order consensus
 *       racon src/window.cpp:65-142 (Window::generate_consensus),
 *     driven from src/polisher.cpp:486-504 (Polisher::polish).
 * In the reference these two seams are the virtual methods that the CUDA
 * plug-in overrides (src/cuda/cudapolisher.hpp:23-24, :43); the C++ host layer
 * of this project (racon_b200/csrc/host) overrides the same two methods and
 * calls the functions below. Inputs are host pointers plus lengths; the
 * library copies them to the device, so nothing here keeps pointers to caller
 * memory after a call returns. Results live in library-owned buffers that stay
 * valid until the next call of the same kind on the same context or
 * rb_destroy().
 *
 * Every function returns RB_OK (0) or a nonzero RB_ERR_* code; the message is
 * in rb_last_error(). There is no CPU fallback: a failing device step is an
 * error, never a silent host computation.
 */
#ifndef RACON_B200_H_
#define RACON_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB_OK 0
#define RB_ERR_ARG 1      /* invalid argument or input outside documented limits */
#define RB_ERR_CUDA 2     /* CUDA runtime error */
#define RB_ERR_NOMEM 3    /* device or pinned host allocation failed */
#define RB_ERR_DEVICE 4   /* a kernel reported a failure status */
#define RB_ERR_NODEV 5    /* no usable sm_100 device */

typedef struct rb_ctx rb_ctx;

/* Scoring and windowing of one polishing job: racon's -m -x -g -w
 * (src/main.cpp:51-67, passed to createPolisher, src/polisher.hpp:42-48). */
typedef struct rb_params {
    int8_t match;
    int8_t mismatch;
    int8_t gap;
    uint32_t window_length;
} rb_params;

/* Creates a context on CUDA device `device`. Replaces the per-device set-up of
 * the reference plug-in (src/cuda/cudapolisher.cpp:27-66). Returns NULL on
 * failure; rb_create_error() then holds the reason. */
rb_ctx* rb_create(int device, const rb_params* params);
const char* rb_create_error(void);
void rb_destroy(rb_ctx* ctx);
const char* rb_last_error(const rb_ctx* ctx);

/* ---------------------------------------------------------------------
 * Overlap alignment (replaces src/overlap.cpp:179-292 per overlap)
 * ------------------------------------------------------------------- */

/* One overlap, already cut to its aligned spans (src/overlap.cpp:193-197):
 * query = read span, reverse-complemented for '-' strand; target = contig
 * span. q_offset is the read coordinate of query[0] in the orientation used
 * (strand ? q_length - q_end : q_begin, src/overlap.cpp:241); t_begin is the
 * target coordinate of target[0]. Spans are limited to 2^24 bases. */
typedef struct rb_pair {
    const char* query;
    uint32_t query_length;
    const char* target;
    uint32_t target_length;
    uint32_t q_offset;
    uint32_t t_begin;
} rb_pair;

/* Results of rb_align_batch, library-owned. breakpoints holds, for pair i,
 * the (t, q) uint32 pairs breakpoints[bp_offsets[i] .. bp_offsets[i+1]) in
 * racon's order (first match, last match + 1 per window,
 * src/overlap.cpp:259-266). cigars holds the standard CIGAR of pair i at
 * cigars[cigar_offsets[i] .. cigar_offsets[i+1]) (not NUL-terminated) when
 * want_cigar was set, else cigars/cigar_offsets are NULL. */
typedef struct rb_aln_result {
    const int32_t* edit_distance;
    const uint32_t* breakpoints;
    const uint64_t* bp_offsets;
    const char* cigars;
    const uint64_t* cigar_offsets;
} rb_aln_result;

/* Aligns n pairs on the device (edlib NW + path semantics, k doubling from 64,
 * Hirschberg above 1 MiB of traceback data) and derives the window breaking
 * points for window_length from rb_params. */
int rb_align_batch(rb_ctx* ctx, const rb_pair* pairs, size_t n, int want_cigar,
                   rb_aln_result* out);

/* ---------------------------------------------------------------------
 * Window consensus (replaces src/window.cpp:65-142 per window)
 * ------------------------------------------------------------------- */

/* One window: the backbone (target slice) and its layers as racon's
 * Window::add_layer stored them (src/window.cpp:42-63). backbone_quality may
 * be NULL (weight 0 everywhere, racon's dummy '!' quality,
 * src/polisher.cpp:171, :393-395). layer_qualities may be NULL or hold NULL
 * entries (weight 1 per base). begins/ends are backbone coordinates. tgs is 1
 * for racon's WindowType::kTGS (mean read length > 1000,
 * src/polisher.cpp:276-277). id and rank only label the chimeric-window
 * warning (src/window.cpp:133-135). Limits: backbone_length <= 65535,
 * n_layers <= 65535, layer_length <= 65535, begin < end < backbone_length
 * (racon's layers always end on a backbone base). */
typedef struct rb_window {
    const char* backbone;
    const char* backbone_quality;
    uint32_t backbone_length;
    uint32_t n_layers;
    const char* const* layers;
    const char* const* layer_qualities;
    const uint32_t* layer_lengths;
    const uint32_t* begins;
    const uint32_t* ends;
    uint8_t tgs;
    uint64_t id;
    uint32_t rank;
} rb_window;

/* Consensus of window i at consensus[offsets[i] .. offsets[i+1]);
 * polished[i] is 1 when the window had at least two layers (the return value
 * of Window::generate_consensus), else 0 and the consensus is the backbone. */
typedef struct rb_poa_result {
    const char* consensus;
    const uint64_t* offsets;
    const uint8_t* polished;
} rb_poa_result;

/* Computes the consensus of n windows on the device; trim is racon's
 * --no-trimming negation (src/window.cpp:118-139). */
int rb_poa_batch(rb_ctx* ctx, const rb_window* windows, size_t n, int trim,
                 rb_poa_result* out);

/* Device-resident form of rb_poa_batch for throughput measurement: stage
 * packs and copies the windows to the device once, run computes the
 * consensus of every staged window with inputs and outputs already in device
 * memory, fetch copies the results back. rb_poa_batch == stage + run + fetch. */
int rb_poa_stage(rb_ctx* ctx, const rb_window* windows, size_t n, int trim);
int rb_poa_run(rb_ctx* ctx);
int rb_poa_fetch(rb_ctx* ctx, rb_poa_result* out);

/* Plain comparison form of rb_poa_run, for measurement only (no counterpart in
 * the reference): the same per-window device code, but one window per
 * one-warp block in input order, one launch per batch and no work queue.
 * Results are identical to rb_poa_run's; fetch them with rb_poa_fetch. */
int rb_poa_run_plain(rb_ctx* ctx);

/* ---------------------------------------------------------------------
 * Device layer assembly (replaces the layer loop of Polisher::initialize,
 * src/polisher.cpp:384-457): the reads stay in device memory and the layers
 * of every window are cut, filtered and ordered there.
 * ------------------------------------------------------------------- */

/* One entry of racon's sequence table: the targets first, then the reads that
 * are not targets (src/polisher.cpp:209-281). data is uppercase; quality is
 * NULL for FASTA input or when every value is '!' (racon drops it then).
 * forward / reverse: whether some overlap uses the read on that strand
 * (has_data / has_reverse_data of Sequence::transmute,
 * src/polisher.cpp:355-372); targets set forward. Entries with neither are
 * not copied. */
typedef struct rb_sequence {
    const char* data;
    const char* quality;
    uint32_t length;
    uint8_t forward;
    uint8_t reverse;
} rb_sequence;

/* Copies the sequence table to the device and builds the reverse complement
 * and reversed quality (src/sequence.cpp:49-84) of every entry with reverse
 * set. Replaces the previous table and drops windows staged from it. */
int rb_sequences_stage(rb_ctx* ctx, const rb_sequence* sequences, size_t n);

/* One overlap after find_overlap_breaking_points: read and target as indices
 * into the staged table, strand 1 for '-'. */
typedef struct rb_layer_overlap {
    uint32_t q_id;
    uint32_t t_id;
    uint32_t strand;
} rb_layer_overlap;

/* One overlap as racon's Overlap holds it, for alignment from the staged
 * table: read q_id span [q_begin, q_end) and target t_id span
 * [t_begin, t_end) in forward coordinates, strand 1 for '-'. The query is the
 * read span, reverse-complemented for '-' (the span
 * [length - q_end, length - q_begin) of the reverse complement,
 * src/overlap.cpp:193-197); the target is the contig span. */
typedef struct rb_store_pair {
    uint32_t q_id;
    uint32_t q_begin, q_end;
    uint32_t t_id;
    uint32_t t_begin, t_end;
    uint32_t strand;
} rb_store_pair;

/* rb_align_stage for pairs cut from the staged table on the device (no
 * sequence bytes cross the bus); then rb_align_run / rb_align_fetch as for
 * rb_align_stage. Results equal rb_align_batch's on the same spans. */
int rb_align_stage_overlaps(rb_ctx* ctx, const rb_store_pair* pairs, size_t n, int want_cigar);

/* find_overlap_breaking_points and the layer assembly in one call
 * (src/polisher.cpp:462-484 then :384-457): aligns every pair from the staged
 * table, turns the breaking points into layers without leaving the device,
 * and stages window consensus as rb_poa_stage_overlaps does. breakpoints may
 * be NULL; otherwise it receives every pair's edit distance and breaking
 * points (no CIGARs), library-owned until the next call on ctx. */
int rb_poa_stage_alignments(rb_ctx* ctx, size_t n_targets, const rb_store_pair* pairs, size_t n,
                            double quality_threshold, int tgs, int trim, rb_aln_result* breakpoints);

/* Stages window consensus with the layers assembled on the device, as
 * racon's initialize() assembles them (src/polisher.cpp:384-457): windows of
 * rb_params.window_length bases over staged targets 0 .. n_targets-1, in
 * racon's window order; overlap i's breaking points are
 * breakpoints[bp_offsets[i] .. bp_offsets[i+1]) as (t, q) uint32 pairs, the
 * layout of rb_aln_result (first match, last match + 1 per window). A pair
 * becomes a layer of the window holding its first target position unless its
 * query span is below 0.02 * window_length or, for a read with qualities, its
 * mean Phred-33 quality is below quality_threshold; inside a window the
 * layers keep overlap order and then take racon's sort by begin
 * (src/window.cpp:78-85). tgs and trim as for rb_window / rb_poa_batch.
 * Then rb_poa_run / rb_poa_run_plain / rb_poa_fetch (results in window
 * order). The staged table must not change in between. */
int rb_poa_stage_overlaps(rb_ctx* ctx, size_t n_targets, const rb_layer_overlap* overlaps, size_t n,
                          const uint32_t* breakpoints, const uint64_t* bp_offsets, double quality_threshold,
                          int tgs, int trim);

/* Breaking points of overlaps that already carry an alignment (SAM input:
 * src/overlap.cpp:192-200 skips the aligner when the CIGAR is set and walks
 * it in find_breaking_points_from_cigar, :226-292). cigar is the SAM CIGAR
 * (M, =, X, I, D, N, S, H, P); q_offset is the read coordinate before the
 * first aligned base in the orientation used (strand ? q_length - q_end :
 * q_begin); the alignment covers target [t_begin, t_end). Results use
 * rb_aln_result with edit_distance entries set to -1 and no CIGARs. */
typedef struct rb_cigar_overlap {
    const char* cigar;
    uint32_t cigar_length;
    uint32_t q_offset;
    uint32_t t_begin;
    uint32_t t_end;
} rb_cigar_overlap;
int rb_cigar_breakpoints(rb_ctx* ctx, const rb_cigar_overlap* overlaps, size_t n,
                         rb_aln_result* out);

/* Same split for the overlap aligner. */
int rb_align_stage(rb_ctx* ctx, const rb_pair* pairs, size_t n, int want_cigar);
int rb_align_run(rb_ctx* ctx);
int rb_align_fetch(rb_ctx* ctx, rb_aln_result* out);

/* Scheduling of a context's kernels, for callers that run several contexts
 * on one device at once (the serving loop); results do not depend on either.
 * rb_set_yield: windows a warp of the consensus kernel, and pairs or
 * Hirschberg tasks a warp of the alignment kernels, take per launch (0, the
 * default: the kernels are persistent until their work queue is empty). Small
 * values make the kernels of a large job return SMs at every launch boundary,
 * where other contexts' waiting kernels can take them.
 * rb_set_priority: 1 puts the context's work on a stream of the highest
 * priority, 0 on a normal one (between calls). */
int rb_set_yield(rb_ctx* ctx, uint32_t consensus_windows, uint32_t alignment_items);
/* Percent of the SMs the context's persistent kernels fill (1..100; 0 or 100:
 * all), leaving the rest to other contexts' kernels. */
int rb_set_sm_share(rb_ctx* ctx, uint32_t percent);
int rb_set_priority(rb_ctx* ctx, int high);

/* ---------------------------------------------------------------------
 * Autotuner (no counterpart in the reference: racon's CUDA plug-in sizes its
 * batches from fixed constants, src/cuda/cudapolisher.cpp:158-180 and
 * BatchConfig(1023, 200, 256, band) at src/cuda/cudabatch.cpp:56-59).
 * ------------------------------------------------------------------- */

/* Launch choices of one device, shared by every context on it. None of them
 * changes a result. */
typedef struct rb_tuning {
    uint32_t consensus_ctas_per_sm;   /* resident consensus CTAs per SM, 1..3 (4 windows each): windows in flight */
    uint32_t consensus_order;         /* queue order: 0 heaviest window first; 1 size buckets interleaved
                                       * (heaviest, lightest, next heaviest, ...) */
    uint32_t alignment_warps_per_sm;  /* resident alignment warps per SM (one pair or split task each): 4..32 */
    uint32_t tuned;                   /* bit 0: consensus choices measured, bit 1: alignment choices measured */
    double consensus_ms;              /* kernel time of the chosen consensus setting on the tuning batch */
    double alignment_ms;              /* kernel time of the chosen alignment setting on the tuning batch */
} rb_tuning;

/* Measures the candidate launch choices on the batch staged in ctx and keeps
 * the fastest for the device: what & 1 sweeps consensus CTAs per SM x queue
 * order over the staged windows (rb_poa_stage*), what & 2 the resident
 * alignment warps over the staged pairs (rb_align_stage*). Every candidate
 * run must give identical results (checked; RB_ERR_DEVICE otherwise). The
 * staged batch and its results stay as after one run. */
int rb_autotune(rb_ctx* ctx, int what);
/* The device's current choices (defaults until tuned or set). */
int rb_tuning_get(int device, rb_tuning* out);
/* Pins the device's choices (values are clamped to their ranges). */
int rb_tuning_set(int device, const rb_tuning* in);

/* Counters of the last run/batch call of each kind. */
typedef struct rb_stats {
    double kernel_ms;        /* device time of the compute kernels (CUDA events) */
    double h2d_ms, d2h_ms;   /* copy time of the last batch call */
    uint64_t h2d_bytes, d2h_bytes;
    uint64_t launches;       /* kernels launched by the last run */
    uint64_t cells;          /* DP cells (POA: |layer| x |aligned graph|) */
    uint64_t items;          /* windows or pairs processed */
    uint32_t max_nodes;      /* POA: largest graph seen */
    double top_kernel_ms;    /* device time of the dominant kernel */
    uint64_t edge_cells;     /* POA: sum over alignments of |layer| x sum_v (1 + in-degree of v)
                              * over the aligned (sub)graph: the DP's max-plus terms */
} rb_stats;
int rb_poa_stats(const rb_ctx* ctx, rb_stats* out);
int rb_align_stats(const rb_ctx* ctx, rb_stats* out);
/* Counters of the last rb_poa_stage_overlaps (kernel_ms: assembly kernels;
 * items: layers kept; cells: breaking-point pairs examined) and of the last
 * rb_sequences_stage (items: sequences; h2d: the store copy). */
int rb_layer_stats(const rb_ctx* ctx, rb_stats* out);
int rb_sequence_stats(const rb_ctx* ctx, rb_stats* out);

/* ---------------------------------------------------------------------
 * Whole pipeline (createPolisher + initialize + polish, src/main.cpp:152-166)
 * ------------------------------------------------------------------- */

/* Runs racon's pipeline with the device hot path and returns the polished
 * FASTA text (">name tags\nsequence\n" records) in *fasta, allocated with
 * malloc (free with rb_free). fragment = -f, drop_unpolished = !-u.
 * On input errors racon prints "[racon::...] error: ..." and exits(1); this
 * entry point returns RB_ERR_ARG with the same message in rb_pipeline_error().
 * device selects the CUDA device; threads is accepted for -t compatibility. */
int rb_polish_files(const char* sequences_path, const char* overlaps_path,
                    const char* target_path, int fragment, uint32_t window_length,
                    double quality_threshold, double error_threshold, int trim,
                    int8_t match, int8_t mismatch, int8_t gap, uint32_t threads,
                    int drop_unpolished, int device, char** fasta, double* stage_seconds);
const char* rb_pipeline_error(void);

/* A polishing job stopped after racon's initialize() (src/polisher.cpp:192-460:
 * loading, overlap filtering, device alignment + breaking points, windows
 * and layers). rb_job_windows exposes its windows, in racon's window order,
 * as rb_window views valid until rb_job_free; they can be passed directly to
 * rb_poa_batch / rb_poa_stage. stage_seconds (may be NULL) receives load,
 * align and layer-assembly wall seconds. Returns NULL on error
 * (rb_pipeline_error() holds the message). */
typedef struct rb_job rb_job;
rb_job* rb_job_prepare(const char* sequences_path, const char* overlaps_path,
                       const char* target_path, int fragment, uint32_t window_length,
                       double quality_threshold, double error_threshold, int8_t match,
                       int8_t mismatch, int8_t gap, int device, double* stage_seconds);
size_t rb_job_windows(const rb_job* job, const rb_window** windows);
/* The same job as device layer assembly input (rb_sequences_stage,
 * rb_poa_stage_overlaps): its sequence table (targets first), the number of
 * targets, the kept overlaps with their breaking points, and racon's window
 * type (1 = kTGS). Views valid until rb_job_free. */
int rb_job_layer_input(const rb_job* job, const rb_sequence** sequences, size_t* n_sequences, size_t* n_targets,
                       const rb_layer_overlap** overlaps, size_t* n_overlaps, const uint32_t** breakpoints,
                       const uint64_t** bp_offsets, int* tgs);
/* The device context a job was prepared on (borrowed; valid until
 * rb_job_free): its rb_align_stats / rb_layer_stats / rb_sequence_stats
 * describe the job's own alignment and layer assembly. */
rb_ctx* rb_job_context(const rb_job* job);
void rb_job_free(rb_job* job);
void rb_free(void* p);

/* ---------------------------------------------------------------------
 * Serving loop (no counterpart in the reference, which polishes one job per
 * process): polishing jobs are submitted while others run.
 * ------------------------------------------------------------------- */

/* workers: jobs in flight at once. Each worker owns one long-lived device
 * context with its own stream, so device buffers stay allocated from job to
 * job and concurrent jobs' kernels overlap on the GPU. hbm_budget: device
 * bytes the jobs in flight may take by estimate; a queued job is admitted,
 * first in first out, when a worker is idle and its estimated footprint fits
 * beside the jobs in flight (a job alone is always admitted). 0 selects
 * 4 workers and 75% of the device memory.
 *
 * Window consensus is continuously batched: one persistent consensus kernel
 * per server takes windows of every job in flight from a shared device work
 * queue, so a job admitted while others run starts on the first free warps
 * instead of waiting for their launches to drain. The queue has four rings
 * by job size, drained smallest first: up to priority_windows windows (0: a
 * quarter of the kernel's resident windows), up to 4x and 16x that, and
 * larger.
 * consensus_ctas_per_sm (0 or more than 2: 2) sizes that kernel; the rest of each
 * SM stays free for the alignment and layer kernels of newly admitted jobs.
 * shared_consensus = 0 turns the shared kernel off (each job then launches
 * its own consensus kernel, with its scratch capped at hbm_budget / workers).
 * alignment_yield > 0 puts jobs of at most priority_windows windows on the
 * high-priority stream and bounds the alignment work of larger jobs to that
 * many pairs per warp and launch, so that a small job's alignment kernels
 * find free SMs between a large job's launches. alignment_share (1..99, 0:
 * 100) sizes larger jobs' persistent alignment grids for that percent of
 * the SMs (and also puts small jobs on the high-priority stream), leaving
 * the rest to small jobs' alignment. Both apply only to jobs aligned on
 * their own kernels.
 *
 * Overlap alignment is continuously batched the same way when
 * shared_alignment is set: one persistent alignment kernel per server takes
 * the distance passes and path-recursion levels of every job in flight from
 * its own four rings, drained smallest first (up to priority_pairs pairs, 0:
 * the kernel's resident warps; then 4x, 16x and larger). A job waits for
 * each level before publishing the next. alignment_ctas_per_sm (0: 1) sizes
 * the kernel (4 warps per CTA). Its scratch is sized for spans up to
 * alignment_max_span bases (0: 131072); a job with a longer query or target
 * span aligns on its own kernels. large_first_every = k > 0 makes every k-th
 * warp of both shared kernels drain the rings largest first, so that the
 * largest jobs keep a share of the warps under a stream of small ones (0:
 * strict smallest first). Results are unchanged either way. */
typedef struct rb_server_params {
    int device;
    uint32_t workers;
    uint64_t hbm_budget;
    int8_t match;
    int8_t mismatch;
    int8_t gap;
    uint32_t window_length;
    int shared_consensus;
    uint32_t consensus_ctas_per_sm;
    uint32_t priority_windows;
    uint32_t alignment_yield;
    uint32_t alignment_share;
    int shared_alignment;
    uint32_t alignment_ctas_per_sm;
    uint32_t alignment_max_span;
    uint32_t priority_pairs;
    uint32_t large_first_every;
} rb_server_params;

/* One job: racon's inputs and per-job flags (-f, -q, -e, --no-trimming, -u). */
typedef struct rb_server_job {
    const char* sequences_path;
    const char* overlaps_path;
    const char* target_path;
    int fragment;
    double quality_threshold;
    double error_threshold;
    int trim;
    int drop_unpolished;
} rb_server_job;

/* Times of one job in seconds on the server's clock (0 = creation), its
 * estimated footprint and the worker that ran it. */
typedef struct rb_server_times {
    double submitted, admitted, finished;
    double stage_seconds[4];  /* load, align, layers, consensus */
    uint64_t footprint;
    uint32_t worker;
} rb_server_times;

typedef struct rb_server rb_server;
/* Returns NULL on failure; rb_create_error() then holds the reason. */
rb_server* rb_server_create(const rb_server_params* params);
/* Queues a job (paths are copied) and returns its ticket. */
int rb_server_submit(rb_server* server, const rb_server_job* job, uint64_t* ticket);
/* Waits for a job. On RB_OK *fasta holds the polished FASTA text (malloc,
 * free with rb_free); on failure *fasta is NULL and rb_server_error() holds
 * the message. times may be NULL. A ticket can be waited for once. */
int rb_server_wait(rb_server* server, uint64_t ticket, char** fasta, rb_server_times* times);
/* Message of the calling thread's last failed rb_server_submit / _wait. */
const char* rb_server_error(void);
/* Jobs queued and in flight. */
int rb_server_load(rb_server* server, uint32_t* queued, uint32_t* in_flight, uint64_t* in_flight_bytes);
/* Cancels queued jobs, waits for the jobs in flight and frees the server. */
void rb_server_destroy(rb_server* server);

/* Edit distance of one pair (edlib NW semantics, the same value as
 * rb_align_batch's edit_distance) that allocates no memory. No counterpart in
 * the reference: racon always aligns through edlibAlign, which allocates.
 *
 * For callers that cannot allocate at the time they align: code that must not
 * synchronise the device (cudaMalloc and cudaFree can wait for all work on
 * it), and code running under a fixed device-memory budget that has already
 * been handed out (a failed allocation there would end the job). Scratch lives in one static device array of about
 * 1.6 MB per device, so each sequence is limited to 131072 bytes; longer
 * inputs return RB_ERR_ARG with that message. The pair must have at most 32
 * distinct byte values, else *distance is set to -1.
 *
 * query, target and distance are DEVICE pointers; the kernel runs one warp on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and the call returns
 * without waiting for it. The current device's first call loads the kernel's
 * module and should come before any stream capture; every call looks up the
 * array's device address again (no allocation), so a call after a
 * cudaDeviceReset uses the array of the new context. All calls on a device share the array: it keeps the last
 * call's contents and nothing in it needs to start at zero, but calls whose
 * kernels can overlap (different streams without ordering) race on it and
 * give wrong results, so order them on one stream. `err` (optional, capacity
 * err_capacity bytes) receives a message on failure; no context is used. */
int rb_nw_distance_noalloc(const char* query, uint32_t query_length, const char* target, uint32_t target_length,
                           int32_t* distance, void* stream, char* err, uint32_t err_capacity);

#ifdef __cplusplus
}
#endif

#endif /* RACON_B200_H_ */
