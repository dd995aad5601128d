// racon's C++ polishing API (drop-in for the reference's src/polisher.hpp:36-98
// and src/sequence.hpp:26-74), backed by the B200 device path.
//
// createPolisher keeps the reference signature (src/polisher.hpp:42-48,
// including the CUDA-plug-in arguments, which are accepted and ignored: the
// device path is always used). Polisher::initialize and Polisher::polish keep
// their signatures and behaviour; the two protected virtuals that the
// reference's CUDA plug-in overrides (find_overlap_breaking_points,
// src/polisher.hpp:75, and polish) run on the device through the C ABI in
// include/racon_b200.h. There is no CPU path.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../../include/racon_b200.h"

struct rb_job;

namespace racon {

class Sequence {
public:
    ~Sequence() = default;
    const std::string& name() const { return name_; }
    const std::string& data() const { return data_; }
    const std::string& reverse_complement() const { return reverse_complement_; }
    const std::string& quality() const { return quality_; }
    const std::string& reverse_quality() const { return reverse_quality_; }
    void create_reverse_complement();
    void transmute(bool has_name, bool has_data, bool has_reverse_data);

    // FASTA record (data uppercased)
    Sequence(const char* name, uint32_t name_length, const char* data, uint32_t data_length);
    // FASTQ record; the quality is dropped when every value is '!'
    Sequence(const char* name, uint32_t name_length, const char* data, uint32_t data_length,
             const char* quality, uint32_t quality_length);
    Sequence(const std::string& name, const std::string& data);
    Sequence(const Sequence&) = delete;
    const Sequence& operator=(const Sequence&) = delete;

private:
    std::string name_;
    std::string data_;
    std::string reverse_complement_;
    std::string quality_;
    std::string reverse_quality_;
};

std::unique_ptr<Sequence> createSequence(const std::string& name, const std::string& data);

enum class PolisherType {
    kC,  // contig polishing
    kF   // fragment error correction
};

class Overlap;
class Window;

class Polisher;
std::unique_ptr<Polisher> createPolisher(const std::string& sequences_path,
    const std::string& overlaps_path, const std::string& target_path,
    PolisherType type, uint32_t window_length, double quality_threshold,
    double error_threshold, bool trim, int8_t match, int8_t mismatch, int8_t gap,
    uint32_t num_threads, uint32_t cuda_batches = 0,
    bool cuda_banded_alignment = false, uint32_t cudaaligner_batches = 0,
    uint32_t cudaaligner_band_width = 0);

class Polisher {
public:
    virtual ~Polisher();

    virtual void initialize();

    virtual void polish(std::vector<std::unique_ptr<Sequence>>& dst,
        bool drop_unpolished_sequences);

    // CUDA device used by this polisher (default 0, or RACON_B200_DEVICE)
    int device() const { return device_; }
    // wall seconds of the stages of the last run: load, align, layers, consensus
    const double* stage_seconds() const { return stage_s_; }

    friend std::unique_ptr<Polisher> createPolisher(const std::string& sequences_path,
        const std::string& overlaps_path, const std::string& target_path,
        PolisherType type, uint32_t window_length, double quality_threshold,
        double error_threshold, bool trim, int8_t match, int8_t mismatch, int8_t gap,
        uint32_t num_threads, uint32_t cuda_batches, bool cuda_banded_alignment,
        uint32_t cudaaligner_batches, uint32_t cudaaligner_band_width);
    friend struct ::rb_job;
    friend rb_ctx* ::rb_job_context(const rb_job*);
    friend int ::rb_job_layer_input(const rb_job*, const rb_sequence**, size_t*, size_t*,
                                    const rb_layer_overlap**, size_t*, const uint32_t**, const uint64_t**, int*);
    friend std::unique_ptr<Polisher> createPolisherOnContext(rb_ctx* ctx, int device,
        const std::string& sequences_path, const std::string& overlaps_path,
        const std::string& target_path, PolisherType type, uint32_t window_length,
        double quality_threshold, double error_threshold, bool trim, int8_t match,
        int8_t mismatch, int8_t gap);

protected:
    Polisher(const std::string& sequences_path, const std::string& overlaps_path,
        const std::string& target_path, int sequences_format, int overlaps_format,
        int target_format, PolisherType type, uint32_t window_length,
        double quality_threshold, double error_threshold, bool trim, int8_t match,
        int8_t mismatch, int8_t gap, uint32_t num_threads, rb_ctx* borrowed_ctx = nullptr,
        int device = 0);
    Polisher(const Polisher&) = delete;
    const Polisher& operator=(const Polisher&) = delete;
    virtual void find_overlap_breaking_points(std::vector<std::unique_ptr<Overlap>>& overlaps);
    // Window layers on the host from the kept overlaps (the loop of
    // src/polisher.cpp:401-457), for callers that want rb_window views; the
    // polishing path assembles them on the device instead.
    void assemble_host_layers();

    std::string sequences_path_, overlaps_path_, target_path_;
    int sequences_format_, overlaps_format_, target_format_;

    PolisherType type_;
    double quality_threshold_;
    double error_threshold_;
    bool trim_;
    int8_t match_, mismatch_, gap_;

    std::vector<std::unique_ptr<Sequence>> sequences_;
    std::vector<uint32_t> targets_coverages_;
    std::string dummy_quality_;

    uint32_t window_length_;
    std::vector<std::shared_ptr<Window>> windows_;
    bool tgs_ = true;

    // input of the device layer assembly (rb_sequences_stage,
    // rb_poa_stage_overlaps): the sequence table with the strands the
    // overlaps use, and each kept overlap's ids, strand and breaking points
    std::vector<rb_sequence> sequence_table_;
    std::vector<rb_layer_overlap> layer_overlaps_;
    std::vector<uint32_t> breakpoints_;
    std::vector<uint64_t> bp_offsets_;
    bool staged_ = false;
    size_t targets_size_ = 0;

    uint32_t num_threads_;
    int device_ = 0;
    rb_ctx* ctx_ = nullptr;
    bool owns_ctx_ = true;
    double stage_s_[4] = {0, 0, 0, 0};
};

// Not part of racon's API: a polisher that runs on an existing context
// (created with the same match / mismatch / gap / window length), which it
// does not destroy. The serving loop gives each worker one long-lived
// context so that device buffers stay allocated from job to job.
std::unique_ptr<Polisher> createPolisherOnContext(rb_ctx* ctx, int device,
    const std::string& sequences_path, const std::string& overlaps_path,
    const std::string& target_path, PolisherType type, uint32_t window_length,
    double quality_threshold, double error_threshold, bool trim, int8_t match,
    int8_t mismatch, int8_t gap);

// One polishing job on a borrowed context, with racon's fatal errors turned
// into a return value: RB_OK and the FASTA text (">name tags\nsequence\n"
// records), or RB_ERR_ARG and the "[racon::...] error: ..." message.
// stage_seconds (may be NULL) receives load, align, layers and consensus
// seconds. Used by the serving loop.
int polish_job_on_context(rb_ctx* ctx, int device, const std::string& sequences_path,
    const std::string& overlaps_path, const std::string& target_path, bool fragment,
    uint32_t window_length, double quality_threshold, double error_threshold, bool trim,
    int8_t match, int8_t mismatch, int8_t gap, bool drop_unpolished, std::string* fasta,
    std::string* error, double* stage_seconds);

// Creates the polisher and runs initialize + polish; used by the CLI and the
// C entry point rb_polish_files. Returns the polished records.
std::vector<std::unique_ptr<Sequence>> polish_files(const std::string& sequences_path,
    const std::string& overlaps_path, const std::string& target_path, PolisherType type,
    uint32_t window_length, double quality_threshold, double error_threshold, bool trim,
    int8_t match, int8_t mismatch, int8_t gap, uint32_t num_threads, bool drop_unpolished,
    double* stage_seconds);

}  // namespace racon
