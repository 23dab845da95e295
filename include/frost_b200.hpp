// C++20 header-only wrapper of the frost_b200 C ABI with frost's stage names
// and error behaviour: invalid arguments throw std::invalid_argument, every
// other failure throws frost::b200::Error (a std::runtime_error carrying the
// status code), as frost's own stages do (lib/cuda/gpu_utils.cuh:13-20).
//
//   frost::b200::RFICleaner   ~ frost::prepare::rfi::RFICleaner
//                               (include/frost/prepare/rfi.hpp:243-297)
//   frost::b200::generate_dm_list ~ frost::dedisp::generate_dm_list
//                               (include/frost/dedisp/dedisp.hpp:29-30)
//   frost::b200::FDMTBoxcar   ~ the dmt::FDMTBoxcar call shape frost uses
//                               (lib/pipeline/pipeline.cpp:316-367, 493-517, 598-608)
//   frost::b200::BeamServer   ~ many beams on one GPU (no frost counterpart)
//   frost::b200::CandWriter, cand_filename ~ frost::output (cand_writer.hpp)
//   frost::b200::GulpPrefetch ~ GulpPrefetch (lib/pipeline/pipeline.cpp:105-262),
//                               delivering gulps on the device
//   frost::b200::CandidatePostprocessPlan, ClusterLabelPlan,
//   MergeCandidatesPlan, SubbandDedupPlan, are_coincident,
//   subband_time_shift_samples, subband_dm_step
//                             ~ frost::search (include/frost/search/*.hpp),
//                               on the device
//
// Link with frost_b200/lib/libfrost_b200.so.
#pragma once

#include <algorithm>
#include <cstdint>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "frost_b200.h"

namespace frost::b200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), m_code(code) {}
    int code() const noexcept { return m_code; }

private:
    int m_code;
};

inline void check(int rc) {
    if (rc == FROST_OK)
        return;
    const std::string msg = frost_last_error();
    if (rc == FROST_ERR_INVALID_ARGUMENT)
        throw std::invalid_argument(msg);
    throw Error(rc, msg);
}

inline std::vector<float> generate_dm_list(const frost_dedisp_plan_config& cfg) {
    size_t n = 0;
    check(frost_generate_dm_list(&cfg, nullptr, 0, &n));
    std::vector<float> out(n);
    check(frost_generate_dm_list(&cfg, out.data(), out.size(), &n));
    return out;
}

/** Bytes of one packed time-major row of `layout`. */
inline size_t row_bytes(const frost_block_layout& layout) {
    static constexpr size_t bits[] = {1, 2, 4, 8, 16, 32, 32};
    if (layout.dtype < FROST_UINT1 || layout.dtype > FROST_FLOAT32)
        throw std::invalid_argument("frost_block_layout: unknown dtype");
    return layout.nchans * bits[layout.dtype] / 8;
}

inline frost_rfi_config default_rfi_config() {
    frost_rfi_config c;
    frost_rfi_config_default(&c);
    return c;
}

/** RFI excision and normalisation of packed time-major gulps on a GPU. */
class RFICleaner {
public:
    RFICleaner(const frost_rfi_config& cfg, const frost_block_layout& layout, float baseline_length,
               int device = 0)
        : m_nchans(layout.nchans), m_row_bytes(row_bytes(layout)) {
        check(frost_rfi_create(&cfg, &layout, baseline_length, device, &m_h));
    }
    RFICleaner(const RFICleaner&)            = delete;
    RFICleaner& operator=(const RFICleaner&) = delete;
    RFICleaner(RFICleaner&& o) noexcept { *this = std::move(o); }
    RFICleaner& operator=(RFICleaner&& o) noexcept {
        std::swap(m_h, o.m_h);
        std::swap(m_nchans, o.m_nchans);
        std::swap(m_row_bytes, o.m_row_bytes);
        m_host.swap(o.m_host);
        m_mask.swap(o.m_mask);
        return *this;
    }
    ~RFICleaner() {
        if (m_h != nullptr)
            frost_rfi_destroy(m_h);
    }

    /** Host block in, calibrated float32 [channel][capacity] out (host, low
     * frequency first), valid until the next call. */
    std::span<const float> execute_normalized(std::span<const uint8_t> block, size_t nsamps = 0) {
        (void)execute_normalized_device(block.data(), block.size(), nsamps, false, nullptr);
        m_host.resize(m_nchans * (block.size() / m_row_bytes));
        check(frost_rfi_download_normalized(m_h, m_host.data(), m_host.size()));
        return m_host;
    }

    /** The same on a host or device block; returns the device waterfall. */
    const float* execute_normalized_device(const uint8_t* block, size_t bytes, size_t nsamps,
                                           bool block_on_device, void* stream) {
        const float* out = nullptr;
        check(frost_rfi_execute_normalized(m_h, block, bytes, nsamps, block_on_device ? 1 : 0, stream,
                                           &out));
        return out;
    }

    /** The cleaner's own stream (a cudaStream_t). */
    void* stream() const {
        void* s = nullptr;
        check(frost_rfi_get_stream(m_h, &s));
        return s;
    }

    /** 1 = good, 0 = masked, in the cleaner's (data) channel order. */
    std::span<const uint8_t> channel_mask() {
        m_mask.resize(m_nchans);
        check(frost_rfi_channel_mask(m_h, m_mask.data(), m_mask.size()));
        return m_mask;
    }

    frost_rfi_report report() const {
        frost_rfi_report r;
        check(frost_rfi_get_report(m_h, &r));
        return r;
    }

    size_t memory_usage() const {
        size_t b = 0;
        check(frost_rfi_memory_usage(m_h, &b));
        return b;
    }

private:
    frost_rfi* m_h = nullptr;
    size_t m_nchans = 0, m_row_bytes = 1;
    std::vector<float> m_host;
    std::vector<uint8_t> m_mask;
};

/** Candidates of one execute/drain plus frost's drop counters. */
struct CandidateResult {
    std::vector<frost_candidate> candidates;
    uint64_t dropped_global = 0, dropped_per_dm = 0;
    bool overflowed() const { return dropped_global > 0 || dropped_per_dm > 0; }
};

/** Streaming FDMT + boxcar/trapezoid search of one beam. */
class FDMTBoxcar {
public:
    FDMTBoxcar(const frost_dedisp_plan_config& plan, const frost_boxcar_config& cfg,
               std::span<const uint8_t> kill_mask = {}, size_t memory_budget = 0, int device = 0)
        : m_nchans(plan.nchans) {
        if (!kill_mask.empty() && kill_mask.size() != plan.nchans)
            throw std::invalid_argument("FDMTBoxcar: kill_mask must have nchans entries");
        check(frost_search_create(&plan, &cfg, kill_mask.empty() ? nullptr : kill_mask.data(),
                                  memory_budget, device, &m_h));
    }
    FDMTBoxcar(const FDMTBoxcar&)            = delete;
    FDMTBoxcar& operator=(const FDMTBoxcar&) = delete;
    FDMTBoxcar(FDMTBoxcar&& o) noexcept { *this = std::move(o); }
    FDMTBoxcar& operator=(FDMTBoxcar&& o) noexcept {
        std::swap(m_h, o.m_h);
        std::swap(m_nchans, o.m_nchans);
        return *this;
    }
    ~FDMTBoxcar() {
        if (m_h != nullptr)
            frost_search_destroy(m_h);
    }

    /** Host waterfall [nchans][nsamps]; an empty mask means the
     * constructor's kill mask. */
    CandidateResult execute(std::span<const float> waterfall, std::span<const uint8_t> mask = {}) {
        if (m_nchans == 0 || waterfall.size() % m_nchans != 0)
            throw std::invalid_argument("FDMTBoxcar: waterfall is not [nchans][nsamps]");
        check(frost_search_execute(m_h, waterfall.data(), waterfall.size() / m_nchans, 0,
                                   mask_ptr(mask), nullptr));
        return result();
    }

    /** The engine's own stream (a cudaStream_t). */
    void* stream() const {
        void* s = nullptr;
        check(frost_search_get_stream(m_h, &s));
        return s;
    }

    /** Device waterfall [nchans][nsamps], read after the work queued on
     * `stream` (default: the engine's own stream; the waterfall must then
     * be complete). */
    CandidateResult execute_device(const float* waterfall, size_t nsamps,
                                   std::span<const uint8_t> mask = {}, void* stream = nullptr) {
        check(frost_search_execute(m_h, waterfall, nsamps, 1, mask_ptr(mask), stream ? stream : this->stream()));
        return result();
    }

    CandidateResult drain() {
        check(frost_search_drain(m_h));
        return result();
    }

    uint64_t get_candidate_frontier() const {
        uint64_t s = 0;
        check(frost_search_frontier(m_h, &s));
        return s;
    }

    frost_search_info info() const {
        frost_search_info i;
        check(frost_search_get_info(m_h, &i));
        return i;
    }

    CandidateResult result() const {
        CandidateResult r;
        size_t n = 0;
        check(frost_search_result_count(m_h, &n, &r.dropped_global, &r.dropped_per_dm));
        r.candidates.resize(n);
        if (n != 0)
            check(frost_search_results(m_h, r.candidates.data(), n, &n));
        return r;
    }

    /** The C handle (for calls that read the engine's results in place). */
    frost_search* handle() const { return m_h; }

private:
    const uint8_t* mask_ptr(std::span<const uint8_t> mask) const {
        if (mask.empty())
            return nullptr;
        if (mask.size() != m_nchans)
            throw std::invalid_argument("FDMTBoxcar: mask must have nchans entries");
        return mask.data();
    }

    frost_search* m_h = nullptr;
    size_t m_nchans   = 0;
};

/** One beam's per-gulp body of frost's Pipeline::execute_block
 * (lib/pipeline/pipeline.cpp:529-619): clean + normalise on the GPU, the
 * channel mask reversed into FDMT (ascending-frequency) order when the data
 * are descending (fdmt_kill_mask, :334-344), search, and frost's
 * searched-samples accounting (:610-614). */
class GulpPipeline {
public:
    GulpPipeline(const frost_rfi_config& rfi, const frost_block_layout& layout, float baseline_length,
                 const frost_dedisp_plan_config& plan, const frost_boxcar_config& search, int device = 0)
        : m_layout(layout), m_rfi(rfi, layout, baseline_length, device),
          m_search(plan, search, fdmt_order(m_rfi.channel_mask()), 0, device) {
        m_max_delay = m_search.info().dt_max;
    }

    /** One host gulp (a whole block of max_nsamps rows, `nread` valid). */
    CandidateResult execute(std::span<const uint8_t> block, size_t nread) {
        return execute_ptr(block.data(), block.size(), nread, false, nullptr);
    }

    /** One gulp at a host or device pointer. */
    CandidateResult execute_ptr(const uint8_t* block, size_t bytes, size_t nread, bool on_device,
                                void* stream) {
        // a device block without a stream is read on the cleaner's stream;
        // the engine reads the waterfall after the cleaner's work
        void* s         = stream != nullptr ? stream : m_rfi.stream();
        const float* wf = m_rfi.execute_normalized_device(block, bytes, nread, on_device, s);
        const auto mask = fdmt_order(m_rfi.channel_mask());
        auto res        = m_search.execute_device(wf, m_layout.max_nsamps, mask, s);
        m_read += nread;
        const uint64_t previous = m_read - nread;
        if (m_read > m_max_delay)
            m_searched += m_read - std::max<uint64_t>(previous, m_max_delay);
        return res;
    }

    /** End of stream: closes the open runs (pipeline.cpp:517). */
    CandidateResult flush() { return m_search.drain(); }

    uint64_t nsamps_processed() const { return m_searched; }
    RFICleaner& rfi() { return m_rfi; }
    FDMTBoxcar& search() { return m_search; }

private:
    std::vector<uint8_t> fdmt_order(std::span<const uint8_t> m) const {
        std::vector<uint8_t> v(m.begin(), m.end());
        if (m_layout.df < 0.0)
            std::reverse(v.begin(), v.end());
        return v;
    }

    frost_block_layout m_layout;
    RFICleaner m_rfi;
    FDMTBoxcar m_search;
    uint64_t m_max_delay = 0, m_read = 0, m_searched = 0;
};

/** Many beams on one GPU (frost_server_*): beams admitted by device memory,
 * queued gulps taken by worker slots, per-gulp latency recorded. */
class BeamServer {
public:
    explicit BeamServer(int device = 0, size_t memory_budget = 0, uint32_t slots = 4) {
        check(frost_server_create(device, memory_budget, slots, &m_h));
    }
    BeamServer(const BeamServer&)            = delete;
    BeamServer& operator=(const BeamServer&) = delete;
    ~BeamServer() {
        if (m_h != nullptr)
            frost_server_destroy(m_h);
    }

    /** Throws Error with code FROST_ERR_OUT_OF_MEMORY when refused. */
    uint32_t add_beam(const frost_rfi_config& rfi, const frost_block_layout& layout, float baseline_length,
                      const frost_dedisp_plan_config& plan, const frost_boxcar_config& search) {
        uint32_t beam = 0;
        check(frost_server_add_beam(m_h, &rfi, &layout, baseline_length, &plan, &search, &beam));
        return beam;
    }
    void remove_beam(uint32_t beam) { check(frost_server_remove_beam(m_h, beam)); }

    /** The block stays owned by the caller until wait() returns the ticket. */
    uint64_t submit(uint32_t beam, const uint8_t* block, size_t bytes, size_t nread, bool on_device) {
        uint64_t t = 0;
        check(frost_server_submit(m_h, beam, block, bytes, nread, on_device ? 1 : 0, &t));
        return t;
    }

    /** Candidates of the gulp (at most `capacity`) and its latency. */
    std::vector<frost_candidate> wait(uint64_t ticket, size_t capacity, double* latency_s = nullptr) {
        std::vector<frost_candidate> out(capacity);
        size_t n = 0;
        check(frost_server_wait(m_h, ticket, out.data(), out.size(), &n, latency_s));
        out.resize(n);
        return out;
    }

    std::vector<frost_candidate> drain(uint32_t beam, size_t capacity) {
        std::vector<frost_candidate> out(capacity);
        size_t n = 0;
        check(frost_server_drain(m_h, beam, out.data(), out.size(), &n));
        out.resize(n);
        return out;
    }

    frost_server_stats stats() const {
        frost_server_stats s;
        check(frost_server_get_stats(m_h, &s));
        return s;
    }
    void reset_stats() { check(frost_server_reset_stats(m_h)); }

    /** Device blocks that pinned host gulps are uploaded into at submit. */
    void set_staging(uint32_t beam, uint32_t slots) { check(frost_server_set_staging(m_h, beam, slots)); }
    /** Caps the beam's level and search kernels at `ctas_per_sm` CTAs per SM. */
    void set_residency(uint32_t beam, int ctas_per_sm) { check(frost_server_set_residency(m_h, beam, ctas_per_sm)); }

    /** Adds CandidatePostprocessPlan after every gulp of `beam`. */
    void set_postprocess(uint32_t beam, const frost_postprocess_config& cfg) {
        check(frost_server_set_postprocess(m_h, beam, &cfg));
    }

    std::vector<frost_giant> wait_giants(uint64_t ticket, size_t capacity, double* latency_s = nullptr) {
        std::vector<frost_giant> out(capacity);
        size_t n = 0;
        check(frost_server_wait_giants(m_h, ticket, out.data(), out.size(), &n, latency_s));
        out.resize(n);
        return out;
    }

    std::vector<frost_giant> drain_giants(uint32_t beam, size_t capacity) {
        std::vector<frost_giant> out(capacity);
        size_t n = 0;
        check(frost_server_drain_giants(m_h, beam, out.data(), out.size(), &n));
        out.resize(n);
        return out;
    }

private:
    frost_server* m_h = nullptr;
};

/** frost's GulpPrefetch (lib/pipeline/pipeline.cpp:105-262) on the device:
 * the next gulp is read and copied to the GPU while the current one is
 * searched. */
class GulpPrefetch {
public:
    /** A file of packed rows after `header_bytes`. */
    GulpPrefetch(const std::string& path, uint64_t header_bytes, size_t block_rows, size_t row_bytes,
                 int depth = 2, int device = 0) {
        check(frost_prefetch_create_file(path.c_str(), header_bytes, block_rows, row_bytes, depth, device, &m_h));
    }
    /** A caller block source (runs on the prefetch thread). */
    GulpPrefetch(frost_read_fn read, void* ctx, size_t block_rows, size_t row_bytes, int depth = 2,
                 int device = 0) {
        check(frost_prefetch_create(block_rows, row_bytes, depth, device, read, ctx, &m_h));
    }
    /** The rows of a SIGPROC filterbank after its header (header()). */
    GulpPrefetch(const std::string& sigproc_path, size_t block_rows, int depth = 2, int device = 0) {
        check(frost_prefetch_create_sigproc(sigproc_path.c_str(), block_rows, depth, device, &m_header, &m_h));
    }
    const frost_sigproc_header& header() const { return m_header; }
    GulpPrefetch(const GulpPrefetch&)            = delete;
    GulpPrefetch& operator=(const GulpPrefetch&) = delete;
    ~GulpPrefetch() {
        if (m_h != nullptr)
            frost_prefetch_destroy(m_h);
    }
    struct Gulp {
        const uint8_t* device = nullptr;
        size_t nread          = 0; // 0 at the end of the source
    };
    Gulp next(void* stream = nullptr) {
        Gulp g;
        check(frost_prefetch_next(m_h, stream, &g.device, &g.nread));
        return g;
    }
    frost_prefetch_stats stats() const {
        frost_prefetch_stats s{};
        check(frost_prefetch_get_stats(m_h, &s));
        return s;
    }

private:
    frost_prefetch* m_h = nullptr;
    frost_sigproc_header m_header{};
};

/** The header of a SIGPROC filterbank (frost's file input,
 * lib/pipeline/input.cpp:32-69). */
inline frost_sigproc_header read_sigproc_header(const std::string& path) {
    frost_sigproc_header h{};
    check(frost_sigproc_read_header(path.c_str(), &h));
    return h;
}

/** BlockLayout of a SIGPROC file's rows for gulps of `block_rows`. */
inline frost_block_layout sigproc_layout(const frost_sigproc_header& h, uint64_t block_rows) {
    frost_block_layout l{};
    check(frost_sigproc_layout(&h, block_rows, &l));
    return l;
}

/** output::CandWriter (include/frost/output/cand_writer.hpp:38-55). */
class CandWriter {
public:
    CandWriter(const std::string& path, double dt, bool append = false) {
        check(frost_cand_writer_open(path.c_str(), dt, append ? 1 : 0, &m_h));
    }
    CandWriter(const CandWriter&)            = delete;
    CandWriter& operator=(const CandWriter&) = delete;
    ~CandWriter() {
        if (m_h != nullptr)
            frost_cand_writer_close(m_h);
    }
    void write(std::span<const frost_giant> giants, uint64_t first_samp_idx = 0) {
        check(frost_cand_writer_write(m_h, giants.data(), giants.size(), first_samp_idx));
    }

private:
    frost_cand_writer* m_h = nullptr;
};

inline std::string cand_filename(int64_t utc, uint64_t beam) {
    char buf[64];
    check(frost_cand_filename(utc, beam, buf, sizeof(buf)));
    return buf;
}

/** frost::pipeline::MemoryEstimate for this implementation's device
 * buffers (frost_estimate_memory); `post` may be null. */
inline frost_memory_estimate estimate_memory(const frost_rfi_config& rfi, const frost_block_layout& layout,
                                             float baseline_length, const frost_dedisp_plan_config& plan,
                                             const frost_boxcar_config& search,
                                             const frost_postprocess_config* post = nullptr) {
    frost_memory_estimate e{};
    check(frost_estimate_memory(&rfi, &layout, baseline_length, &plan, &search, post, &e));
    return e;
}

/** frost::pipeline::check_memory on the device (frost_check_memory): may
 * lower the gulp in `layout` and `plan`; throws frost::b200::Error with
 * FROST_ERR_OUT_OF_MEMORY when it cannot. */
inline frost_memory_check check_memory(const frost_rfi_config& rfi, frost_block_layout& layout, float baseline_length,
                                       frost_dedisp_plan_config& plan, const frost_boxcar_config& search,
                                       bool gulp_is_default, uint64_t available_bytes = 0,
                                       const frost_postprocess_config* post = nullptr,
                                       uint64_t memory_limit_bytes = 0, int device = 0) {
    frost_memory_check c{};
    check(frost_check_memory(&rfi, &layout, baseline_length, &plan, &search, post, gulp_is_default ? 1 : 0,
                             available_bytes, memory_limit_bytes, device, &c));
    return c;
}

/** config::SearchConfig's post-processing defaults (config.hpp:57-97). */
inline frost_postprocess_config default_postprocess_config() {
    frost_postprocess_config c{};
    c.boxcar_max        = 4096;
    c.max_candidates    = 131072;
    c.cand_sep_time     = 3;
    c.cand_sep_filter   = 3;
    c.cand_sep_dm       = 200;
    c.detect_thresh     = 6.0F;
    c.cand_sep_dm_smear = 8.0F;
    c.cluster           = 1;
    c.subband_dedup     = FROST_DEDUP_TRANSITIVE;
    return c;
}

struct CandidatePostprocessResult {
    std::vector<frost_giant> candidates;
    double cluster_s = 0.0;
    double dedup_s   = 0.0;
    uint64_t pending_candidates = 0;
};

/** search::CandidatePostprocessPlan (postprocess.hpp:28-62) on the device. */
class CandidatePostprocessPlan {
public:
    CandidatePostprocessPlan(const frost_postprocess_config& cfg, const frost_postprocess_layout& layout,
                             int device = 0) {
        check(frost_postprocess_create(&cfg, &layout, device, &m_h));
    }
    CandidatePostprocessPlan(const CandidatePostprocessPlan&)            = delete;
    CandidatePostprocessPlan& operator=(const CandidatePostprocessPlan&) = delete;
    ~CandidatePostprocessPlan() {
        if (m_h != nullptr)
            frost_postprocess_destroy(m_h);
    }

    /** Over raw rows (host memory, or device memory when on_device). */
    CandidatePostprocessResult execute(std::span<const frost_candidate> rows, uint64_t samples_read,
                                       uint64_t duration_samples, bool final_call, uint64_t frontier,
                                       bool on_device = false) {
        frost_postprocess_result r{};
        check(frost_postprocess_execute(m_h, rows.data(), rows.size(), on_device ? 1 : 0, samples_read,
                                        duration_samples, final_call ? 1 : 0, frontier, &r));
        return collect(r);
    }
    /** Over the search engine's last results, in place on the device. */
    CandidatePostprocessResult execute(FDMTBoxcar& engine, uint64_t samples_read, uint64_t duration_samples,
                                       bool final_call, uint64_t frontier) {
        frost_postprocess_result r{};
        check(frost_postprocess_execute_search(m_h, engine.handle(), samples_read, duration_samples,
                                               final_call ? 1 : 0, frontier, &r));
        return collect(r);
    }
    uint64_t memory_usage() const {
        uint64_t b = 0;
        check(frost_postprocess_memory_usage(m_h, &b));
        return b;
    }
    static uint64_t estimate_memory(const frost_postprocess_config& cfg) {
        uint64_t b = 0;
        check(frost_postprocess_estimate_memory(&cfg, &b));
        return b;
    }

private:
    CandidatePostprocessResult collect(const frost_postprocess_result& r) {
        CandidatePostprocessResult out;
        out.candidates.resize(r.count);
        size_t n = 0;
        check(frost_postprocess_results(m_h, out.candidates.data(), out.candidates.size(), &n));
        out.cluster_s          = r.cluster_s;
        out.dedup_s            = r.dedup_s;
        out.pending_candidates = r.pending_candidates;
        return out;
    }
    frost_postprocess* m_h = nullptr;
};

/** search::ClusterLabelPlan (clustering.hpp:51-66) on the device. */
class ClusterLabelPlan {
public:
    explicit ClusterLabelPlan(int mode = FROST_CLUSTER_CHAIN, int device = 0) : m_mode(mode), m_device(device) {}
    std::vector<uint64_t> execute(std::span<const frost_giant> giants, const frost_cluster_tolerances& tol) const {
        std::vector<uint64_t> labels(giants.size());
        check(frost_cluster_labels(giants.data(), giants.size(), &tol, m_mode, labels.data(), m_device));
        return labels;
    }

private:
    int m_mode, m_device;
};

/** search::MergeCandidatesPlan (merge.hpp:16-24) on the device. */
class MergeCandidatesPlan {
public:
    explicit MergeCandidatesPlan(int device = 0) : m_device(device) {}
    std::vector<frost_giant> execute(std::span<const frost_giant> giants, std::span<const uint64_t> labels) const {
        if (giants.size() != labels.size())
            throw std::invalid_argument("candidates/labels size mismatch");
        std::vector<frost_giant> out(giants.size());
        size_t n = 0;
        check(frost_merge_candidates(giants.data(), labels.data(), giants.size(), out.data(), &n, m_device));
        out.resize(n);
        return out;
    }

private:
    int m_device;
};

/** search::SubbandDedupPlan (subband_dedup.hpp:62-77) on the device. */
class SubbandDedupPlan {
public:
    explicit SubbandDedupPlan(int mode = FROST_DEDUP_TRANSITIVE, int device = 0) : m_mode(mode), m_device(device) {}
    std::vector<frost_giant> execute(std::span<const frost_giant> giants, const frost_cluster_tolerances& tol,
                                     float tsamp) const {
        std::vector<frost_giant> out(giants.size());
        size_t n = 0;
        check(frost_subband_dedup(giants.data(), giants.size(), &tol, tsamp, m_mode, out.data(), &n, m_device));
        out.resize(n);
        return out;
    }

private:
    int m_mode, m_device;
};

inline bool are_coincident(const frost_giant& a, const frost_giant& b, uint64_t time_tol, uint64_t filter_tol,
                           uint64_t dm_tol) {
    const frost_cluster_tolerances t{time_tol, filter_tol, dm_tol, 0.0, 0.0, 0.0};
    return frost_are_coincident(&a, &b, &t, 0) != 0;
}
inline bool are_coincident(const frost_giant& a, const frost_giant& b, const frost_cluster_tolerances& tol) {
    return frost_are_coincident(&a, &b, &tol, 1) != 0;
}
inline double subband_time_shift_samples(float dm, float f_wide, float f_narrow, float tsamp) {
    return frost_subband_time_shift_samples(dm, f_wide, f_narrow, tsamp);
}
inline double subband_dm_step(float f_low, float f_high, float tsamp) {
    return frost_subband_dm_step(f_low, f_high, tsamp);
}

} // namespace frost::b200
