// extern "C" entry points of include/frost_b200.h. Each wraps the C++
// implementation, converts exceptions to frost_status codes and records the
// message for frost_last_error(); nothing throws across this boundary.

#include <algorithm>
#include <cstdio>
#include <memory>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "common.hpp"
#include "dedisp.hpp"
#include "batch.hpp"
#include "rfi_decide.hpp"
#include "sigproc.hpp"
#include "cand_writer.hpp"
#include "memory_plan.hpp"
#include "postprocess.hpp"
#include "prefetch.hpp"
#include "pp_math.cuh"
#include "rfi_cleaner.hpp"
#include "search_engine.hpp"
#include "server.hpp"

namespace fb {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

bool is_finite(float x) {
    uint32_t b;
    std::memcpy(&b, &x, sizeof(b));
    return is_finite_bits32(b);
}

bool is_finite(double x) {
    uint64_t b;
    std::memcpy(&b, &x, sizeof(b));
    return is_finite_bits64(b);
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return FROST_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code();
    } catch (const std::bad_alloc& e) {
        set_last_error(std::string("host allocation failed: ") + e.what());
        return FROST_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return FROST_ERR_INTERNAL;
    } catch (...) {
        set_last_error("unknown error");
        return FROST_ERR_INTERNAL;
    }
}

} // namespace fb

struct frost_rfi {
    fb::rfi::Cleaner impl;
    template <class... A> explicit frost_rfi(A&&... a) : impl(std::forward<A>(a)...) {}
};

struct frost_search {
    fb::fdmt::Engine impl;
    template <class... A> explicit frost_search(A&&... a) : impl(std::forward<A>(a)...) {}
};

struct frost_server {
    fb::serve::Server impl;
    template <class... A> explicit frost_server(A&&... a) : impl(std::forward<A>(a)...) {}
};

struct frost_batch {
    fb::serve::Batch impl;
    template <class... A> explicit frost_batch(A&&... a) : impl(std::forward<A>(a)...) {}
};

struct frost_cand_writer {
    fb::output::CandWriter impl;
    template <class... A> explicit frost_cand_writer(A&&... a) : impl(std::forward<A>(a)...) {}
};

struct frost_prefetch {
    std::FILE* file = nullptr;        // the built-in file source, when used
    const uint8_t* memory = nullptr;  // the built-in memory source, when used
    size_t total_rows = 0, next_row = 0;
    size_t row_bytes = 0;
    std::unique_ptr<fb::staging::Prefetch> impl;
    ~frost_prefetch() {
        impl.reset(); // joins the reader before the file closes
        if (file != nullptr)
            std::fclose(file);
    }
};

struct frost_postprocess {
    fb::pp::PostprocessPlan impl;
    template <class... A> explicit frost_postprocess(A&&... a) : impl(std::forward<A>(a)...) {}
};

namespace {
/** Device copy of host giants for a standalone plan call (one stream). */
struct PlanCall {
    fb::DeviceGuard guard;
    cudaStream_t s = nullptr;
    fb::pp::Workspace ws;
    fb::DeviceBuffer rows, out, aux;
    explicit PlanCall(int device) : guard(device) {
        FB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    }
    ~PlanCall() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    const frost_giant* upload(const frost_giant* g, size_t n) {
        rows.reserve(std::max<size_t>(n, 1) * sizeof(frost_giant));
        if (n)
            FB_CUDA(cudaMemcpyAsync(rows.get(), g, n * sizeof(frost_giant), cudaMemcpyHostToDevice, s));
        return rows.as<frost_giant>();
    }
};

void check_rows(size_t n, const char* what) {
    if (n >= (size_t{1} << 31))
        fb::invalid(std::string(what) + ": at most 2^31 - 1 rows per call");
}

int copy_candidates(const std::vector<frost_candidate>& c, frost_candidate* out, size_t capacity,
                    size_t* count) {
    if (count != nullptr)
        *count = c.size();
    const size_t n = std::min(capacity, c.size());
    if (out != nullptr && n)
        std::memcpy(out, c.data(), n * sizeof(frost_candidate));
    if (c.size() > capacity) {
        fb::set_last_error("candidate buffer holds " + std::to_string(capacity) + " of " +
                           std::to_string(c.size()));
        return FROST_ERR_OVERFLOW;
    }
    return FROST_OK;
}
} // namespace

using fb::guarded;
using fb::invalid;

extern "C" {

const char* frost_last_error(void) { return fb::g_last_error.c_str(); }

const char* frost_version(void) { return "frost_b200 0.1.0 (sm_100a)"; }

void frost_rfi_config_default(frost_rfi_config* cfg) {
    if (cfg != nullptr)
        fb::rfi::config_default(cfg);
}

int frost_rfi_config_validate(const frost_rfi_config* cfg) {
    return guarded([&] {
        if (cfg == nullptr)
            invalid("null config");
        fb::rfi::Config::from(*cfg).validate();
    });
}

int frost_rfi_create(const frost_rfi_config* cfg, const frost_block_layout* layout,
                     float baseline_length, int device, frost_rfi** out) {
    return guarded([&] {
        if (cfg == nullptr || layout == nullptr || out == nullptr)
            invalid("frost_rfi_create: null argument");
        *out = nullptr;
        *out = new frost_rfi(*cfg, *layout, baseline_length, device);
    });
}

int frost_rfi_destroy(frost_rfi* rfi) {
    return guarded([&] { delete rfi; });
}

int frost_rfi_execute_normalized(frost_rfi* rfi, const uint8_t* block, size_t block_bytes,
                                 size_t nsamps, int block_on_device, void* stream,
                                 const float** out_device) {
    return guarded([&] {
        if (rfi == nullptr)
            invalid("frost_rfi_execute_normalized: null handle");
        // frost's device RFI path takes the pipeline's stream and refuses the
        // null stream (lib/cuda/device_rfi_detail.cuh:77-83): a device block
        // is read only after the work queued on the caller's stream.
        if (block_on_device != 0 && stream == nullptr)
            invalid("RFICleaner: a device block requires the pipeline stream, not the null stream");
        const float* out = rfi->impl.execute_normalized(block, block_bytes, nsamps,
                                                        block_on_device != 0,
                                                        static_cast<cudaStream_t>(stream));
        if (out_device != nullptr)
            *out_device = out;
    });
}

int frost_rfi_download_normalized(frost_rfi* rfi, float* host, size_t count) {
    return guarded([&] {
        if (rfi == nullptr || (host == nullptr && count != 0))
            invalid("frost_rfi_download_normalized: null argument");
        const size_t have = rfi->impl.capacity() * rfi->impl.nchans();
        if (count < have)
            invalid("frost_rfi_download_normalized: buffer holds " + std::to_string(count) +
                    " floats, need " + std::to_string(have));
        fb::DeviceGuard g(rfi->impl.device());
        if (have)
            FB_CUDA(cudaMemcpy(host, rfi->impl.output(), have * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

int frost_rfi_channel_mask(const frost_rfi* rfi, uint8_t* out, size_t nchans) {
    return guarded([&] {
        if (rfi == nullptr || out == nullptr)
            invalid("frost_rfi_channel_mask: null argument");
        const auto& m = rfi->impl.channel_mask();
        if (nchans < m.size())
            invalid("frost_rfi_channel_mask: buffer too small");
        std::memcpy(out, m.data(), m.size());
    });
}

int frost_rfi_get_report(const frost_rfi* rfi, frost_rfi_report* out) {
    return guarded([&] {
        if (rfi == nullptr || out == nullptr)
            invalid("frost_rfi_get_report: null argument");
        *out = rfi->impl.report();
    });
}

int frost_rfi_time_flags(const frost_rfi* rfi, uint8_t* out, size_t nsamps) {
    return guarded([&] {
        if (rfi == nullptr || out == nullptr)
            invalid("frost_rfi_time_flags: null argument");
        const auto& f = rfi->impl.time_flags();
        if (nsamps < f.size())
            invalid("frost_rfi_time_flags: buffer too small");
        std::memcpy(out, f.data(), f.size());
    });
}

int frost_rfi_memory_usage(const frost_rfi* rfi, size_t* bytes) {
    return guarded([&] {
        if (rfi == nullptr || bytes == nullptr)
            invalid("frost_rfi_memory_usage: null argument");
        *bytes = rfi->impl.memory_usage();
    });
}

int frost_rfi_normalize_static(const frost_block_layout* layout, float baseline_length,
                               const uint8_t* block, size_t block_bytes, size_t nsamps, float* out,
                               size_t out_count, void* stream) {
    return guarded([&] {
        if (layout == nullptr)
            invalid("frost_rfi_normalize_static: null layout");
        if (stream == nullptr)
            invalid("normalize_static: requires the caller's stream, not the null stream");
        fb::rfi::normalize_static(*layout, baseline_length, block, block_bytes, nsamps, out,
                                  out_count, static_cast<cudaStream_t>(stream));
    });
}

int frost_rfi_launch_count(const frost_rfi* rfi, uint64_t* launches) {
    return guarded([&] {
        if (rfi == nullptr || launches == nullptr)
            invalid("frost_rfi_launch_count: null argument");
        *launches = rfi->impl.launches();
    });
}

int frost_rfi_get_stream(const frost_rfi* rfi, void** stream) {
    return guarded([&] {
        if (rfi == nullptr || stream == nullptr)
            invalid("frost_rfi_get_stream: null argument");
        *stream = static_cast<void*>(rfi->impl.stream());
    });
}

int frost_iqrm_mask(const float* x, size_t n, uint64_t radius, float threshold,
                    const uint8_t* ignore, uint8_t* out) {
    return guarded([&] {
        if ((x == nullptr || out == nullptr) && n != 0)
            invalid("frost_iqrm_mask: null argument");
        fb::rfi::iqrm_mask_host(x, n, radius, threshold, ignore, out);
    });
}

int frost_apply_manual_killmask(uint8_t* killmask, size_t nchans, const frost_channel_range* zaps,
                                size_t nzaps) {
    return guarded([&] {
        if ((killmask == nullptr && nchans) || (zaps == nullptr && nzaps))
            invalid("frost_apply_manual_killmask: null argument");
        fb::rfi::apply_manual_killmask({killmask, nchans}, {zaps, nzaps});
    });
}

int frost_read_kill_file(const char* path, size_t nchans, frost_channel_range* out,
                         size_t capacity, size_t* count) {
    return guarded([&] {
        if (path == nullptr || count == nullptr)
            invalid("frost_read_kill_file: null argument");
        const auto r = fb::rfi::read_kill_file(path, nchans);
        *count       = r.size();
        if (out != nullptr) {
            if (capacity < r.size())
                invalid("frost_read_kill_file: output holds too few ranges");
            std::memcpy(out, r.data(), r.size() * sizeof(frost_channel_range));
        }
    });
}

int frost_generate_dm_list(const frost_dedisp_plan_config* cfg, float* out, size_t capacity,
                           size_t* count) {
    return guarded([&] {
        if (cfg == nullptr || count == nullptr)
            invalid("frost_generate_dm_list: null argument");
        const auto dms = fb::dedisp::generate_dm_list(*cfg);
        *count         = dms.size();
        if (out != nullptr) {
            if (capacity < dms.size())
                invalid("frost_generate_dm_list: output holds too few trials");
            std::memcpy(out, dms.data(), dms.size() * sizeof(float));
        }
    });
}

int frost_fdmt_band_edges(const frost_dedisp_plan_config* cfg, float* f_min, float* f_max) {
    return guarded([&] {
        if (cfg == nullptr || f_min == nullptr || f_max == nullptr)
            invalid("frost_fdmt_band_edges: null argument");
        fb::dedisp::band_edges(*cfg, *f_min, *f_max);
    });
}

} // extern "C"

extern "C" {

int frost_search_create(const frost_dedisp_plan_config* plan, const frost_boxcar_config* cfg,
                        const uint8_t* kill_mask, size_t memory_budget, int device,
                        frost_search** out) {
    return guarded([&] {
        if (plan == nullptr || cfg == nullptr || out == nullptr)
            invalid("frost_search_create: null argument");
        *out = nullptr;
        *out = new frost_search(*plan, *cfg, kill_mask, memory_budget, device);
    });
}

int frost_search_destroy(frost_search* s) {
    return guarded([&] { delete s; });
}

int frost_search_execute(frost_search* s, const float* waterfall, size_t nsamps, int on_device,
                         const uint8_t* mask, void* stream) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_execute: null handle");
        if (on_device != 0 && stream == nullptr)
            invalid("search: a device waterfall requires the pipeline stream, not the null stream");
        s->impl.execute(waterfall, nsamps, on_device != 0, mask, static_cast<cudaStream_t>(stream));
    });
}

int frost_search_drain(frost_search* s) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_drain: null handle");
        s->impl.drain();
    });
}

int frost_search_result_count(const frost_search* s, size_t* count, uint64_t* dropped_global,
                              uint64_t* dropped_per_dm) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_result_count: null handle");
        if (count != nullptr)
            *count = s->impl.results().size();
        if (dropped_global != nullptr)
            *dropped_global = s->impl.dropped_global();
        if (dropped_per_dm != nullptr)
            *dropped_per_dm = s->impl.dropped_per_dm();
    });
}

int frost_search_results(const frost_search* s, frost_candidate* out, size_t capacity,
                         size_t* count) {
    return guarded([&] {
        if (s == nullptr || count == nullptr)
            invalid("frost_search_results: null argument");
        const auto& r = s->impl.results();
        *count        = r.size();
        if (out != nullptr) {
            if (capacity < r.size())
                invalid("frost_search_results: output holds too few candidates");
            std::memcpy(out, r.data(), r.size() * sizeof(frost_candidate));
        }
    });
}

int frost_search_frontier(const frost_search* s, uint64_t* sample) {
    return guarded([&] {
        if (s == nullptr || sample == nullptr)
            invalid("frost_search_frontier: null argument");
        *sample = const_cast<frost_search*>(s)->impl.frontier();
    });
}

int frost_search_get_info(const frost_search* s, frost_search_info* out) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_search_get_info: null argument");
        *out = s->impl.info();
    });
}

int frost_search_plane_info(const frost_search* s, size_t plane, frost_search_plane* out,
                            float* dm_grid, uint32_t* warmup) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_search_plane_info: null argument");
        const auto& planes = s->impl.plan().planes();
        if (plane >= planes.size())
            invalid("frost_search_plane_info: plane index out of range");
        const auto& p     = planes[plane];
        out->subband_level = static_cast<uint32_t>(p.subband_level);
        out->subband_idx   = static_cast<uint32_t>(p.subband_idx);
        out->level         = static_cast<uint32_t>(p.height);
        out->chan_begin    = static_cast<uint32_t>(p.chan_begin);
        out->chan_end      = static_cast<uint32_t>(p.chan_end);
        out->staggered     = static_cast<uint32_t>(p.staggered);
        out->ndm           = p.delay.size();
        out->f_low         = p.f_lo;
        out->f_high        = p.f_hi;
        for (size_t i = 0; i < p.delay.size(); ++i) {
            if (dm_grid != nullptr)
                dm_grid[i] = p.dm[i];
            if (warmup != nullptr)
                warmup[i] = static_cast<uint32_t>(p.delay[i]);
        }
    });
}

int frost_search_widths(const frost_search* s, uint32_t* out, size_t capacity, size_t* count) {
    return guarded([&] {
        if (s == nullptr || count == nullptr)
            invalid("frost_search_widths: null argument");
        const auto& w = s->impl.plan().widths();
        *count        = w.size();
        if (out != nullptr) {
            if (capacity < w.size())
                invalid("frost_search_widths: output too small");
            for (size_t i = 0; i < w.size(); ++i)
                out[i] = static_cast<uint32_t>(w[i]);
        }
    });
}

int frost_search_variance_grid(const frost_search* s, size_t plane, uint32_t width,
                               const uint8_t* mask, double* out, size_t capacity) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_search_variance_grid: null argument");
        if (width == 0)
            invalid("frost_search_variance_grid: width must be > 0");
        const auto v = s->impl.variance_grid(plane, width, mask);
        if (capacity < v.size())
            invalid("frost_search_variance_grid: output too small");
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    });
}

int frost_search_capture_planes(frost_search* s, int enable) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_capture_planes: null handle");
        s->impl.capture(enable != 0);
    });
}

int frost_server_create(int device, size_t memory_budget, uint32_t slots, frost_server** out) {
    return guarded([&] {
        if (out == nullptr)
            invalid("frost_server_create: null argument");
        *out = nullptr;
        *out = new frost_server(device, memory_budget, slots);
    });
}

int frost_server_destroy(frost_server* s) {
    return guarded([&] { delete s; });
}

int frost_server_add_beam(frost_server* s, const frost_rfi_config* rfi,
                          const frost_block_layout* layout, float baseline_length,
                          const frost_dedisp_plan_config* plan, const frost_boxcar_config* search,
                          uint32_t* beam) {
    return guarded([&] {
        if (s == nullptr || rfi == nullptr || layout == nullptr || plan == nullptr ||
            search == nullptr || beam == nullptr)
            invalid("frost_server_add_beam: null argument");
        fb::serve::BeamSpec spec;
        spec.rfi = *rfi;
        if (rfi->n_zap_chans)
            spec.zap_chans.assign(rfi->zap_chans, rfi->zap_chans + rfi->n_zap_chans);
        if (rfi->n_zap_freqs)
            spec.zap_freqs.assign(rfi->zap_freqs, rfi->zap_freqs + rfi->n_zap_freqs);
        spec.layout          = *layout;
        spec.baseline_length = baseline_length;
        spec.plan            = *plan;
        spec.search          = *search;
        *beam                = s->impl.add_beam(spec);
    });
}

int frost_batch_create(int device, size_t memory_budget, frost_batch** out) {
    return guarded([&] {
        if (out == nullptr)
            invalid("frost_batch_create: null output");
        *out = nullptr;
        *out = new frost_batch(device, memory_budget);
    });
}

int frost_batch_destroy(frost_batch* b) {
    return guarded([&] { delete b; });
}

int frost_batch_add_beam(frost_batch* b, const frost_rfi_config* rfi, const frost_block_layout* layout,
                         float baseline_length, const frost_dedisp_plan_config* plan,
                         const frost_boxcar_config* search, uint32_t* beam) {
    return guarded([&] {
        if (b == nullptr || rfi == nullptr || layout == nullptr || plan == nullptr || search == nullptr ||
            beam == nullptr)
            invalid("frost_batch_add_beam: null argument");
        fb::serve::BeamSpec spec;
        spec.rfi = *rfi;
        if (rfi->n_zap_chans)
            spec.zap_chans.assign(rfi->zap_chans, rfi->zap_chans + rfi->n_zap_chans);
        if (rfi->n_zap_freqs)
            spec.zap_freqs.assign(rfi->zap_freqs, rfi->zap_freqs + rfi->n_zap_freqs);
        spec.layout          = *layout;
        spec.baseline_length = baseline_length;
        spec.plan            = *plan;
        spec.search          = *search;
        *beam                = b->impl.add_beam(spec);
    });
}

int frost_batch_execute(frost_batch* b, const uint8_t* const* blocks, const size_t* nread, int on_device) {
    return guarded([&] {
        if (b == nullptr)
            invalid("frost_batch_execute: null handle");
        b->impl.execute(blocks, nread, on_device != 0);
    });
}

int frost_batch_results(const frost_batch* b, uint32_t beam, frost_candidate* out, size_t capacity, size_t* count) {
    int rc      = FROST_OK;
    const int g = guarded([&] {
        if (b == nullptr)
            invalid("frost_batch_results: null handle");
        rc = copy_candidates(b->impl.results(beam), out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_batch_drain(frost_batch* b, uint32_t beam, frost_candidate* out, size_t capacity, size_t* count) {
    int rc      = FROST_OK;
    const int g = guarded([&] {
        if (b == nullptr)
            invalid("frost_batch_drain: null handle");
        rc = copy_candidates(b->impl.drain(beam), out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_batch_use_graph(frost_batch* b, int enable) {
    return guarded([&] {
        if (b == nullptr)
            invalid("frost_batch_use_graph: null handle");
        b->impl.use_graph(enable != 0);
    });
}

int frost_batch_get_stats(const frost_batch* b, frost_batch_stats* out) {
    return guarded([&] {
        if (b == nullptr || out == nullptr)
            invalid("frost_batch_get_stats: null argument");
        *out = b->impl.stats();
    });
}

int frost_server_remove_beam(frost_server* s, uint32_t beam) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_server_remove_beam: null handle");
        s->impl.remove_beam(beam);
    });
}

int frost_server_submit(frost_server* s, uint32_t beam, const uint8_t* block, size_t block_bytes,
                        size_t nread, int on_device, uint64_t* ticket) {
    return guarded([&] {
        if (s == nullptr || ticket == nullptr)
            invalid("frost_server_submit: null argument");
        *ticket = s->impl.submit(beam, block, block_bytes, nread, on_device != 0);
    });
}

int frost_server_wait(frost_server* s, uint64_t ticket, frost_candidate* out, size_t capacity,
                      size_t* count, double* latency_s) {
    int rc = FROST_OK;
    const int g = guarded([&] {
        if (s == nullptr)
            invalid("frost_server_wait: null handle");
        const auto c = s->impl.wait(ticket, latency_s);
        rc           = copy_candidates(c, out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_server_drain(frost_server* s, uint32_t beam, frost_candidate* out, size_t capacity,
                       size_t* count) {
    int rc = FROST_OK;
    const int g = guarded([&] {
        if (s == nullptr)
            invalid("frost_server_drain: null handle");
        rc = copy_candidates(s->impl.drain(beam), out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_server_set_residency(frost_server* s, uint32_t beam, int ctas_per_sm) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_server_set_residency: null handle");
        s->impl.set_residency(beam, ctas_per_sm);
    });
}

int frost_server_set_staging(frost_server* s, uint32_t beam, uint32_t slots) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_server_set_staging: null handle");
        s->impl.set_staging(beam, slots);
    });
}

int frost_server_set_postprocess(frost_server* s, uint32_t beam, const frost_postprocess_config* cfg) {
    return guarded([&] {
        if (s == nullptr || cfg == nullptr)
            invalid("frost_server_set_postprocess: null argument");
        s->impl.set_postprocess(beam, *cfg);
    });
}

namespace {
int copy_giants(const std::vector<frost_giant>& g, frost_giant* out, size_t capacity, size_t* count) {
    if (count != nullptr)
        *count = g.size();
    const size_t n = std::min(capacity, g.size());
    if (out != nullptr && n)
        std::memcpy(out, g.data(), n * sizeof(frost_giant));
    if (g.size() > capacity) {
        fb::set_last_error("giant buffer holds " + std::to_string(capacity) + " of " + std::to_string(g.size()));
        return FROST_ERR_OVERFLOW;
    }
    return FROST_OK;
}
} // namespace

int frost_server_wait_giants(frost_server* s, uint64_t ticket, frost_giant* out, size_t capacity, size_t* count,
                             double* latency_s) {
    int rc      = FROST_OK;
    const int g = guarded([&] {
        if (s == nullptr)
            invalid("frost_server_wait_giants: null handle");
        rc = copy_giants(s->impl.wait_giants(ticket, latency_s), out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_server_drain_giants(frost_server* s, uint32_t beam, frost_giant* out, size_t capacity, size_t* count) {
    int rc      = FROST_OK;
    const int g = guarded([&] {
        if (s == nullptr)
            invalid("frost_server_drain_giants: null handle");
        rc = copy_giants(s->impl.drain_giants(beam), out, capacity, count);
    });
    return g != FROST_OK ? g : rc;
}

int frost_server_reset_stats(frost_server* s) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_server_reset_stats: null handle");
        s->impl.reset_stats();
    });
}

int frost_server_get_stats(frost_server* s, frost_server_stats* out) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_server_get_stats: null argument");
        *out = s->impl.stats();
    });
}

int frost_search_autotune(frost_search* s, int* fused, int* tiles_per_cta, double* ms, int* cached) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_autotune: null handle");
        const auto t = s->impl.autotune();
        if (fused != nullptr)
            *fused = t.fuse ? 1 : 0;
        if (tiles_per_cta != nullptr)
            *tiles_per_cta = t.tiles_per_cta;
        if (ms != nullptr)
            *ms = t.ms;
        if (cached != nullptr)
            *cached = t.cached ? 1 : 0;
    });
}

int frost_search_set_launch_shape(frost_search* s, int fused, int tiles_per_cta, int stages, int search_chunk) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_set_launch_shape: null handle");
        s->impl.set_launch_shape(fused != 0, tiles_per_cta, stages, search_chunk);
    });
}

int frost_search_get_launch_shape(const frost_search* s, int* fused, int* tiles_per_cta, int* stages,
                                  int* search_chunk) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_get_launch_shape: null handle");
        const auto t = s->impl.launch_shape();
        if (fused != nullptr)
            *fused = t.fuse ? 1 : 0;
        if (tiles_per_cta != nullptr)
            *tiles_per_cta = t.tiles_per_cta;
        if (stages != nullptr)
            *stages = t.stages;
        if (search_chunk != nullptr)
            *search_chunk = t.search_chunk;
    });
}

int frost_search_set_residency(frost_search* s, int ctas_per_sm) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_set_residency: null handle");
        s->impl.set_residency(ctas_per_sm);
    });
}

int frost_search_get_residency(const frost_search* s, int* ctas_per_sm) {
    return guarded([&] {
        if (s == nullptr || ctas_per_sm == nullptr)
            invalid("frost_search_get_residency: null argument");
        *ctas_per_sm = s->impl.residency();
    });
}

int frost_search_set_fused_search(frost_search* s, int on) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_set_fused_search: null handle");
        s->impl.set_fused_search(on);
    });
}

int frost_search_get_fused_search(const frost_search* s, int* on) {
    return guarded([&] {
        if (s == nullptr || on == nullptr)
            invalid("frost_search_get_fused_search: null argument");
        *on = s->impl.fused_search_mode();
    });
}

int frost_search_set_wait_limit(frost_search* s, int64_t tries) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_set_wait_limit: null handle");
        s->impl.set_wait_limit(tries);
    });
}

int frost_search_restart(frost_search* s) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_restart: null handle");
        s->impl.restart();
    });
}

int frost_search_get_stream(const frost_search* s, void** stream) {
    return guarded([&] {
        if (s == nullptr || stream == nullptr)
            invalid("frost_search_get_stream: null argument");
        *stream = static_cast<void*>(s->impl.stream());
    });
}

int frost_search_use_graphs(frost_search* s, int enable) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_use_graphs: null handle");
        s->impl.use_graphs(enable != 0);
    });
}

int frost_search_enable_timing(frost_search* s, int enable) {
    return guarded([&] {
        if (s == nullptr)
            invalid("frost_search_enable_timing: null handle");
        s->impl.enable_timing(enable != 0);
    });
}

int frost_search_get_timing(const frost_search* s, frost_search_timing* out) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_search_get_timing: null argument");
        *out = s->impl.timing();
    });
}

int frost_search_plane_data(const frost_search* s, size_t plane, float* out, size_t capacity) {
    return guarded([&] {
        if (s == nullptr || out == nullptr)
            invalid("frost_search_plane_data: null argument");
        s->impl.plane_data(plane, out, capacity);
    });
}

// ---- candidate post-processing ------------------------------------------------

int frost_postprocess_create(const frost_postprocess_config* cfg, const frost_postprocess_layout* layout,
                             int device, frost_postprocess** out) {
    return guarded([&] {
        if (cfg == nullptr || layout == nullptr || out == nullptr)
            invalid("frost_postprocess_create: null argument");
        *out = nullptr;
        *out = new frost_postprocess(*cfg, *layout, device);
    });
}

int frost_postprocess_destroy(frost_postprocess* p) {
    return guarded([&] { delete p; });
}

int frost_postprocess_execute(frost_postprocess* p, const frost_candidate* cands, size_t n, int on_device,
                              uint64_t samples_read, uint64_t duration_samples, int final_call,
                              uint64_t candidate_frontier, frost_postprocess_result* out) {
    return guarded([&] {
        if (p == nullptr || out == nullptr || (cands == nullptr && n > 0))
            invalid("frost_postprocess_execute: null argument");
        fb::DeviceGuard g(p->impl.device());
        *out = p->impl.execute(cands, n, on_device != 0, samples_read, duration_samples, final_call != 0,
                               candidate_frontier);
    });
}

int frost_postprocess_execute_search(frost_postprocess* p, frost_search* s, uint64_t samples_read,
                                     uint64_t duration_samples, int final_call, uint64_t candidate_frontier,
                                     frost_postprocess_result* out) {
    return guarded([&] {
        if (p == nullptr || s == nullptr || out == nullptr)
            invalid("frost_postprocess_execute_search: null argument");
        if (p->impl.device() != s->impl.device())
            invalid("frost_postprocess_execute_search: the handles are on different devices");
        fb::DeviceGuard g(p->impl.device());
        *out = p->impl.execute(s->impl.device_results(), s->impl.results().size(), true, samples_read,
                               duration_samples, final_call != 0, candidate_frontier);
    });
}

int frost_postprocess_results(const frost_postprocess* p, frost_giant* out, size_t capacity, size_t* count) {
    return guarded([&] {
        if (p == nullptr || count == nullptr)
            invalid("frost_postprocess_results: null argument");
        const auto& r = p->impl.results();
        *count        = r.size();
        if (out != nullptr) {
            if (capacity < r.size())
                invalid("frost_postprocess_results: output holds too few giants");
            std::memcpy(out, r.data(), r.size() * sizeof(frost_giant));
        }
    });
}

int frost_postprocess_memory_usage(const frost_postprocess* p, uint64_t* bytes) {
    return guarded([&] {
        if (p == nullptr || bytes == nullptr)
            invalid("frost_postprocess_memory_usage: null argument");
        *bytes = p->impl.memory_usage();
    });
}

int frost_postprocess_estimate_memory(const frost_postprocess_config* cfg, uint64_t* bytes) {
    return guarded([&] {
        if (cfg == nullptr || bytes == nullptr)
            invalid("frost_postprocess_estimate_memory: null argument");
        *bytes = fb::pp::PostprocessPlan::estimate_memory(*cfg);
    });
}

int frost_cluster_labels(const frost_giant* giants, size_t n, const frost_cluster_tolerances* tol, int mode,
                         uint64_t* labels, int device) {
    return guarded([&] {
        if (tol == nullptr || ((giants == nullptr || labels == nullptr) && n > 0))
            invalid("frost_cluster_labels: null argument");
        if (mode != FROST_CLUSTER_CHAIN && mode != FROST_CLUSTER_SEEDED)
            invalid("frost_cluster_labels: unknown mode");
        check_rows(n, "frost_cluster_labels");
        if (n == 0)
            return;
        PlanCall c(device);
        const frost_giant* rows = c.upload(giants, n);
        c.out.reserve(n * sizeof(uint32_t));
        fb::pp::cluster_labels(c.ws, rows, n, *tol, mode, c.out.as<uint32_t>(), c.s);
        std::vector<uint32_t> l(n);
        FB_CUDA(cudaMemcpyAsync(l.data(), c.out.get(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.s));
        FB_CUDA(cudaStreamSynchronize(c.s));
        for (size_t i = 0; i < n; ++i)
            labels[i] = l[i];
    });
}

int frost_merge_candidates(const frost_giant* giants, const uint64_t* labels, size_t n, frost_giant* out,
                           size_t* count, int device) {
    return guarded([&] {
        if (count == nullptr || ((giants == nullptr || labels == nullptr || out == nullptr) && n > 0))
            invalid("frost_merge_candidates: null argument");
        check_rows(n, "frost_merge_candidates");
        *count = 0;
        if (n == 0)
            return;
        PlanCall c(device);
        const frost_giant* rows = c.upload(giants, n);
        c.aux.reserve(n * sizeof(uint64_t));
        FB_CUDA(cudaMemcpyAsync(c.aux.get(), labels, n * sizeof(uint64_t), cudaMemcpyHostToDevice, c.s));
        c.out.reserve(n * sizeof(frost_giant));
        const size_t m = fb::pp::merge_candidates(c.ws, rows, c.aux.as<uint64_t>(), n,
                                                  c.out.as<frost_giant>(), c.s);
        FB_CUDA(cudaMemcpyAsync(out, c.out.get(), m * sizeof(frost_giant), cudaMemcpyDeviceToHost, c.s));
        FB_CUDA(cudaStreamSynchronize(c.s));
        *count = m;
    });
}

int frost_subband_dedup(const frost_giant* giants, size_t n, const frost_cluster_tolerances* tol, float tsamp,
                        int mode, frost_giant* out, size_t* count, int device) {
    return guarded([&] {
        if (tol == nullptr || count == nullptr || ((giants == nullptr || out == nullptr) && n > 0))
            invalid("frost_subband_dedup: null argument");
        if (mode != FROST_DEDUP_TRANSITIVE && mode != FROST_DEDUP_SEEDED)
            invalid("frost_subband_dedup: unknown mode");
        check_rows(n, "frost_subband_dedup");
        *count = 0;
        if (n == 0)
            return;
        if (!fb::pp::posfin_f(tsamp))
            invalid("sub-band dedup requires tsamp > 0");
        PlanCall c(device);
        const frost_giant* rows = c.upload(giants, n);
        c.out.reserve(n * sizeof(frost_giant));
        const size_t m = fb::pp::subband_dedup(c.ws, rows, n, *tol, tsamp, mode, c.out.as<frost_giant>(), c.s);
        FB_CUDA(cudaMemcpyAsync(out, c.out.get(), m * sizeof(frost_giant), cudaMemcpyDeviceToHost, c.s));
        FB_CUDA(cudaStreamSynchronize(c.s));
        *count = m;
    });
}

int frost_are_coincident(const frost_giant* a, const frost_giant* b, const frost_cluster_tolerances* tol,
                         int physical) {
    if (a == nullptr || b == nullptr || tol == nullptr) {
        fb::set_last_error("frost_are_coincident: null argument");
        return 0;
    }
    const fb::pp::Pt pa = fb::pp::pt_of(*a), pb = fb::pp::pt_of(*b);
    if (physical != 0)
        return fb::pp::coincident(pa, pb, *tol) ? 1 : 0;
    return fb::pp::coincident_basic(pa, pb, tol->time_tol, tol->filter_tol, tol->dm_tol) ? 1 : 0;
}

double frost_subband_time_shift_samples(float dm, float f_wide, float f_narrow, float tsamp) {
    return fb::pp::time_shift(dm, f_wide, f_narrow, tsamp);
}

double frost_subband_dm_step(float f_low, float f_high, float tsamp) {
    return fb::pp::dm_step(f_low, f_high, tsamp);
}

// ---- input staging ----------------------------------------------------------------

namespace {
long read_file_rows(void* ctx, uint8_t* buf, size_t max_rows) {
    auto* p        = static_cast<frost_prefetch*>(ctx);
    const size_t n = std::fread(buf, p->row_bytes, max_rows, p->file);
    if (n < max_rows && std::ferror(p->file))
        return -1;
    return static_cast<long>(n);
}
long read_memory_rows(void* ctx, uint8_t* buf, size_t max_rows) {
    auto* p        = static_cast<frost_prefetch*>(ctx);
    const size_t n = std::min(max_rows, p->total_rows - p->next_row);
    if (n > 0)
        std::memcpy(buf, p->memory + p->next_row * p->row_bytes, n * p->row_bytes);
    p->next_row += n;
    return static_cast<long>(n);
}
} // namespace

int frost_prefetch_create_memory(const uint8_t* rows, size_t total_rows, size_t block_rows, size_t row_bytes,
                                 int depth, int device, frost_prefetch** out) {
    return guarded([&] {
        if ((rows == nullptr && total_rows > 0) || out == nullptr)
            invalid("frost_prefetch_create_memory: null argument");
        *out            = nullptr;
        auto p          = std::make_unique<frost_prefetch>();
        p->memory       = rows;
        p->total_rows   = total_rows;
        p->row_bytes    = row_bytes;
        p->impl = std::make_unique<fb::staging::Prefetch>(block_rows, row_bytes, depth, device, read_memory_rows,
                                                          p.get());
        *out = p.release();
    });
}

int frost_prefetch_create(size_t block_rows, size_t row_bytes, int depth, int device, frost_read_fn read,
                          void* ctx, frost_prefetch** out) {
    return guarded([&] {
        if (read == nullptr || out == nullptr)
            invalid("frost_prefetch_create: null argument");
        *out      = nullptr;
        auto p    = std::make_unique<frost_prefetch>();
        p->impl   = std::make_unique<fb::staging::Prefetch>(block_rows, row_bytes, depth, device, read, ctx);
        *out      = p.release();
    });
}

int frost_prefetch_create_file(const char* path, uint64_t header_bytes, size_t block_rows, size_t row_bytes,
                               int depth, int device, frost_prefetch** out) {
    return guarded([&] {
        if (path == nullptr || out == nullptr)
            invalid("frost_prefetch_create_file: null argument");
        *out = nullptr;
        if (row_bytes == 0)
            invalid("frost_prefetch_create_file: row bytes must be positive");
        auto p  = std::make_unique<frost_prefetch>();
        p->file = std::fopen(path, "rb");
        if (p->file == nullptr)
            throw fb::Error(FROST_ERR_IO, std::string("frost_prefetch_create_file: cannot open ") + path);
        if (std::fseek(p->file, static_cast<long>(header_bytes), SEEK_SET) != 0)
            throw fb::Error(FROST_ERR_IO, "frost_prefetch_create_file: cannot seek past the header");
        p->row_bytes = row_bytes;
        p->impl = std::make_unique<fb::staging::Prefetch>(block_rows, row_bytes, depth, device, read_file_rows,
                                                          p.get());
        *out = p.release();
    });
}

int frost_sigproc_read_header(const char* path, frost_sigproc_header* out) {
    return guarded([&] {
        if (path == nullptr || out == nullptr)
            invalid("frost_sigproc_read_header: null argument");
        *out = fb::io::read_sigproc_header(path);
    });
}

int frost_sigproc_layout(const frost_sigproc_header* header, uint64_t block_rows, frost_block_layout* out) {
    return guarded([&] {
        if (header == nullptr || out == nullptr)
            invalid("frost_sigproc_layout: null argument");
        *out = fb::io::sigproc_layout(*header, block_rows);
    });
}

int frost_prefetch_create_sigproc(const char* path, size_t block_rows, int depth, int device,
                                  frost_sigproc_header* header, frost_prefetch** out) {
    return guarded([&] {
        if (path == nullptr || out == nullptr)
            invalid("frost_prefetch_create_sigproc: null argument");
        *out                         = nullptr;
        const frost_sigproc_header h = fb::io::read_sigproc_header(path);
        (void)fb::io::sigproc_layout(h, block_rows); // a supported sample type
        const int rc = frost_prefetch_create_file(path, h.header_bytes, block_rows, h.row_bytes, depth, device, out);
        if (rc != FROST_OK)
            throw fb::Error(rc, frost_last_error());
        if (header != nullptr)
            *header = h;
    });
}

int frost_prefetch_next(frost_prefetch* p, void* stream, const uint8_t** block_device, size_t* nread) {
    return guarded([&] {
        if (p == nullptr || block_device == nullptr || nread == nullptr)
            invalid("frost_prefetch_next: null argument");
        fb::SizeType n = 0;
        *block_device  = p->impl->next(&n, static_cast<cudaStream_t>(stream));
        *nread         = n;
    });
}

int frost_prefetch_get_stats(const frost_prefetch* p, frost_prefetch_stats* out) {
    return guarded([&] {
        if (p == nullptr || out == nullptr)
            invalid("frost_prefetch_get_stats: null argument");
        *out = p->impl->stats();
    });
}

int frost_prefetch_destroy(frost_prefetch* p) {
    return guarded([&] { delete p; });
}

// ---- candidate file -------------------------------------------------------------

int frost_cand_writer_open(const char* path, double dt, int append, frost_cand_writer** out) {
    return guarded([&] {
        if (path == nullptr || out == nullptr)
            invalid("frost_cand_writer_open: null argument");
        *out = nullptr;
        *out = new frost_cand_writer(std::string(path), dt, append != 0);
    });
}

int frost_cand_writer_write(frost_cand_writer* w, const frost_giant* giants, size_t n, uint64_t first_samp_idx) {
    return guarded([&] {
        if (w == nullptr || (giants == nullptr && n > 0))
            invalid("frost_cand_writer_write: null argument");
        w->impl.write(giants, n, first_samp_idx);
    });
}

int frost_cand_writer_close(frost_cand_writer* w) {
    return guarded([&] { delete w; });
}

int frost_cand_filename(int64_t utc, uint64_t beam, char* out, size_t capacity) {
    return guarded([&] {
        if (out == nullptr)
            invalid("frost_cand_filename: null argument");
        const std::string s = fb::output::cand_filename(static_cast<std::time_t>(utc), beam);
        if (s.size() + 1 > capacity)
            invalid("frost_cand_filename: output holds too few characters");
        std::memcpy(out, s.c_str(), s.size() + 1);
    });
}

int frost_estimate_memory(const frost_rfi_config* rfi, const frost_block_layout* layout, float baseline_length,
                          const frost_dedisp_plan_config* plan, const frost_boxcar_config* search,
                          const frost_postprocess_config* post, frost_memory_estimate* out) {
    return guarded([&] {
        if (rfi == nullptr || layout == nullptr || plan == nullptr || search == nullptr || out == nullptr)
            invalid("frost_estimate_memory: null argument");
        *out = fb::memplan::estimate(*rfi, *layout, baseline_length, *plan, *search, post);
    });
}

int frost_check_memory(const frost_rfi_config* rfi, frost_block_layout* layout, float baseline_length,
                       frost_dedisp_plan_config* plan, const frost_boxcar_config* search,
                       const frost_postprocess_config* post, int gulp_is_default, uint64_t available_bytes,
                       uint64_t memory_limit_bytes, int device, frost_memory_check* out) {
    return guarded([&] {
        if (rfi == nullptr || layout == nullptr || plan == nullptr || search == nullptr || out == nullptr)
            invalid("frost_check_memory: null argument");
        *out = fb::memplan::check(*rfi, *layout, baseline_length, *plan, *search, post, gulp_is_default != 0,
                                  available_bytes, memory_limit_bytes, device);
    });
}

} // extern "C"
