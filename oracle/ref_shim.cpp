// TEST INFRASTRUCTURE ONLY. extern "C" wrapper around the reference's own
// CPU RFI cleaner, statistics, IQRM, kill-file reader and DM grid, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/. Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as
// the checker; nothing in frost_b200/ links or calls it.
//
// Wrapped reference entry points:
//   RFICleaner (include/frost/prepare/rfi.hpp:243-297, lib/cpu/rfi_cpu.cpp)
//   iqrm_mask (lib/cpu/rfi_masks_cpu.cpp:29-122)
//   broadband_time_flags (lib/cpu/device_rfi_flags_cpu.cpp:17-75)
//   spectra::measure_bandpass (lib/cpu/spectra_cpu.cpp:73-130)
//   KadaneState (lib/cpu/rfi_kernels.hpp:65-133)
//   generate_dm_list / make_dmt_fdmt_plan (lib/dedisp/dedisp.cpp:16-89)
//   read_kill_file (lib/prepare/kill_file.cpp:15-65)

#include <cstdio>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

#include <frost/dedisp/dedisp.hpp>
#include <frost/prepare/rfi.hpp>
#include <frost/prepare/spectra.hpp>

#include "lib/cpu/rfi_kernels.hpp"
#include "lib/prepare/device_rfi.hpp"

#include "frost_b200.h"

using namespace frost;
using namespace frost::prepare::rfi;

namespace {

thread_local std::string g_err;

int fail(const std::exception& e, int code) {
    g_err = e.what();
    return code;
}

RfiConfig to_cfg(const frost_rfi_config& c) {
    RfiConfig r;
    for (uint64_t i = 0; i < c.n_zap_chans; ++i)
        r.zap_chans.push_back({c.zap_chans[i].start, c.zap_chans[i].end});
    for (uint64_t i = 0; i < c.n_zap_freqs; ++i)
        r.zap_freqs.push_back({c.zap_freqs[i].lo, c.zap_freqs[i].hi});
    r.narrow.enabled           = c.narrow_enabled != 0;
    r.narrow.threshold         = c.narrow_threshold;
    r.broad.enabled            = c.broad_enabled != 0;
    r.broad.threshold          = c.broad_threshold;
    r.broad.boxcar_max         = c.broad_boxcar_max;
    r.dropout.enabled          = c.dropout_enabled != 0;
    r.dropout.min_std_fraction = c.dropout_min_std_fraction;
    r.moments.enabled          = c.moments_enabled != 0;
    r.moments.threshold        = c.moments_threshold;
    r.moments.mean             = c.moments_mean != 0;
    r.moments.std              = c.moments_std != 0;
    r.moments.skewness         = c.moments_skewness != 0;
    r.moments.kurtosis         = c.moments_kurtosis != 0;
    r.moments.autocorr         = c.moments_autocorr != 0;
    r.moments.kurtosis_max     = c.moments_kurtosis_max;
    r.iqrm.enabled             = c.iqrm_enabled != 0;
    r.iqrm.threshold           = c.iqrm_threshold;
    r.iqrm.radius              = c.iqrm_radius;
    r.mask_grow                = c.mask_grow;
    r.kadane_channel.enabled   = c.kadane_channel_enabled != 0;
    r.kadane_channel.threshold = c.kadane_channel_threshold;
    r.kadane_channel.min_duration         = c.kadane_channel_min_duration;
    r.kadane_spectrum.enabled             = c.kadane_spectrum_enabled != 0;
    r.kadane_spectrum.threshold           = c.kadane_spectrum_threshold;
    r.kadane_spectrum.min_bandwidth       = c.kadane_spectrum_min_bandwidth;
    r.kadane_spectrum.whole_band_fraction = c.kadane_spectrum_whole_band_fraction;
    r.zero_dm  = static_cast<ZeroDMMode>(c.zero_dm);
    r.equalize = c.equalize != 0;
    r.fill     = static_cast<FillMode>(c.fill);
    r.seed     = c.seed;
    return r;
}

void to_report(const RfiReport& r, frost_rfi_report* o) {
    o->calibration_reused    = r.calibration_reused ? 1 : 0;
    o->nsamps                = r.nsamps;
    o->chans_zapped          = r.chans_zapped;
    o->chans_dead            = r.chans_dead;
    o->chans_moments         = r.chans_moments;
    o->chans_iqrm            = r.chans_iqrm;
    o->chans_grown           = r.chans_grown;
    o->chans_masked          = r.chans_masked;
    o->samps_broad           = r.samps_broad;
    o->samps_dropout         = r.samps_dropout;
    o->samps_kadane          = r.samps_kadane;
    o->samps_flagged         = r.samps_flagged;
    o->cells_narrow          = r.cells_narrow;
    o->cells_kadane_spectrum = r.cells_kadane_spectrum;
    o->cells_kadane_channel  = r.cells_kadane_channel;
    o->fill_fallbacks        = r.fill_fallbacks;
    o->t_bandpass            = r.t_bandpass;
    o->t_moments             = r.t_moments;
    o->t_scan                = r.t_scan;
    o->t_flags               = r.t_flags;
    o->t_apply               = r.t_apply;
}

dedisp::DedispPlanConfig to_dd(const frost_dedisp_plan_config& c) {
    dedisp::DedispPlanConfig d;
    d.nchans         = c.nchans;
    d.dt             = c.dt;
    d.f0             = c.f0;
    d.df             = c.df;
    d.dm_min         = c.dm_min;
    d.dm_max         = c.dm_max;
    d.dm_pulse_width = c.dm_pulse_width;
    d.dm_tol         = c.dm_tol;
    d.block_nsamps   = c.block_nsamps;
    d.subband_depth  = c.subband_depth;
    return d;
}

} // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_rfi_create(const frost_rfi_config* cfg,
                     const frost_block_layout* layout,
                     float baseline_length) {
    try {
        BlockLayout l;
        l.nchans     = layout->nchans;
        l.max_nsamps = layout->max_nsamps;
        l.dtype      = static_cast<DataType>(layout->dtype);
        l.tsamp      = layout->tsamp;
        l.f0         = layout->f0;
        l.df         = layout->df;
        return new RFICleaner(to_cfg(*cfg), l, baseline_length);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ref_rfi_destroy(void* h) { delete static_cast<RFICleaner*>(h); }

// execute_normalized; copies the [nchans][capacity] result to `out`.
int ref_rfi_execute_normalized(void* h,
                               uint8_t* block,
                               size_t bytes,
                               size_t nsamps,
                               float* out,
                               size_t out_count) {
    try {
        auto* r        = static_cast<RFICleaner*>(h);
        const auto res = r->execute_normalized({block, bytes}, nsamps);
        if (out != nullptr) {
            if (out_count < res.size())
                throw std::invalid_argument("ref shim: output too small");
            std::memcpy(out, res.data(), res.size() * sizeof(float));
        }
        return static_cast<int>(res.size() > 0);
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    } catch (const std::exception& e) {
        return fail(e, FROST_ERR_INTERNAL);
    }
}

// Byte-cleaning execute (in place).
int ref_rfi_execute(void* h, uint8_t* block, size_t bytes) {
    try {
        static_cast<RFICleaner*>(h)->execute({block, bytes});
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    } catch (const std::exception& e) {
        return fail(e, FROST_ERR_INTERNAL);
    }
}

int ref_rfi_channel_mask(void* h, uint8_t* out, size_t n) {
    const auto m = static_cast<RFICleaner*>(h)->channel_mask();
    if (n < m.size())
        return FROST_ERR_INVALID_ARGUMENT;
    std::memcpy(out, m.data(), m.size());
    return 0;
}

int ref_rfi_report(void* h, frost_rfi_report* out) {
    to_report(static_cast<RFICleaner*>(h)->report(), out);
    return 0;
}

int ref_rfi_config_validate(const frost_rfi_config* cfg) {
    try {
        to_cfg(*cfg).validate();
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    }
}

int ref_iqrm_mask(const float* x,
                  size_t n,
                  size_t radius,
                  float threshold,
                  const uint8_t* ignore,
                  uint8_t* out) {
    try {
        std::span<const uint8_t> ig;
        if (ignore != nullptr)
            ig = {ignore, n};
        const auto m = iqrm_mask({x, n}, radius, threshold, ig);
        std::memcpy(out, m.data(), n);
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    }
}

long ref_broadband_time_flags(const float* series,
                              size_t n,
                              size_t smooth_radius,
                              float threshold,
                              size_t boxcar_max,
                              uint8_t* flags) {
    try {
        std::vector<float> s(series, series + n);
        return static_cast<long>(pipeline::device::broadband_time_flags(
            std::move(s), smooth_radius, threshold, boxcar_max, {flags, n}));
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    }
}

int ref_measure_bandpass(const float* in,
                         size_t nsamps,
                         size_t nchans,
                         float* bandpass,
                         float* rms) {
    try {
        frost::prepare::spectra::measure_bandpass({in, nsamps * nchans}, {bandpass, nchans},
                                  {rms, nchans}, nsamps, nchans);
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    }
}

// Kadane over positions idx[] (increasing) with values u[]; chunk_len > 0
// splits the sequence into chunks combined with KadaneState::combine.
int ref_kadane(const int64_t* idx,
               const double* u,
               size_t n,
               size_t chunk_len,
               double* best_sum,
               int64_t* best_start,
               int64_t* best_end,
               double* total) {
    kernels::KadaneState acc;
    const size_t step = chunk_len == 0 ? (n == 0 ? 1 : n) : chunk_len;
    for (size_t i0 = 0; i0 < n; i0 += step) {
        kernels::KadaneState part;
        for (size_t i = i0; i < n && i < i0 + step; ++i)
            part.append(idx[i], u[i]);
        acc = kernels::KadaneState::combine(acc, part);
    }
    *best_sum   = acc.best.sum;
    *best_start = acc.best.start;
    *best_end   = acc.best.end;
    *total      = acc.total;
    return 0;
}

int ref_generate_dm_list(const frost_dedisp_plan_config* cfg,
                         float* out,
                         size_t capacity,
                         size_t* count) {
    try {
        const auto dms = dedisp::generate_dm_list(to_dd(*cfg));
        *count         = dms.size();
        if (out != nullptr) {
            if (capacity < dms.size())
                return FROST_ERR_INVALID_ARGUMENT;
            std::memcpy(out, dms.data(), dms.size() * sizeof(float));
        }
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    } catch (const std::exception& e) {
        return fail(e, FROST_ERR_INTERNAL);
    }
}

int ref_fdmt_band_edges(const frost_dedisp_plan_config* cfg,
                        float* f_min,
                        float* f_max) {
    try {
        const auto plan = dedisp::make_dmt_fdmt_plan(to_dd(*cfg));
        *f_min          = plan.get_f_min();
        *f_max          = plan.get_f_max();
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    } catch (const std::exception& e) {
        return fail(e, FROST_ERR_INTERNAL);
    }
}

int ref_read_kill_file(const char* path,
                       size_t nchans,
                       frost_channel_range* out,
                       size_t capacity,
                       size_t* count) {
    try {
        const auto r = read_kill_file(path, nchans);
        *count       = r.size();
        for (size_t i = 0; i < r.size() && i < capacity; ++i)
            out[i] = {r[i].start, r[i].end};
        return 0;
    } catch (const std::invalid_argument& e) {
        return fail(e, FROST_ERR_INVALID_ARGUMENT);
    } catch (const std::exception& e) {
        return fail(e, FROST_ERR_IO);
    }
}

} // extern "C"
