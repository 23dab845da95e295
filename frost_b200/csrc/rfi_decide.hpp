// Per-gulp RFI decisions on the device: the channel mask (moment outliers,
// IQRM, growth), dead channels, the time flags (broad-band zero-DM
// detector, dropouts, whole-band Kadane spans), the zero-DM fit and the
// Kadane-along-time segment acceptance. They read the reductions the
// measurement kernels leave on the device and write what the apply and
// normalise kernels read, so a gulp needs no device-to-host copy between
// its phases. Decisions reproduce frost's CPU cleaner bit for bit: every
// threshold-deciding quantity is computed with the same operations in the
// same order (the file is compiled --fmad=false), and order statistics come
// from sorts and exact selections, not approximations.
//
// Reference behaviour: lib/cpu/rfi_cpu_measure.cpp:56-84,140-300 (channel
// mask), lib/cpu/rfi_masks_cpu.cpp:29-122 (IQRM), lib/cpu/rfi_cpu.cpp:
// 347-468 (flags), lib/cpu/device_rfi_flags_cpu.cpp:17-75 and
// lib/cpu/stats_cpu.cpp:77-93,153-278 (broad-band detector).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.hpp"
#include "rfi_kernels.hpp"

namespace fb::rfi {

/** Report counters the decision kernels accumulate on the device, in the
 * slots after the apply counters. */
enum {
    kRepMoments = kCountSlots,
    kRepIqrm,
    kRepGrown,
    kRepMasked,
    kRepDead,
    kRepBroad,
    kRepDropout,
    kRepKadane,
    kRepFlagged,
    kRepSlots
};

/** IQRM lags 1, then max(lag + lag/2, lag + 1) while <= radius, stopping
 * after the first lag >= n - 1 (larger lags repeat its edge-clamped
 * comparisons). */
std::vector<uint64_t> iqrm_lags(uint64_t n, uint64_t radius);

/** Settings of the channel-mask decision. */
struct ChannelMaskParams {
    uint64_t n           = 0;
    uint64_t nwin        = 0;
    int moments          = 0;  // moment outlier strategy
    int need_clip        = 0;  // write the clipped-moment tables
    int stat_on[5]       = {}; // mean, std, skewness, kurtosis, lag-1 autocorrelation
    double k             = 0;  // IQR multiple
    double kurt_max      = 0;  // |excess kurtosis| cap; <= 0 is off
    int iqrm             = 0;
    float iqrm_threshold = 0;
    uint64_t grow        = 0;
};

/** Device scratch of the channel-mask decision, sized by size_for(). */
struct ChannelScratch {
    double* stat     = nullptr; // [5][n]
    uint8_t* good    = nullptr; // [n]
    uint8_t* ignore  = nullptr; // [n]
    float* iqrm_x    = nullptr; // [n]
    uint8_t* flags   = nullptr; // [5][n]
    int32_t* votes   = nullptr; // [n][2 * nlags]
    uint32_t* cast   = nullptr; // [n]
    uint8_t* dynamic = nullptr; // [n]
    uint32_t* prefix = nullptr; // [n + 1]
    uint64_t* lags   = nullptr; // [nlags]
    double* sort_buf = nullptr; // [(5 + 2 * nlags) * pow2(n)] when the sorts do not fit shared memory
    uint64_t nlags   = 0;

    static size_t size_for(uint64_t n, uint64_t nlags);
    void carve(void* base, uint64_t n, uint64_t nlags);
};

/** The channel mask of one gulp: per-channel statistics from the window
 * moment sums, the IQR outlier tests, IQRM on the scale-weighted std, the
 * growth, then mask = static & ~dynamic and its exclusive prefix count.
 * Also writes the clipped-moment tables when p.need_clip. */
void decide_channel_mask(const ChannelMaskParams& p, const ChannelScratch& w, const MomentSums* mom,
                         const float* scale, const uint32_t* unmeasured, const uint8_t* static_mask,
                         float* clip_mean, float* clip_inv, uint8_t* mask, uint64_t* good_prefix,
                         unsigned long long* counters, cudaStream_t s);

/** IQRM alone on a device statistic (the standalone iqrm_mask): 1 = flagged,
 * ignored channels included. */
void iqrm_device(uint64_t n, const float* x, const uint8_t* ignore, float threshold,
                 const ChannelScratch& w, uint8_t* out, cudaStream_t s);

/** iqrm_mask (include/frost/prepare/rfi.hpp:56-59) of a host statistic,
 * run on the current device: uploads x (and `ignore`, which may be null),
 * runs iqrm_device and copies the n flags back to `out`. Validates as
 * frost does (radius > 0, threshold positive and finite). */
void iqrm_mask_host(const float* x, uint64_t n, uint64_t radius, float threshold, const uint8_t* ignore,
                    uint8_t* out);

/** Settings of the time-flag decisions. */
struct FlagParams {
    uint64_t nsamps        = 0;
    uint64_t nchans        = 0;
    uint64_t nwin          = 0;
    int broad              = 0;
    uint64_t smooth_radius = 0;
    float broad_threshold  = 0;
    uint64_t boxcar_max    = 0;
    int dropout            = 0;
    float dropout_fraction = 0;
    int kspec              = 0;
    int zdot               = 0;
    int kchan              = 0;
    double kchan_min_len   = 0;
    double kchan_threshold = 0;
};

/** Device scratch of the time-flag decisions, sized by size_for(). */
struct FlagScratch {
    float* series    = nullptr; // [T]
    float* buf_a     = nullptr; // [2T + 4] baseline resampling
    float* buf_b     = nullptr; // [2T + 4]
    float* scanned   = nullptr; // [T + 1]
    uint32_t* words  = nullptr; // [nwidths][W] detection bits per boxcar width
    uint32_t* wpre   = nullptr; // [nwidths][W + 1]
    uint8_t* bb      = nullptr; // [T]
    float* scalars   = nullptr; // [4]: MAD rms, dropout cut
    uint32_t nwidths = 0;

    static size_t size_for(uint64_t nsamps, uint64_t boxcar_max);
    void carve(void* base, uint64_t nsamps, uint64_t boxcar_max);
};

/** Dead channels, the time flags (broad-band, dropouts, whole-band Kadane
 * spans, in that order; each count is of the samples it newly flags), the
 * zero-DM fit, the accepted Kadane-along-time segments and the list of
 * flagged samples (increasing; its length in counters[kRepFlagged]). Every
 * step is skipped when no channel is good (good_prefix[n] == 0), as frost
 * skips them. */
void decide_flags(const FlagParams& p, const FlagScratch& w, const uint64_t* good_prefix,
                  const uint32_t* unmeasured, const float* lo, const float* hi, const float* s_det,
                  const float* row_std, const uint8_t* kspec_whole, const ZdotSums* zsum,
                  const Run* kpos_best, const Run* kneg_best, uint8_t* mask, uint8_t* time_flags,
                  float* zdot_a, float* zdot_b, Segment* kchan_pos, Segment* kchan_neg,
                  uint8_t* kchan_any, uint64_t* flagged, unsigned long long* counters, cudaStream_t s);

/** Kernels launched by this file's launchers in this process. */
uint64_t decide_launch_counter();

} // namespace fb::rfi
