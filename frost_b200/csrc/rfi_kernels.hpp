// Host-callable launchers of the RFI excision kernels (rfi_kernels.cu).
// All pointers are device pointers unless named h_*; every launcher is
// asynchronous on `stream`.
#pragma once

#include <cstdint>

#include <cuda_runtime_api.h>

#include "rfi_types.hpp"

namespace fb::rfi {

/** Block geometry of one execute call. */
struct Dims {
    int dtype;          // enum frost_dtype of the packed input
    uint64_t nchans;
    uint64_t row_bytes;
    uint64_t nsamps;    // valid rows measured and cleaned
    uint64_t window;    // window length in rows
    uint64_t nwin;      // windows (the last absorbs the remainder)
    uint64_t nchunks;   // row-scan chunks
    uint64_t chunk;     // rows per chunk
};

/** Settings of the apply (fill/transform) pass. */
struct ApplyParams {
    uint64_t seed;
    uint64_t block_index;
    uint64_t chan_fill_radius;
    uint64_t time_fill_radius;
    float clip;
    float eq_loc;
    float eq_scale;
    int32_t narrow_active;
    int32_t kspec;
    int32_t kchan;
    int32_t neighbour;  // fill == neighbour
    int32_t noise;      // fill == noise
    int32_t zero_dm;    // enum frost_zero_dm
    int32_t equalize;
    int32_t transform;
};

/** Kadane-across-frequency acceptance (lib/cpu/rfi_cpu_measure.cpp:313-349). */
struct KspecParams {
    int32_t enabled;
    double min_bw_chans;
    double whole_chans;
    double threshold;
};

/** Kernels launched by this file's launchers in this process. */
uint64_t launch_counter();

/** Counters the apply passes accumulate (device, 4 x uint64). */
enum { kCountNarrow = 0, kCountKspec = 1, kCountKchan = 2, kCountFallback = 3, kCountSlots = 4 };

// Writes the lowest index of a non-finite float32 word into *first_bad
// (initialised by the caller to nwords).
void launch_check_finite(const uint8_t* raw, uint64_t nwords, unsigned long long* first_bad,
                         cudaStream_t s);

// Gathers the evenly spaced bandpass rows of every window into
// samples[nwin][kMaxBandpassRows][nchans] as float.
void launch_sample_rows(const Dims& d, const uint8_t* raw, float* samples, cudaStream_t s);

// Remedian level + MAD and the clipped refinement per (window, channel).
// Writes loc/scale/inv [nwin][nchans]; unmeasured[c] counts windows whose
// refinement failed (must be zeroed by the caller).
void launch_bandpass(const Dims& d, const float* samples, float* loc, float* scale, float* inv,
                     uint32_t* unmeasured, cudaStream_t s);

// Raw and clipped moments per (window, channel) of z = (x - loc) * inv.
void launch_moments(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                    const uint8_t* static_mask, float clip, MomentSums* out, cudaStream_t s);

// Per-row detection series and the Kadane-across-frequency spans;
// row_clip[t] = 1 when a measured cell of row t is past the clip.
void launch_scan_rows(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                      const uint8_t* mask, float clip, const KspecParams& kp,
                      const uint64_t* good_prefix, float* s_det, double* s_keep_d, float* s_keep_f,
                      float* row_std, Span32* kspec_pos, Span32* kspec_neg, uint8_t* kspec_whole,
                      uint8_t* row_clip, cudaStream_t s);

// Per (chunk, channel): min/max of unmeasured cells, zdot sums and the
// Kadane-along-time states; then combined over chunks per channel in chunk
// order into lo/hi, zdot and the best runs.
void launch_scan_cols(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                      const uint8_t* mask, float clip, const double* s_keep_d, int zdot, int kchan,
                      const float* clip_mean, const float* clip_inv_std, float* chunk_min,
                      float* chunk_max, ZdotSums* chunk_zdot, KadaneState* chunk_kpos,
                      KadaneState* chunk_kneg, float* lo, float* hi, ZdotSums* zdot_sum,
                      Run* kpos_best, Run* kneg_best, cudaStream_t s);

// row_kchan[t] = 1 for the rows some channel's Kadane-along-time segment
// covers, else 0.
void launch_kchan_rows(const Dims& d, const Segment* kchan_pos, const Segment* kchan_neg,
                       const uint8_t* kchan_any, uint8_t* row_kchan, cudaStream_t s);

// Cleans unflagged rows into work[nsamps][nchans] (float). kchan_any[c]
// marks the channels with a Kadane-along-time segment (only those read
// their segments); a row with no clipped cell (row_clip), no segment
// (row_kchan) and no span across frequency writes its clean values
// without classifying its cells, the others are listed in slow_rows
// (*nslow of them; nsamps entries of room) and cleaned cell by cell.
void launch_apply_unflagged(const Dims& d, const ApplyParams& p, const uint8_t* raw,
                            const float* loc, const float* scale, const float* inv,
                            const uint8_t* mask, const uint8_t* time_flags, const Span32* kspec_pos,
                            const Span32* kspec_neg, const Segment* kchan_pos,
                            const Segment* kchan_neg, const uint8_t* kchan_any,
                            const float* s_keep_f, const float* zdot_a,
                            const float* zdot_b, const uint8_t* row_clip, const uint8_t* row_kchan,
                            uint32_t* slow_rows, unsigned int* nslow, float* work,
                            unsigned long long* counters, cudaStream_t s);

// Refills the flagged rows flagged[0 .. *nflagged) of work from unflagged
// rows (the count is read on the device).
void launch_apply_flagged(const Dims& d, const ApplyParams& p, const uint64_t* flagged,
                          const unsigned long long* nflagged, const float* loc, const float* scale,
                          const float* inv, const uint8_t* mask, const uint8_t* time_flags,
                          float* work, unsigned long long* counters, cudaStream_t s);

// Unpacks raw rows into work (short blocks).
void launch_unpack(const Dims& d, const uint8_t* raw, float* work, cudaStream_t s);

// Per (window, channel) Welford mean/rms of work rows in that window.
/** Per (window, channel) Welford mean / std of the cleaned float rows.
 * `recip[2n]`, `recip[2n + 1]` = RN(1/n), RN((1 - n RN(1/n)) / n) for n up
 * to the longest window let the update divide with one multiply and one
 * fused multiply-add instead of a full division (same bits); null uses the
 * plain division. */
void launch_welford(const Dims& d, const float* work, const double* recip, float* loc, float* scale,
                    cudaStream_t s);

// out[dst][t] = (work[t][c] - loc) / scale for t < nsamps and unmasked c;
// zero elsewhere; dst = flip ? nchans-1-c : c; out has `capacity` columns.
void launch_normalize(const Dims& d, const float* work, const float* loc, const float* scale,
                      const uint8_t* mask, int flip, uint64_t capacity, float* out, cudaStream_t s);

// Short-tail normalisation with the retained calibration
// (lib/cpu/rfi_cpu.cpp:262-315).
void launch_normalize_short(const Dims& d, const ApplyParams& p, const float* work,
                            const float* tail_loc, const float* tail_scale,
                            const float* tail_out_loc, const float* tail_out_scale,
                            const uint8_t* mask, const float* zdot_a, const float* zdot_b,
                            int flip, uint64_t capacity, float* out, cudaStream_t s);

} // namespace fb::rfi
