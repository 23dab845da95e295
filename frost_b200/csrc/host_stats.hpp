// Host-side statistics on per-gulp series (length T or C, never T x C): the
// broad-band zero-DM detector, IQRM and IQR outlier flags. They run on the
// small series the GPU passes reduce the block to, in the same split frost's
// own device cleaner uses (lib/cuda/device_rfi_cuda.cu:232-262), and are
// compiled with strict IEEE flags so their decisions match the reference
// cleaner's bit for bit.
#pragma once

#include <cstdint>
#include <span>
#include <vector>

#include "common.hpp"

namespace fb::stats {

/** numpy-style linear-interpolation quantile of ascending `sorted`
 * (lib/cpu/rfi_kernels.hpp:136-142). */
double quantile_sorted(std::span<const double> sorted, double q);

/** Gaussian-equivalent scale of zero-centred data: median(|x|) / 0.67449
 * over every sample (lib/cpu/stats_cpu.cpp:77-93). */
float mad_scale(std::span<const float> data);

/** Subtracts a median-of-5 scrunched, linearly re-stretched baseline with
 * knots every `smooth_radius` samples (lib/cpu/stats_cpu.cpp:210-278). */
void baseline_subtract(std::vector<float>& data, SizeType smooth_radius);

/** Broad-band time flags: baseline removal, MAD normalisation and
 * |x| > threshold at boxcar widths 1, 2, 4, ..., boxcar_max, each detection
 * widened by its boxcar (lib/cpu/device_rfi_flags_cpu.cpp:17-75). Sets new
 * flags in `flags` and returns how many it set. */
SizeType broadband_time_flags(std::vector<float> series, SizeType smooth_radius, float threshold,
                              SizeType boxcar_max, std::span<uint8_t> flags);

/** IQRM (Morello et al. 2022) on a per-channel statistic
 * (lib/cpu/rfi_masks_cpu.cpp:29-122). */
std::vector<uint8_t> iqrm_mask(std::span<const float> x, SizeType radius, float threshold,
                               std::span<const uint8_t> ignore);

/** Flags values more than k IQRs outside [Q1, Q3] among `good` entries
 * (lib/cpu/rfi_cpu_measure.cpp:56-84). */
void flag_iqr_outliers(std::span<const double> stat, std::span<const uint8_t> good, double k,
                       std::span<uint8_t> flags);

} // namespace fb::stats
