// GPU RFICleaner orchestration. Per gulp:
//   decode checks -> bandpass (sampled remedian + clipped refinement) ->
//   moments -> channel mask (moments IQR outliers, IQRM, growth) ->
//   row scan + column scan -> flags -> apply (fills, transforms) ->
//   optional Welford re-measure -> normalise + transpose to [channel][time].
// Every T x C pass is a kernel (rfi_kernels.cu) and every per-gulp decision
// on the O(T) / O(C) series those passes reduce the block to is a kernel
// too (rfi_decide.cu): the whole gulp is queued on one stream and the host
// reads back only the mask and the report counters at the end. Semantics
// follow RFICleaner::Impl (lib/cpu/rfi_cpu.cpp, lib/cpu/rfi_cpu_measure.cpp).

#include "rfi_cleaner.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <string_view>

namespace fb::rfi {

namespace {

template <class T> void h2d(DeviceBuffer& dst, const T* src, SizeType count, cudaStream_t s) {
    dst.reserve(std::max<SizeType>(count * sizeof(T), 1));
    if (count)
        FB_CUDA(cudaMemcpyAsync(dst.get(), src, count * sizeof(T), cudaMemcpyHostToDevice, s));
}

SizeType count_zeros(const std::vector<uint8_t>& v) {
    return static_cast<SizeType>(std::count(v.begin(), v.end(), uint8_t{0}));
}

} // namespace

// ---- configuration ---------------------------------------------------------

void config_default(frost_rfi_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->narrow_enabled                      = 1;
    c->narrow_threshold                    = 5.0F;
    c->broad_enabled                       = 1;
    c->broad_threshold                     = 5.0F;
    c->broad_boxcar_max                    = 1;
    c->dropout_enabled                     = 0;
    c->dropout_min_std_fraction            = 0.1F;
    c->moments_enabled                     = 0;
    c->moments_threshold                   = 4.0F;
    c->moments_mean                        = 1;
    c->moments_std                         = 1;
    c->moments_skewness                    = 1;
    c->moments_kurtosis                    = 1;
    c->moments_autocorr                    = 1;
    c->moments_kurtosis_max                = 0.0F;
    c->iqrm_enabled                        = 0;
    c->iqrm_threshold                      = 3.0F;
    c->iqrm_radius                         = 0;
    c->mask_grow                           = 0;
    c->kadane_channel_enabled              = 0;
    c->kadane_channel_threshold            = 7.0F;
    c->kadane_channel_min_duration         = 0.05F;
    c->kadane_spectrum_enabled             = 0;
    c->kadane_spectrum_threshold           = 7.0F;
    c->kadane_spectrum_min_bandwidth       = 10.0F;
    c->kadane_spectrum_whole_band_fraction = 0.8F;
    c->zero_dm                             = FROST_ZERO_DM_OFF;
    c->equalize                            = 0;
    c->fill                                = FROST_FILL_NEIGHBOUR;
    c->seed                                = 0x5EED;
}

Config Config::from(const frost_rfi_config& in) {
    Config out;
    out.c = in;
    if (in.n_zap_chans && in.zap_chans == nullptr)
        invalid("rfi.zap_chans is null");
    if (in.n_zap_freqs && in.zap_freqs == nullptr)
        invalid("rfi.zap_freqs is null");
    out.zap_chans.assign(in.zap_chans, in.zap_chans + in.n_zap_chans);
    out.zap_freqs.assign(in.zap_freqs, in.zap_freqs + in.n_zap_freqs);
    out.c.zap_chans = nullptr;
    out.c.zap_freqs = nullptr;
    return out;
}

// RfiConfig::validate (lib/prepare/rfi_config.cpp:14-77).
void Config::validate() const {
    auto positive = [](float v, const char* name) {
        if (!is_positive_finite(v))
            invalid(std::string("rfi.") + name + " must be finite and > 0");
    };
    auto nonnegative = [](float v, const char* name) {
        if (!is_finite(v) || v < 0.0F)
            invalid(std::string("rfi.") + name + " must be finite and >= 0");
    };
    auto fraction = [](float v, const char* name) {
        if (!is_finite(v) || v < 0.0F || v > 1.0F)
            invalid(std::string("rfi.") + name + " must be finite and in [0, 1]");
    };
    positive(c.narrow_threshold, "narrow.threshold");
    positive(c.broad_threshold, "broad.threshold");
    positive(c.moments_threshold, "moments.threshold");
    positive(c.iqrm_threshold, "iqrm.threshold");
    positive(c.kadane_channel_threshold, "kadane_channel.threshold");
    positive(c.kadane_spectrum_threshold, "kadane_spectrum.threshold");
    nonnegative(c.moments_kurtosis_max, "moments.kurtosis_max");
    nonnegative(c.kadane_channel_min_duration, "kadane_channel.min_duration");
    nonnegative(c.kadane_spectrum_min_bandwidth, "kadane_spectrum.min_bandwidth");
    fraction(c.dropout_min_std_fraction, "dropout.min_std_fraction");
    fraction(c.kadane_spectrum_whole_band_fraction, "kadane_spectrum.whole_band_fraction");
    if (c.broad_boxcar_max == 0)
        invalid("rfi.broad.boxcar_max must be >= 1");
    for (const auto& r : zap_chans)
        if (r.start > r.end)
            invalid("rfi.zap_chans ranges need start <= end");
    for (const auto& r : zap_freqs)
        if (!is_finite(r.lo) || !is_finite(r.hi) || r.lo > r.hi)
            invalid("rfi.zap_freqs ranges must be finite with lo <= hi");
    if (c.fill < FROST_FILL_NEIGHBOUR || c.fill > FROST_FILL_NOISE)
        invalid("Invalid rfi.fill");
    if (c.zero_dm < FROST_ZERO_DM_OFF || c.zero_dm > FROST_ZERO_DM_ZDOT)
        invalid("Invalid rfi.zero_dm");
}

// validate_layout (lib/prepare/rfi_config.cpp:79-110).
void validate_layout(const frost_block_layout& l, float baseline_length) {
    if (l.nchans == 0 || l.max_nsamps == 0)
        invalid("RFI: nchans and max_nsamps must be > 0");
    if (l.dtype < FROST_UINT1 || l.dtype > FROST_FLOAT32)
        invalid("RFI: unsupported dtype");
    const auto width    = static_cast<SizeType>(bits_of(l.dtype));
    constexpr auto kMax = std::numeric_limits<SizeType>::max();
    if (l.nchans > kMax / width || l.nchans > (kMax / sizeof(float)) / l.max_nsamps)
        invalid("RFI: packed or normalized block geometry overflows");
    if ((l.nchans * width) % 8 != 0)
        invalid("RFI: each time sample must be a whole number of bytes");
    if (!is_positive_finite(l.tsamp) || !is_positive_finite(baseline_length))
        invalid("RFI: tsamp and baseline_length must be finite and > 0");
    if (!is_finite(l.f0) || !is_finite(l.df))
        invalid("RFI: f0 and df must be finite");
    if (l.tsamp <= static_cast<double>(baseline_length) / static_cast<double>(kMax))
        invalid("RFI: baseline sample count is not representable");
}

// apply_manual_killmask (lib/cpu/rfi_masks_cpu.cpp:16-27).
void apply_manual_killmask(std::span<uint8_t> mask, std::span<const frost_channel_range> zaps) {
    if (mask.empty())
        return;
    for (const auto& r : zaps) {
        const auto end = std::min<uint64_t>(r.end, mask.size() - 1);
        for (uint64_t c = r.start; c <= end; ++c)
            mask[c] = 0;
    }
}

// read_kill_file (lib/prepare/kill_file.cpp:15-65): one 0/1 per line,
// '#' comments and blank lines ignored, exactly nchans entries.
std::vector<frost_channel_range> read_kill_file(const std::string& path, SizeType nchans) {
    std::ifstream in(path);
    if (!in)
        throw Error(FROST_ERR_IO, "cannot read kill file " + path);
    std::vector<frost_channel_range> killed;
    SizeType channel = 0;
    std::string line;
    for (SizeType number = 1; std::getline(in, line); ++number) {
        std::string_view text(line);
        if (const auto hash = text.find('#'); hash != std::string_view::npos)
            text = text.substr(0, hash);
        constexpr std::string_view kSpace = " \t\r\f\v";
        const auto first                  = text.find_first_not_of(kSpace);
        if (first == std::string_view::npos)
            continue;
        text = text.substr(first, text.find_last_not_of(kSpace) - first + 1);
        if (text != "0" && text != "1")
            invalid("kill file " + path + " line " + std::to_string(number) +
                    ": expected 0 (kill) or 1 (keep), got '" + std::string(text) + "'");
        if (channel == nchans)
            invalid("kill file " + path + " has more than " + std::to_string(nchans) +
                    " channel entries");
        if (text == "0") {
            if (!killed.empty() && killed.back().end + 1 == channel)
                killed.back().end = channel;
            else
                killed.push_back({channel, channel});
        }
        ++channel;
    }
    if (in.bad())
        throw Error(FROST_ERR_IO, "error reading kill file " + path);
    if (channel != nchans)
        invalid("kill file " + path + " has " + std::to_string(channel) +
                " channel entries; the input has " + std::to_string(nchans));
    return killed;
}

// ---- cleaner -----------------------------------------------------------------

Cleaner::Cleaner(const frost_rfi_config& cfg, const frost_block_layout& layout,
                 float baseline_length, int device)
    : m_cfg(Config::from(cfg)), m_layout(layout), m_device(device), m_n(layout.nchans),
      m_row_bytes(0) {
    m_cfg.validate();
    validate_layout(layout, baseline_length);
    const auto& c = m_cfg.c;
    if ((c.zero_dm != FROST_ZERO_DM_OFF || c.equalize) && layout.dtype != FROST_FLOAT32 &&
        bits_of(layout.dtype) < 8)
        invalid("RFICleaner: zero_dm and equalize need >= 8-bit data");
    if ((c.kadane_spectrum_enabled || !m_cfg.zap_freqs.empty()) && layout.df == 0.0)
        invalid("RFICleaner: zap_freqs and kadane_spectrum need the channel spacing (df)");
    int ndev = 0;
    FB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        invalid("RFICleaner: device " + std::to_string(device) + " does not exist");
    DeviceGuard g(device);

    m_row_bytes = layout.nchans * static_cast<SizeType>(bits_of(layout.dtype)) / 8;
    const double window_samples = static_cast<double>(baseline_length) / layout.tsamp;
    m_window_len       = std::max(static_cast<SizeType>(window_samples), SizeType{kMinWindow});
    m_smooth_radius    = std::max<SizeType>(static_cast<SizeType>(window_samples / 2), 1);
    m_time_fill_radius = std::max<SizeType>(m_smooth_radius / 4, 1);
    m_chan_fill_radius = std::max<SizeType>(m_n / 60, 1);
    m_clip             = c.narrow_threshold;
    m_narrow_active    = c.narrow_enabled && (layout.dtype == FROST_FLOAT32 || bits_of(layout.dtype) > 4);
    m_transform        = c.zero_dm != FROST_ZERO_DM_OFF || c.equalize;
    m_need_moments     = c.moments_enabled || c.iqrm_enabled || c.kadane_channel_enabled;
    if (layout.dtype == FROST_FLOAT32) {
        m_eq_loc   = 0.0F;
        m_eq_scale = 1.0F;
    } else {
        const int nbits = bits_of(layout.dtype);
        m_eq_loc        = static_cast<float>(uint64_t{1} << (nbits - 1));
        m_eq_scale      = static_cast<float>(uint64_t{1} << nbits) / 16.0F;
    }
    build_static_mask();
    m_mask                = m_static_mask;
    m_report              = frost_rfi_report{};
    m_report.chans_zapped = count_zeros(m_static_mask);
    m_report.chans_masked = m_report.chans_zapped;
    FB_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
    for (auto& e : m_ev)
        FB_CUDA(cudaEventCreate(&e));
    h2d(m_static_mask_d, m_static_mask.data(), m_n, m_stream);
    // zero-DM fit of the last full block (read by short tails); zero until one
    m_zdot_a_d.reserve(m_n * sizeof(float));
    m_zdot_b_d.reserve(m_n * sizeof(float));
    FB_CUDA(cudaMemsetAsync(m_zdot_a_d.get(), 0, m_n * sizeof(float), m_stream));
    FB_CUDA(cudaMemsetAsync(m_zdot_b_d.get(), 0, m_n * sizeof(float), m_stream));
    m_counters.reserve(kRepSlots * sizeof(unsigned long long));
    m_pinned.reserve(kRepSlots * sizeof(unsigned long long) + m_n);
    // channel-decision scratch; IQRM lags of this band
    if (c.iqrm_enabled)
        m_lags = iqrm_lags(m_n, c.iqrm_radius > 0 ? c.iqrm_radius : std::max<SizeType>(m_n / 10, 1));
    m_chan_scratch.reserve(ChannelScratch::size_for(m_n, m_lags.size()));
    m_cw.carve(m_chan_scratch.get(), m_n, m_lags.size());
    if (!m_lags.empty())
        FB_CUDA(cudaMemcpyAsync(m_cw.lags, m_lags.data(), m_lags.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, m_stream));
    // Two-term reciprocals of the Welford counts: y_hi = RN(1/n) and
    // y_lo = RN((1 - n y_hi) / n), the residual exact by a fused multiply-add.
    std::vector<double> recip(2 * (layout.max_nsamps + 1), 0.0);
    for (SizeType n = 1; n <= layout.max_nsamps; ++n) {
        const double dn = static_cast<double>(n);
        const double yh = 1.0 / dn;
        recip[2 * n]     = yh;
        recip[2 * n + 1] = std::fma(-dn, yh, 1.0) / dn;
    }
    h2d(m_recip, recip.data(), recip.size(), m_stream);
    FB_CUDA(cudaStreamSynchronize(m_stream));
}

Cleaner::~Cleaner() {
    if (m_stream != nullptr) {
        cudaSetDevice(m_device);
        cudaStreamSynchronize(m_stream);
        for (auto e : m_ev)
            if (e != nullptr)
                cudaEventDestroy(e);
        cudaStreamDestroy(m_stream);
    }
}

const std::vector<uint8_t>& Cleaner::time_flags() const {
    if (!m_flags_fresh) {
        m_time_flags.assign(m_flags_len, 0U);
        if (m_flags_on_device && m_flags_len > 0) {
            DeviceGuard g(m_device);
            FB_CUDA(cudaMemcpyAsync(m_time_flags.data(), m_time_flags_d.get(), m_flags_len,
                                    cudaMemcpyDeviceToHost, m_stream));
            FB_CUDA(cudaStreamSynchronize(m_stream));
        }
        m_flags_fresh = true;
    }
    return m_time_flags;
}

void Cleaner::build_static_mask() {
    m_static_mask.assign(m_n, 1U);
    apply_manual_killmask(m_static_mask, m_cfg.zap_chans);
    for (SizeType c = 0; c < m_n; ++c) {
        const double f = m_layout.f0 + (static_cast<double>(c) * m_layout.df);
        for (const auto& r : m_cfg.zap_freqs)
            if (f >= r.lo && f <= r.hi)
                m_static_mask[c] = 0;
    }
}

SizeType Cleaner::memory_usage() const {
    const DeviceBuffer* all[] = {
        &m_raw, &m_samples, &m_loc, &m_scale, &m_inv, &m_loc2, &m_scale2, &m_unmeasured,
        &m_moments, &m_clip_mean, &m_clip_inv, &m_mask_d, &m_static_mask_d, &m_good_prefix,
        &m_s_det, &m_s_keep_d, &m_s_keep_f, &m_row_std, &m_kspec_pos, &m_kspec_neg,
        &m_kspec_whole, &m_row_clip, &m_row_kchan, &m_slow_rows, &m_nslow, &m_chunk_min, &m_chunk_max, &m_chunk_zdot, &m_chunk_kpos, &m_chunk_kneg,
        &m_lo, &m_hi, &m_zdot_sum, &m_kpos_best, &m_kneg_best, &m_time_flags_d, &m_zdot_a_d,
        &m_zdot_b_d, &m_kchan_pos_d, &m_kchan_neg_d, &m_kchan_any_d, &m_flagged_d, &m_work, &m_out, &m_counters,
        &m_first_bad, &m_tail_loc, &m_tail_scale, &m_tail_out_loc, &m_tail_out_scale, &m_recip,
        &m_chan_scratch, &m_flag_scratch};
    SizeType total = 0;
    for (const auto* b : all)
        total += b->bytes();
    return total;
}

SizeType Cleaner::estimate_memory(const frost_rfi_config& cfg, const frost_block_layout& layout,
                                  float baseline_length) {
    Config conf = Config::from(cfg);
    conf.validate();
    validate_layout(layout, baseline_length);
    const auto& c         = conf.c;
    const SizeType n      = layout.nchans;
    const SizeType T      = layout.max_nsamps;
    const SizeType row    = n * static_cast<SizeType>(bits_of(layout.dtype)) / 8;
    const SizeType window = std::max(static_cast<SizeType>(static_cast<double>(baseline_length) / layout.tsamp),
                                     SizeType{kMinWindow});
    const SizeType nwin   = std::max<SizeType>(T / window, 1);
    const SizeType nck    = std::clamp<SizeType>((T + kMinChunkRows - 1) / kMinChunkRows, 1, kMaxChunks) * n;
    const bool moments    = c.moments_enabled || c.iqrm_enabled || c.kadane_channel_enabled;
    const bool zdot       = c.zero_dm == FROST_ZERO_DM_ZDOT;
    const bool kchan      = c.kadane_channel_enabled != 0;
    const SizeType T1     = std::max<SizeType>(T, 1);
    const SizeType f      = sizeof(float);
    SizeType total        = 0;
    // ensure_capacity(T, T): raw block, float work and output, per-window
    // statistics, tails, counters
    total += std::max<SizeType>(T * row, 16) + 2 * std::max<SizeType>(T * n * f, 16);
    total += 5 * nwin * n * f + 4 * n * f + kRepSlots * sizeof(unsigned long long) + sizeof(unsigned long long);
    // decision scratch (channel mask, time flags)
    const SizeType nlags = c.iqrm_enabled
                               ? iqrm_lags(n, c.iqrm_radius > 0 ? c.iqrm_radius : std::max<SizeType>(n / 10, 1)).size()
                               : 0;
    total += ChannelScratch::size_for(n, nlags) + FlagScratch::size_for(T, c.broad_boxcar_max);
    // reserve_phase_buffers
    total += nwin * kMaxBandpassRows * n * f + n * sizeof(uint32_t);
    total += (moments ? nwin * n * sizeof(MomentSums) : 0) + 2 * std::max<SizeType>(moments ? nwin * n * f : 0, f);
    total += T * (f + sizeof(double) + f + f) + 2 * T1 * sizeof(Span32) + 2 * T1;
    total += 2 * T1 + T1 * sizeof(uint32_t) + 16; // row_clip, row_kchan, the listed rows and their count
    total += 2 * nck * f + std::max<SizeType>(zdot ? nck : 1, 1) * sizeof(ZdotSums) +
             2 * std::max<SizeType>(kchan ? nck : 1, 1) * sizeof(KadaneState);
    total += 2 * n * f + n * sizeof(ZdotSums) + 2 * n * sizeof(Run);
    // tables uploaded per gulp: masks, good-channel prefix, zero-DM fit,
    // Kadane segments, flagged samples (at most every sample), Welford
    // two-term reciprocals
    total += 2 * n + (n + 1) * sizeof(uint64_t) + 2 * n * f + 2 * (kchan ? n : 1) * sizeof(Segment) + n;
    total += T1 * sizeof(uint64_t) + 2 * (T + 1) * sizeof(double);
    return total;
}

Dims Cleaner::dims(SizeType nsamps, int dtype) const {
    Dims d{};
    d.dtype     = dtype;
    d.nchans    = m_n;
    d.row_bytes = m_row_bytes;
    d.nsamps    = nsamps;
    d.window    = m_window_len;
    d.nwin      = std::max<SizeType>(nsamps / m_window_len, 1);
    const SizeType by_rows = (nsamps + kMinChunkRows - 1) / kMinChunkRows;
    d.nchunks   = std::clamp<SizeType>(by_rows, 1, kMaxChunks);
    d.chunk     = (nsamps + d.nchunks - 1) / d.nchunks;
    return d;
}

ApplyParams Cleaner::apply_params() const {
    const auto& c = m_cfg.c;
    ApplyParams p{};
    p.seed             = c.seed;
    p.block_index      = m_block_index;
    p.chan_fill_radius = m_chan_fill_radius;
    p.time_fill_radius = m_time_fill_radius;
    p.clip             = m_clip;
    p.eq_loc           = m_eq_loc;
    p.eq_scale         = m_eq_scale;
    p.narrow_active    = m_narrow_active ? 1 : 0;
    p.kspec            = c.kadane_spectrum_enabled ? 1 : 0;
    p.kchan            = c.kadane_channel_enabled ? 1 : 0;
    p.neighbour        = c.fill == FROST_FILL_NEIGHBOUR ? 1 : 0;
    p.noise            = c.fill == FROST_FILL_NOISE ? 1 : 0;
    p.zero_dm          = c.zero_dm;
    p.equalize         = c.equalize;
    p.transform        = m_transform ? 1 : 0;
    return p;
}

void Cleaner::ensure_capacity(SizeType capacity, SizeType valid) {
    const SizeType n = m_n;
    m_raw.reserve(std::max<SizeType>(capacity * m_row_bytes, 16));
    m_work.reserve(std::max<SizeType>(valid * n * sizeof(float), 16));
    m_out.reserve(std::max<SizeType>(capacity * n * sizeof(float), 16));
    const SizeType nwin_max = std::max<SizeType>(valid / m_window_len, 1);
    m_loc.reserve(nwin_max * n * sizeof(float));
    m_scale.reserve(nwin_max * n * sizeof(float));
    m_inv.reserve(nwin_max * n * sizeof(float));
    m_loc2.reserve(nwin_max * n * sizeof(float));
    m_scale2.reserve(nwin_max * n * sizeof(float));
    m_tail_loc.reserve(n * sizeof(float));
    m_tail_scale.reserve(n * sizeof(float));
    m_tail_out_loc.reserve(n * sizeof(float));
    m_tail_out_scale.reserve(n * sizeof(float));
    m_counters.reserve(kRepSlots * sizeof(unsigned long long));
    m_first_bad.reserve(sizeof(unsigned long long));
}

const float* Cleaner::execute_normalized(const uint8_t* block, SizeType bytes, SizeType valid,
                                         bool on_device, cudaStream_t stream) {
    if (bytes % m_row_bytes != 0 || bytes / m_row_bytes > m_layout.max_nsamps)
        invalid("RFICleaner: invalid normalized block size");
    if (block == nullptr && bytes != 0)
        invalid("RFICleaner: null block");
    const SizeType capacity = bytes / m_row_bytes;
    if (valid == 0)
        valid = capacity;
    if (valid > capacity)
        invalid("RFICleaner: nsamps exceeds block");
    DeviceGuard g(m_device);
    cudaStream_t s = stream != nullptr ? stream : m_stream;
    ensure_capacity(capacity, valid);
    m_capacity = capacity;
    struct CountLaunches {
        uint64_t& total;
        uint64_t before = launch_counter();
        ~CountLaunches() { total += launch_counter() - before; }
    } counting{m_launches};

    // Raw block on the device.
    // A device block that does not start on a 16-byte boundary is copied
    // into the cleaner's own buffer first: the kernels read whole samples
    // and 16-byte row segments, which a misaligned pointer would fault.
    const uint8_t* raw = block;
    if (!on_device) {
        if (bytes)
            FB_CUDA(cudaMemcpyAsync(m_raw.get(), block, bytes, cudaMemcpyHostToDevice, s));
        raw = m_raw.as<uint8_t>();
    } else if (reinterpret_cast<uintptr_t>(block) % 16 != 0) {
        if (bytes)
            FB_CUDA(cudaMemcpyAsync(m_raw.get(), block, bytes, cudaMemcpyDeviceToDevice, s));
        raw = m_raw.as<uint8_t>();
    }
    // Non-finite float32 input is rejected before any statistics.
    if (m_layout.dtype == FROST_FLOAT32 && valid > 0) {
        const uint64_t words = valid * m_n;
        unsigned long long first = words;
        FB_CUDA(cudaMemcpyAsync(m_first_bad.get(), &first, sizeof(first), cudaMemcpyHostToDevice, s));
        launch_check_finite(raw, words, m_first_bad.as<unsigned long long>(), s);
        FB_CUDA(cudaMemcpyAsync(&first, m_first_bad.get(), sizeof(first), cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaStreamSynchronize(s));
        if (first != words)
            invalid("RFI: non-finite float32 input at sample " + std::to_string(first / m_n) +
                    ", channel " + std::to_string(first % m_n));
    }

    const bool short_block = valid < static_cast<SizeType>(std::max(kMinWindow, kMinBlockSamps));
    const int flip         = m_layout.df < 0.0 ? 1 : 0;
    FB_CUDA(cudaMemsetAsync(m_out.get(), 0, capacity * m_n * sizeof(float), s));
    if (short_block && m_tail_ready) {
        Dims d = dims(valid, m_layout.dtype);
        launch_unpack(d, raw, m_work.as<float>(), s);
        normalize_short(capacity, valid, s);
        FB_CUDA(cudaStreamSynchronize(s));
        m_flags_len       = valid;
        m_flags_on_device = false;
        m_flags_fresh     = false;
        return m_out.as<float>();
    }

    // The full suite on float samples (lib/cpu/rfi_cpu.cpp:191-208).
    m_report              = frost_rfi_report{};
    m_report.nsamps       = valid;
    m_mask                = m_static_mask;
    m_report.chans_zapped = count_zeros(m_static_mask);
    m_report.chans_masked = m_report.chans_zapped;
    m_raw_ptr           = raw;
    Dims d                = dims(valid, m_layout.dtype);
    const float* loc      = m_loc.as<float>();
    const float* scale    = m_scale.as<float>();
    if (short_block) {
        // Too short for statistics: data unchanged, static mask; calibrate
        // each channel by its own mean/std.
        ++m_block_index;
        d.nwin = 1;
        launch_unpack(d, raw, m_work.as<float>(), s);
        h2d(m_mask_d, m_mask.data(), m_n, s);
        launch_welford(d, m_work.as<float>(), m_recip.as<double>(), m_loc2.as<float>(), m_scale2.as<float>(), s);
        loc   = m_loc2.as<float>();
        scale = m_scale2.as<float>();
    } else {
        run_full(d, s);
        ++m_block_index;
        if (m_transform) {
            launch_welford(d, m_work.as<float>(), m_recip.as<double>(), m_loc2.as<float>(), m_scale2.as<float>(), s);
            loc   = m_loc2.as<float>();
            scale = m_scale2.as<float>();
        }
        const SizeType last = (d.nwin - 1) * m_n;
        FB_CUDA(cudaMemcpyAsync(m_tail_loc.get(), m_loc.as<float>() + last, m_n * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
        FB_CUDA(cudaMemcpyAsync(m_tail_scale.get(), m_scale.as<float>() + last, m_n * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
        FB_CUDA(cudaMemcpyAsync(m_tail_out_loc.get(), loc + last, m_n * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
        FB_CUDA(cudaMemcpyAsync(m_tail_out_scale.get(), scale + last, m_n * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
    }
    launch_normalize(d, m_work.as<float>(), loc, scale, m_mask_d.as<uint8_t>(), flip, capacity,
                     m_out.as<float>(), s);
    if (short_block)
        FB_CUDA(cudaStreamSynchronize(s));
    else
        read_back(s);
    m_flags_len       = valid;
    m_flags_on_device = !short_block;
    m_flags_fresh     = false;
    m_tail_ready      = !short_block;
    return m_out.as<float>();
}

// The gulp's channel mask and report counters, copied back once the whole
// gulp (normalisation included) is queued; the stage times are the device
// intervals between the phase events.
void Cleaner::read_back(cudaStream_t s) {
    auto* counts = m_pinned.as<unsigned long long>();
    auto* mask   = reinterpret_cast<uint8_t*>(counts + kRepSlots);
    FB_CUDA(cudaMemcpyAsync(counts, m_counters.get(), kRepSlots * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(mask, m_mask_d.get(), m_n, cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    m_mask.assign(mask, mask + m_n);
    m_report.chans_moments         = counts[kRepMoments];
    m_report.chans_iqrm            = counts[kRepIqrm];
    m_report.chans_grown           = counts[kRepGrown];
    m_report.chans_masked          = counts[kRepMasked];
    m_report.chans_dead            = counts[kRepDead];
    m_report.samps_broad           = counts[kRepBroad];
    m_report.samps_dropout         = counts[kRepDropout];
    m_report.samps_kadane          = counts[kRepKadane];
    m_report.samps_flagged         = counts[kRepFlagged];
    m_report.cells_narrow          = counts[kCountNarrow];
    m_report.cells_kadane_spectrum = counts[kCountKspec];
    m_report.cells_kadane_channel  = counts[kCountKchan];
    m_report.fill_fallbacks        = counts[kCountFallback];
    double* t[] = {&m_report.t_bandpass, &m_report.t_moments, &m_report.t_scan, &m_report.t_flags,
                   &m_report.t_apply};
    for (int i = 0; i < 5; ++i) {
        float ms = 0.0F;
        FB_CUDA(cudaEventElapsedTime(&ms, m_ev[i], m_ev[i + 1]));
        *t[i] = 1e-3 * static_cast<double>(ms);
    }
}

void Cleaner::normalize_short(SizeType capacity, SizeType valid, cudaStream_t s) {
    m_report                    = frost_rfi_report{};
    m_report.nsamps             = valid;
    m_report.chans_zapped       = count_zeros(m_static_mask);
    m_report.chans_masked       = count_zeros(m_mask);
    m_report.calibration_reused = 1;
    Dims d                      = dims(valid, m_layout.dtype);
    h2d(m_mask_d, m_mask.data(), m_n, s);
    launch_normalize_short(d, apply_params(), m_work.as<float>(), m_tail_loc.as<float>(),
                           m_tail_scale.as<float>(), m_tail_out_loc.as<float>(),
                           m_tail_out_scale.as<float>(), m_mask_d.as<uint8_t>(),
                           m_zdot_a_d.as<float>(), m_zdot_b_d.as<float>(),
                           m_layout.df < 0.0 ? 1 : 0, capacity, m_out.as<float>(), s);
    ++m_block_index;
}

// Device buffers of the full cleaning path for a block of d.nsamps rows.
void Cleaner::reserve_phase_buffers(const Dims& d) {
    const SizeType n    = m_n;
    const SizeType nwin = d.nwin;
    const SizeType T    = d.nsamps;
    const auto& c       = m_cfg.c;
    const bool zdot     = c.zero_dm == FROST_ZERO_DM_ZDOT;
    const bool kchan    = c.kadane_channel_enabled != 0;
    m_samples.reserve(nwin * kMaxBandpassRows * n * sizeof(float));
    m_unmeasured.reserve(n * sizeof(uint32_t));
    if (m_need_moments) {
        m_moments.reserve(nwin * n * sizeof(MomentSums));
        m_clip_mean.reserve(nwin * n * sizeof(float));
        m_clip_inv.reserve(nwin * n * sizeof(float));
    }
    m_s_det.reserve(T * sizeof(float));
    m_s_keep_d.reserve(T * sizeof(double));
    m_s_keep_f.reserve(T * sizeof(float));
    m_row_std.reserve(T * sizeof(float));
    m_kspec_pos.reserve(std::max<SizeType>(T, 1) * sizeof(Span32));
    m_kspec_neg.reserve(std::max<SizeType>(T, 1) * sizeof(Span32));
    m_kspec_whole.reserve(std::max<SizeType>(T, 1));
    m_row_clip.reserve(std::max<SizeType>(T, 1));
    m_row_kchan.reserve(std::max<SizeType>(T, 1));
    m_slow_rows.reserve(std::max<SizeType>(T, 1) * sizeof(uint32_t));
    m_nslow.reserve(16);
    m_time_flags_d.reserve(std::max<SizeType>(T, 1));
    const SizeType nck = d.nchunks * n;
    m_chunk_min.reserve(nck * sizeof(float));
    m_chunk_max.reserve(nck * sizeof(float));
    m_chunk_zdot.reserve(std::max<SizeType>(zdot ? nck : 1, 1) * sizeof(ZdotSums));
    m_chunk_kpos.reserve(std::max<SizeType>(kchan ? nck : 1, 1) * sizeof(KadaneState));
    m_chunk_kneg.reserve(std::max<SizeType>(kchan ? nck : 1, 1) * sizeof(KadaneState));
    m_lo.reserve(n * sizeof(float));
    m_hi.reserve(n * sizeof(float));
    m_zdot_sum.reserve(n * sizeof(ZdotSums));
    m_kpos_best.reserve(n * sizeof(Run));
    m_kneg_best.reserve(n * sizeof(Run));
    m_clip_mean.reserve(sizeof(float));
    m_clip_inv.reserve(sizeof(float));
    // decision outputs
    m_mask_d.reserve(n);
    m_good_prefix.reserve((n + 1) * sizeof(uint64_t));
    m_flagged_d.reserve(std::max<SizeType>(T, 1) * sizeof(uint64_t));
    m_kchan_pos_d.reserve((kchan ? n : 1) * sizeof(Segment));
    m_kchan_neg_d.reserve((kchan ? n : 1) * sizeof(Segment));
    m_kchan_any_d.reserve(n);
    m_flag_scratch.reserve(FlagScratch::size_for(T, c.broad_boxcar_max));
    m_fw.carve(m_flag_scratch.get(), T, c.broad_boxcar_max);
}

ChannelMaskParams Cleaner::channel_params(const Dims& d) const {
    const auto& c = m_cfg.c;
    ChannelMaskParams p{};
    p.n              = m_n;
    p.nwin           = d.nwin;
    p.moments        = c.moments_enabled ? 1 : 0;
    p.need_clip      = m_need_moments ? 1 : 0;
    p.stat_on[0]     = c.moments_mean ? 1 : 0;
    p.stat_on[1]     = c.moments_std ? 1 : 0;
    p.stat_on[2]     = c.moments_skewness ? 1 : 0;
    p.stat_on[3]     = c.moments_kurtosis ? 1 : 0;
    p.stat_on[4]     = c.moments_autocorr ? 1 : 0;
    p.k              = c.moments_threshold;
    p.kurt_max       = c.moments_kurtosis_max;
    p.iqrm           = c.iqrm_enabled ? 1 : 0;
    p.iqrm_threshold = c.iqrm_threshold;
    p.grow           = c.mask_grow;
    return p;
}

FlagParams Cleaner::flag_params(const Dims& d) const {
    const auto& c = m_cfg.c;
    FlagParams p{};
    p.nsamps           = d.nsamps;
    p.nchans           = m_n;
    p.nwin             = d.nwin;
    p.broad            = c.broad_enabled ? 1 : 0;
    p.smooth_radius    = m_smooth_radius;
    p.broad_threshold  = c.broad_threshold;
    p.boxcar_max       = c.broad_boxcar_max;
    p.dropout          = c.dropout_enabled ? 1 : 0;
    p.dropout_fraction = c.dropout_min_std_fraction;
    p.kspec            = c.kadane_spectrum_enabled ? 1 : 0;
    p.zdot             = c.zero_dm == FROST_ZERO_DM_ZDOT ? 1 : 0;
    p.kchan            = c.kadane_channel_enabled ? 1 : 0;
    p.kchan_min_len    = static_cast<double>(c.kadane_channel_min_duration) / m_layout.tsamp;
    p.kchan_threshold  = c.kadane_channel_threshold;
    return p;
}

void Cleaner::preallocate() {
    DeviceGuard g(m_device);
    const SizeType T = m_layout.max_nsamps;
    ensure_capacity(T, T);
    reserve_phase_buffers(dims(T, m_layout.dtype));
}

void Cleaner::run_full(const Dims& d, cudaStream_t s) {
    reserve_phase_buffers(d);
    const SizeType n   = m_n;
    const auto& c      = m_cfg.c;
    const uint8_t* raw = m_raw_ptr;
    const bool zdot    = c.zero_dm == FROST_ZERO_DM_ZDOT;
    const bool kchan   = c.kadane_channel_enabled != 0;
    const bool kspec   = c.kadane_spectrum_enabled != 0;
    auto* counters     = m_counters.as<unsigned long long>();
    FB_CUDA(cudaMemsetAsync(counters, 0, kRepSlots * sizeof(unsigned long long), s));

    // ---- bandpass ----
    FB_CUDA(cudaEventRecord(m_ev[0], s));
    FB_CUDA(cudaMemsetAsync(m_unmeasured.get(), 0, n * sizeof(uint32_t), s));
    launch_sample_rows(d, raw, m_samples.as<float>(), s);
    launch_bandpass(d, m_samples.as<float>(), m_loc.as<float>(), m_scale.as<float>(),
                    m_inv.as<float>(), m_unmeasured.as<uint32_t>(), s);
    FB_CUDA(cudaEventRecord(m_ev[1], s));

    // ---- moments and channel mask (lib/cpu/rfi_cpu_measure.cpp:140-300) ----
    if (m_need_moments)
        launch_moments(d, raw, m_loc.as<float>(), m_inv.as<float>(), m_static_mask_d.as<uint8_t>(),
                       m_clip, m_moments.as<MomentSums>(), s);
    decide_channel_mask(channel_params(d), m_cw, m_need_moments ? m_moments.as<MomentSums>() : nullptr,
                        m_scale.as<float>(), m_unmeasured.as<uint32_t>(), m_static_mask_d.as<uint8_t>(),
                        m_clip_mean.as<float>(), m_clip_inv.as<float>(), m_mask_d.as<uint8_t>(),
                        m_good_prefix.as<uint64_t>(), counters, s);
    FB_CUDA(cudaEventRecord(m_ev[2], s));

    // ---- scan (masked channels are skipped; with no good channel the
    // series come out as frost's empty ones) ----
    KspecParams kp{};
    kp.enabled      = kspec ? 1 : 0;
    kp.min_bw_chans = kspec ? static_cast<double>(c.kadane_spectrum_min_bandwidth) / std::abs(m_layout.df) : 0.0;
    kp.whole_chans  = static_cast<double>(c.kadane_spectrum_whole_band_fraction) * static_cast<double>(n);
    kp.threshold    = c.kadane_spectrum_threshold;
    launch_scan_rows(d, raw, m_loc.as<float>(), m_inv.as<float>(), m_mask_d.as<uint8_t>(), m_clip, kp,
                     m_good_prefix.as<uint64_t>(), m_s_det.as<float>(), m_s_keep_d.as<double>(),
                     m_s_keep_f.as<float>(), m_row_std.as<float>(), m_kspec_pos.as<Span32>(),
                     m_kspec_neg.as<Span32>(), m_kspec_whole.as<uint8_t>(), m_row_clip.as<uint8_t>(), s);
    launch_scan_cols(d, raw, m_loc.as<float>(), m_inv.as<float>(), m_mask_d.as<uint8_t>(), m_clip,
                     m_s_keep_d.as<double>(), zdot ? 1 : 0, kchan ? 1 : 0, m_clip_mean.as<float>(),
                     m_clip_inv.as<float>(), m_chunk_min.as<float>(), m_chunk_max.as<float>(),
                     m_chunk_zdot.as<ZdotSums>(), m_chunk_kpos.as<KadaneState>(), m_chunk_kneg.as<KadaneState>(),
                     m_lo.as<float>(), m_hi.as<float>(), m_zdot_sum.as<ZdotSums>(), m_kpos_best.as<Run>(),
                     m_kneg_best.as<Run>(), s);
    FB_CUDA(cudaEventRecord(m_ev[3], s));

    // ---- flags (lib/cpu/rfi_cpu.cpp:347-468) ----
    decide_flags(flag_params(d), m_fw, m_good_prefix.as<uint64_t>(), m_unmeasured.as<uint32_t>(),
                 m_lo.as<float>(), m_hi.as<float>(), m_s_det.as<float>(), m_row_std.as<float>(),
                 m_kspec_whole.as<uint8_t>(), m_zdot_sum.as<ZdotSums>(), m_kpos_best.as<Run>(),
                 m_kneg_best.as<Run>(), m_mask_d.as<uint8_t>(), m_time_flags_d.as<uint8_t>(),
                 m_zdot_a_d.as<float>(), m_zdot_b_d.as<float>(), m_kchan_pos_d.as<Segment>(),
                 m_kchan_neg_d.as<Segment>(), m_kchan_any_d.as<uint8_t>(), m_flagged_d.as<uint64_t>(), counters,
                 s);
    FB_CUDA(cudaEventRecord(m_ev[4], s));

    // ---- apply (lib/cpu/rfi_cpu.cpp:526-720) ----
    const ApplyParams p = apply_params();
    if (kchan)
        launch_kchan_rows(d, m_kchan_pos_d.as<Segment>(), m_kchan_neg_d.as<Segment>(), m_kchan_any_d.as<uint8_t>(),
                          m_row_kchan.as<uint8_t>(), s);
    launch_apply_unflagged(d, p, raw, m_loc.as<float>(), m_scale.as<float>(), m_inv.as<float>(),
                           m_mask_d.as<uint8_t>(), m_time_flags_d.as<uint8_t>(), m_kspec_pos.as<Span32>(),
                           m_kspec_neg.as<Span32>(), m_kchan_pos_d.as<Segment>(), m_kchan_neg_d.as<Segment>(),
                           m_kchan_any_d.as<uint8_t>(), m_s_keep_f.as<float>(), m_zdot_a_d.as<float>(),
                           m_zdot_b_d.as<float>(), m_row_clip.as<uint8_t>(), m_row_kchan.as<uint8_t>(),
                           m_slow_rows.as<uint32_t>(), m_nslow.as<unsigned int>(), m_work.as<float>(), counters, s);
    launch_apply_flagged(d, p, m_flagged_d.as<uint64_t>(), counters + kRepFlagged, m_loc.as<float>(),
                         m_scale.as<float>(), m_inv.as<float>(), m_mask_d.as<uint8_t>(),
                         m_time_flags_d.as<uint8_t>(), m_work.as<float>(), counters, s);
    FB_CUDA(cudaEventRecord(m_ev[5], s));
}

} // namespace fb::rfi
