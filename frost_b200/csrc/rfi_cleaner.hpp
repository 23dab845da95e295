// RFICleaner on the GPU: frost's per-gulp RFI excision and normalisation
// (include/frost/prepare/rfi.hpp:243-297, lib/cpu/rfi_cpu.cpp) with every
// T x C pass as a CUDA kernel and the per-gulp decisions as device kernels
// on the short series those passes reduce the block to (rfi_decide.cu), so
// a gulp runs without host round trips until its results are read back.
#pragma once

#include <cstdint>
#include <span>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.hpp"
#include "rfi_decide.hpp"
#include "rfi_kernels.hpp"

namespace fb::rfi {

/** Owned copy of frost_rfi_config (the zap arrays are copied). */
struct Config {
    frost_rfi_config c{};
    std::vector<frost_channel_range> zap_chans;
    std::vector<frost_frequency_range> zap_freqs;
    static Config from(const frost_rfi_config& in);
    void validate() const;
};

void config_default(frost_rfi_config* cfg);
void validate_layout(const frost_block_layout& l, float baseline_length);
void apply_manual_killmask(std::span<uint8_t> mask, std::span<const frost_channel_range> zaps);
std::vector<frost_channel_range> read_kill_file(const std::string& path, SizeType nchans);

/** Quiet-configuration clean + normalise of one device block into `out`
 * using only the static scratch array of rfi_static.cu (no allocation). */
void normalize_static(const frost_block_layout& layout, float baseline_length, const uint8_t* block,
                      size_t block_bytes, size_t nsamps, float* out, size_t out_count,
                      cudaStream_t stream);

class Cleaner {
public:
    Cleaner(const frost_rfi_config& cfg, const frost_block_layout& layout, float baseline_length,
            int device);
    ~Cleaner();
    Cleaner(const Cleaner&)            = delete;
    Cleaner& operator=(const Cleaner&) = delete;

    /** execute_normalized on a host or device block; returns the device
     * [nchans][capacity] waterfall (valid until the next call). */
    const float* execute_normalized(const uint8_t* block, SizeType bytes, SizeType valid,
                                    bool on_device, cudaStream_t stream);

    const std::vector<uint8_t>& channel_mask() const { return m_mask; }
    const frost_rfi_report& report() const { return m_report; }
    /** Per-sample flags of the last call (1 = flagged), read back from the
     * device on first use after the call. */
    const std::vector<uint8_t>& time_flags() const;
    const float* output() const { return m_out.as<float>(); }
    SizeType capacity() const { return m_capacity; }
    SizeType nchans() const { return m_n; }
    int device() const { return m_device; }
    cudaStream_t stream() const { return m_stream; }
    SizeType memory_usage() const;
    /** Device bytes a cleaner for (cfg, layout) holds once its whole-block
     * buffers are in place (preallocate, then any gulp), computed on the
     * host without allocating: the buffers sized by data (flagged samples,
     * Kadane segments) at their largest. RFICleaner::estimate_memory
     * (include/frost/prepare/rfi.hpp) for the device path. */
    static SizeType estimate_memory(const frost_rfi_config& cfg, const frost_block_layout& layout,
                                    float baseline_length);
    /** Allocates every device buffer a full block of max_nsamps rows needs,
     * so memory_usage() is the cleaner's steady-state footprint. */
    void preallocate();
    uint64_t launches() const { return m_launches; }

private:
    uint64_t m_launches = 0;
    Config m_cfg;
    frost_block_layout m_layout;
    int m_device;
    cudaStream_t m_stream = nullptr;
    SizeType m_n, m_row_bytes;
    SizeType m_window_len = 0, m_smooth_radius = 0, m_time_fill_radius = 0,
             m_chan_fill_radius = 0;
    float m_clip = 0.0F;
    bool m_narrow_active = false, m_transform = false, m_need_moments = false;
    float m_eq_loc = 0.0F, m_eq_scale = 1.0F;
    uint64_t m_block_index = 0;

    std::vector<uint8_t> m_static_mask, m_mask;
    frost_rfi_report m_report{};
    SizeType m_capacity = 0;
    // time flags of the last call: m_flags_len samples, on the device unless
    // the call flagged nothing by construction (short blocks)
    mutable std::vector<uint8_t> m_time_flags;
    mutable bool m_flags_fresh = true;
    SizeType m_flags_len       = 0;
    bool m_flags_on_device     = false;

    // Retained calibration for short tails (lib/cpu/rfi_cpu.cpp:209-244);
    // the zero-DM fit stays in m_zdot_a_d / m_zdot_b_d.
    bool m_tail_ready = false;

    // Decision scratch (rfi_decide.hpp) and the IQRM lags of this band.
    std::vector<uint64_t> m_lags;
    DeviceBuffer m_chan_scratch, m_flag_scratch;
    ChannelScratch m_cw{};
    FlagScratch m_fw{};
    cudaEvent_t m_ev[6] = {};

    // Device workspace.
    DeviceBuffer m_raw, m_samples, m_loc, m_scale, m_inv, m_loc2, m_scale2, m_unmeasured,
        m_moments, m_clip_mean, m_clip_inv, m_mask_d, m_static_mask_d, m_good_prefix, m_s_det,
        m_s_keep_d, m_s_keep_f, m_row_std, m_kspec_pos, m_kspec_neg, m_kspec_whole, m_row_clip, m_row_kchan, m_slow_rows, m_nslow, m_chunk_min,
        m_chunk_max, m_chunk_zdot, m_chunk_kpos, m_chunk_kneg, m_lo, m_hi, m_zdot_sum, m_kpos_best,
        m_kneg_best, m_time_flags_d, m_zdot_a_d, m_zdot_b_d, m_kchan_pos_d, m_kchan_neg_d, m_kchan_any_d,
        m_flagged_d, m_work, m_out, m_counters, m_first_bad, m_tail_loc, m_tail_scale,
        m_tail_out_loc, m_tail_out_scale;
    DeviceBuffer m_recip; // [max_nsamps + 1] pairs: RN(1/n) and RN((1 - n RN(1/n)) / n)
    PinnedBuffer m_pinned;
    const uint8_t* m_raw_ptr = nullptr; // raw block of the current call (device)

    void build_static_mask();
    void ensure_capacity(SizeType capacity, SizeType valid);
    void reserve_phase_buffers(const Dims& d);
    ApplyParams apply_params() const;
    Dims dims(SizeType nsamps, int dtype) const;

    void run_full(const Dims& d, cudaStream_t s);
    void normalize_short(SizeType capacity, SizeType valid, cudaStream_t s);
    ChannelMaskParams channel_params(const Dims& d) const;
    FlagParams flag_params(const Dims& d) const;
    void read_back(cudaStream_t s);
};

} // namespace fb::rfi
