// Self-written stand-in for dmt's candidate record and result view, holding
// the fields the reference's lib/search/postprocess.cpp:79-116 and
// lib/pipeline/pipeline.cpp:478-487 read (dmt v0.8.0 is not vendored).
#pragma once
#include <cstddef>
#include <cstdint>
#include <span>
namespace dmt {
struct RawCandidate {
    float snr                 = 0.0F;
    std::size_t peak_sample   = 0;
    std::size_t begin_sample  = 0;
    std::size_t end_sample    = 0;
    std::size_t filter_idx    = 0;
    std::size_t width         = 0;
    std::size_t dm_idx        = 0;
    float dm                  = 0.0F;
    float f_low_mhz           = 0.0F;
    float f_high_mhz          = 0.0F;
    std::size_t chan_begin    = 0;
    std::size_t chan_end      = 0;
    std::size_t beam_idx      = 0;
    std::size_t subband_level = 0;
    std::size_t subband_idx   = 0;
};
struct CandidateResultView {
    std::span<const RawCandidate> candidates;
    std::size_t dropped_global = 0;
    std::size_t dropped_per_dm = 0;
    [[nodiscard]] bool overflowed() const noexcept { return dropped_global + dropped_per_dm > 0; }
};
} // namespace dmt
