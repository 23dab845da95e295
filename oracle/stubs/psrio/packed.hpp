// Self-written stand-in for psrio's packed-sample reader: LSB-first sub-byte
// samples in byte-aligned rows, little-endian multi-byte samples. Test
// infrastructure for compiling the reference's spectra_cpu.cpp only.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <span>
#include <psrio/common/types.hpp>
namespace psrio {
class DataExtractor {
public:
    DataExtractor(std::span<const std::byte> data, std::size_t nsamps,
                  std::size_t nchans, SampleType type)
        : m_data(data), m_nsamps(nsamps), m_nchans(nchans), m_type(type) {}
    float extract_sample(std::size_t t, std::size_t c) const {
        const auto* p = reinterpret_cast<const std::uint8_t*>(m_data.data());
        const std::size_t i = t * m_nchans + c;
        switch (m_type) {
        case SampleType::kUInt1: return float((p[i >> 3] >> (i & 7)) & 1U);
        case SampleType::kUInt2: return float((p[(2 * i) >> 3] >> ((2 * i) & 7)) & 3U);
        case SampleType::kUInt4: return float((p[(4 * i) >> 3] >> ((4 * i) & 7)) & 15U);
        case SampleType::kUInt8: return float(p[i]);
        case SampleType::kUInt16: { std::uint16_t v; std::memcpy(&v, p + 2 * i, 2); return float(v); }
        case SampleType::kUInt32: { std::uint32_t v; std::memcpy(&v, p + 4 * i, 4); return float(v); }
        case SampleType::kFloat32: { float v; std::memcpy(&v, p + 4 * i, 4); return v; }
        case SampleType::kInt8: return float(static_cast<std::int8_t>(p[i]));
        case SampleType::kInt16: { std::int16_t v; std::memcpy(&v, p + 2 * i, 2); return float(v); }
        }
        return 0.0F;
    }
private:
    std::span<const std::byte> m_data;
    std::size_t m_nsamps, m_nchans;
    SampleType m_type;
};
} // namespace psrio
