// Self-written stand-in for dmt::plans::FDMTPlan, recording only the
// constructor arguments that the reference's lib/dedisp/dedisp.cpp passes
// (band edges, geometry, DM list, mode, sub-band depth). dmt v0.8.0 is not
// vendored; the FDMT itself is restated separately in fdmt_oracle.c.
#pragma once
#include <cstddef>
#include <string>
#include <utility>
#include <vector>
namespace dmt::plans {
class FDMTPlan {
public:
    FDMTPlan(float f_min, float f_max, std::size_t nchans, std::size_t nsamps,
             float dt, std::vector<float> dm_list, std::string mode,
             std::size_t depth)
        : m_f_min(f_min), m_f_max(f_max), m_nchans(nchans), m_nsamps(nsamps),
          m_dt(dt), m_dms(std::move(dm_list)), m_mode(std::move(mode)),
          m_depth(depth) {}
    float get_f_min() const { return m_f_min; }
    float get_f_max() const { return m_f_max; }
    std::size_t get_subband_depth() const { return m_depth; }
    const std::vector<float>& get_dm_grid_final() const { return m_dms; }
private:
    float m_f_min, m_f_max;
    std::size_t m_nchans, m_nsamps;
    float m_dt;
    std::vector<float> m_dms;
    std::string m_mode;
    std::size_t m_depth;
};
} // namespace dmt::plans
