// DM trial grid and FDMT band edges (include/frost/dedisp/dedisp.hpp,
// lib/dedisp/dedisp.cpp:16-89). The grid is the Levin/Barsdell
// dispersion-smearing recurrence evaluated in double; each trial is stored as
// float and the next one grows from that float, so the list must be computed
// with the reference's exact operation order to reproduce it bit for bit.

#include "dedisp.hpp"

#include <algorithm>
#include <cmath>
#include <string>

namespace fb::dedisp {

namespace {
constexpr std::size_t kMaxDmTrials = std::size_t{1} << 22;
}

std::vector<float> generate_dm_list(const frost_dedisp_plan_config& cfg) {
    if (!is_finite(cfg.dm_tol) || !(cfg.dm_tol > 1.0F))
        invalid("generate_dm_list: dm_tol must be > 1");
    if (!is_finite(cfg.dm_min) || !is_finite(cfg.dm_max) || !is_finite(cfg.dm_pulse_width) ||
        !is_finite(cfg.dt) || !is_finite(cfg.f0) || !is_finite(cfg.df) || !(cfg.dt > 0.0F) ||
        cfg.nchans == 0)
        invalid("generate_dm_list: dm range, dt, f0 and df must be finite");
    const double dt = static_cast<double>(cfg.dt) * 1e6; // microseconds
    const double ti = static_cast<double>(cfg.dm_pulse_width);
    const double f  = (static_cast<double>(cfg.f0) +
                      (((static_cast<double>(cfg.nchans) / 2.0) - 0.5) * cfg.df)) *
                     1e-3; // GHz
    const double tol2 = static_cast<double>(cfg.dm_tol) * cfg.dm_tol;
    const double a    = 8.3 * cfg.df / (f * f * f);
    const double a2   = a * a;
    const double b2   = a2 * (static_cast<double>(cfg.nchans) * cfg.nchans / 16.0);
    const double c    = ((dt * dt) + (ti * ti)) * (tol2 - 1.0);

    std::vector<float> dms;
    dms.push_back(cfg.dm_min);
    while (dms.back() < cfg.dm_max) {
        const double prev  = dms.back();
        const double prev2 = prev * prev;
        const double k     = c + (tol2 * a2 * prev2);
        const double dm    = ((b2 * prev) + std::sqrt((-a2 * b2 * prev2) + ((a2 + b2) * k))) / (a2 + b2);
        const auto next    = static_cast<float>(dm);
        if (!is_finite(next) || !(next > static_cast<float>(prev)))
            throw Error(FROST_ERR_INTERNAL,
                        "generate_dm_list: the DM trial spacing collapsed at DM " + std::to_string(prev));
        if (dms.size() >= kMaxDmTrials)
            invalid("generate_dm_list: more than 4M DM trials; raise dm_tol or narrow the DM range");
        dms.push_back(next);
    }
    return dms;
}

void band_edges(const frost_dedisp_plan_config& cfg, float& f_min, float& f_max) {
    if (cfg.nchans < 2 || !is_finite(cfg.f0) || !is_finite(cfg.df) || cfg.df == 0.0F)
        invalid("FDMT requires at least two channels and a finite, nonzero frequency step");
    const float last = cfg.f0 + static_cast<float>(cfg.nchans - 1) * cfg.df;
    f_min            = std::min(cfg.f0, last) - 0.5F * std::abs(cfg.df);
    f_max            = f_min + static_cast<float>(cfg.nchans) * std::abs(cfg.df);
    if (!is_positive_finite(f_min) || !is_positive_finite(f_max) || !(f_max > f_min))
        invalid("FDMT requires positive ascending frequency edges");
}

} // namespace fb::dedisp
