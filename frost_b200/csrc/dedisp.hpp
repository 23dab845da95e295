// DM trial grid and ascending FDMT band edges.
#pragma once

#include <vector>

#include "common.hpp"

namespace fb::dedisp {

/** generate_dm_list (lib/dedisp/dedisp.cpp:16-69). */
std::vector<float> generate_dm_list(const frost_dedisp_plan_config& cfg);

/** Band edges of make_dmt_fdmt_plan (lib/dedisp/dedisp.cpp:71-89):
 * f_min = min(f0, last) - |df|/2, f_max = f_min + nchans |df|, in float. */
void band_edges(const frost_dedisp_plan_config& cfg, float& f_min, float& f_max);

} // namespace fb::dedisp
