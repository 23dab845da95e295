// Memory planning for one beam on the device (memory_plan.cpp).
#pragma once

#include "common.hpp"
#include "frost_b200.h"

namespace fb::memplan {

/** The device bytes of one beam (frost_estimate_memory). */
frost_memory_estimate estimate(const frost_rfi_config& rfi, const frost_block_layout& layout, float baseline,
                               const frost_dedisp_plan_config& plan, const frost_boxcar_config& search,
                               const frost_postprocess_config* post);

/** check_memory for the device (frost_check_memory); may lower the gulp in
 * `layout` and `plan`. */
frost_memory_check check(const frost_rfi_config& rfi, frost_block_layout& layout, float baseline,
                         frost_dedisp_plan_config& plan, const frost_boxcar_config& search,
                         const frost_postprocess_config* post, bool gulp_is_default, SizeType available_bytes,
                         SizeType memory_limit_bytes, int device);

} // namespace fb::memplan
