// Memory planning for one beam on the device: the host-side footprint of
// the RFI cleaner, the FDMT/search engine and the post-processor, and the
// gulp check frost runs before building them (the device counterpart of
// lib/pipeline/memory.cpp:294-508, MemoryCheck and check_memory).

#include "memory_plan.hpp"

#include <algorithm>
#include <cstdio>
#include <string>

#include <cuda_runtime_api.h>

#include "postprocess.hpp"
#include "rfi_cleaner.hpp"
#include "search_engine.hpp"

namespace fb::memplan {

namespace {

constexpr SizeType kGulpRounding = 1024;

std::string gib(SizeType bytes) {
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%.2f GiB", static_cast<double>(bytes) / static_cast<double>(SizeType{1} << 30));
    return buf;
}

frost_memory_estimate at_gulp(const frost_rfi_config& rfi, frost_block_layout layout, float baseline,
                              frost_dedisp_plan_config plan, const frost_boxcar_config& search,
                              const frost_postprocess_config* post, SizeType gulp) {
    layout.max_nsamps  = gulp;
    plan.block_nsamps  = gulp;
    return estimate(rfi, layout, baseline, plan, search, post);
}

} // namespace

frost_memory_estimate estimate(const frost_rfi_config& rfi, const frost_block_layout& layout, float baseline,
                               const frost_dedisp_plan_config& plan, const frost_boxcar_config& search,
                               const frost_postprocess_config* post) {
    if (layout.max_nsamps != plan.block_nsamps)
        invalid("memory: the layout's max_nsamps and the plan's block_nsamps must be the same gulp");
    frost_memory_estimate e{};
    e.rfi_bytes                    = rfi::Cleaner::estimate_memory(rfi, layout, baseline);
    const fdmt::Engine::Footprint f = fdmt::Engine::estimate(plan, search);
    e.fdmt_bytes                   = f.level_bytes + f.history_bytes;
    e.search_bytes                 = f.table_bytes + f.candidate_bytes;
    e.postprocess_bytes            = post != nullptr ? pp::PostprocessPlan::estimate_memory(*post) : 0;
    e.transient_bytes              = f.transient_bytes;
    e.total_bytes = e.rfi_bytes + e.fdmt_bytes + e.search_bytes + e.postprocess_bytes + e.transient_bytes;
    e.max_delay   = static_cast<uint64_t>(f.dt_max);
    return e;
}

frost_memory_check check(const frost_rfi_config& rfi, frost_block_layout& layout, float baseline,
                         frost_dedisp_plan_config& plan, const frost_boxcar_config& search,
                         const frost_postprocess_config* post, bool gulp_is_default, SizeType available_bytes,
                         SizeType memory_limit_bytes, int device) {
    frost_memory_check out{};
    out.device_memory  = 1;
    out.gulp_requested = layout.max_nsamps;
    out.gulp_used      = layout.max_nsamps;
    SizeType avail     = available_bytes;
    if (avail == 0) {
        size_t free_b = 0, total_b = 0;
        int cur       = 0;
        if (cudaGetDevice(&cur) == cudaSuccess) {
            const bool other = cur != device;
            if ((!other || cudaSetDevice(device) == cudaSuccess) && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
                avail = free_b;
            if (other)
                cudaSetDevice(cur);
        }
        cudaGetLastError(); // no device: availability unknown
    }
    if (memory_limit_bytes != 0)
        avail = avail != 0 ? std::min(avail, memory_limit_bytes) : memory_limit_bytes;
    out.available_bytes = avail;
    out.estimate        = estimate(rfi, layout, baseline, plan, search, post);
    out.requested_bytes = out.estimate.total_bytes;
    if (avail == 0)
        return out; // cannot tell; do not guess
    const SizeType budget = avail - avail / 10;
    if (out.estimate.total_bytes <= budget)
        return out;
    // The smallest gulp the engine accepts exceeds max_delay + boxcar_max.
    const SizeType delay      = out.estimate.max_delay;
    const SizeType needed     = delay + search.max_boxcar + 1;
    const SizeType floor_gulp = std::max<SizeType>((needed + kGulpRounding - 1) / kGulpRounding * kGulpRounding,
                                                   kGulpRounding);
    auto fits = [&](SizeType gulp) {
        return at_gulp(rfi, layout, baseline, plan, search, post, gulp).total_bytes <= budget;
    };
    // largest multiple of kGulpRounding in [floor_gulp, requested] that fits
    SizeType lo = floor_gulp / kGulpRounding, hi = out.gulp_requested / kGulpRounding, best = 0;
    while (lo <= hi) {
        const SizeType mid = lo + (hi - lo) / 2;
        if (fits(mid * kGulpRounding)) {
            best = mid;
            lo   = mid + 1;
        } else {
            if (mid == 0)
                break;
            hi = mid - 1;
        }
    }
    const std::string what = "estimated device memory " + gib(out.estimate.total_bytes) + " for " +
                             std::to_string(layout.nchans) + " channels, max_delay " + std::to_string(delay) +
                             " and nsamps_gulp " + std::to_string(out.gulp_requested) + " exceeds the " +
                             gib(budget) + " available (90% of " + gib(avail) + ")";
    if (best == 0)
        throw Error(FROST_ERR_OUT_OF_MEMORY,
                    what + "; not even nsamps_gulp " + std::to_string(floor_gulp) + " (about max_delay " +
                        std::to_string(delay) + " + boxcar_max " + std::to_string(search.max_boxcar) +
                        ") fits. Reduce dm_max, use fewer channels, or raise the memory limit");
    const SizeType rounded = best * kGulpRounding;
    if (!gulp_is_default)
        throw Error(FROST_ERR_OUT_OF_MEMORY,
                    what + "; the largest nsamps_gulp that fits is " + std::to_string(rounded) + " (or reduce dm_max)");
    layout.max_nsamps = rounded;
    plan.block_nsamps = rounded;
    out.gulp_used     = rounded;
    out.lowered       = 1;
    out.estimate      = estimate(rfi, layout, baseline, plan, search, post);
    return out;
}

} // namespace fb::memplan
