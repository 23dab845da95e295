// Drives the C++20 wrapper (include/frost_b200.hpp) the way a frost host
// program would. Modes:
//   wrapper_test cpu
//       host-only calls: DM list, validation errors as std::invalid_argument
//   wrapper_test gpu <block.bin> <nchans> <gulp> <ngulps> <out.bin>
//       uint8 gulps through GulpPipeline (default RFI, DM 0-80, depth 1,
//       boxcar 1..32, threshold 7); writes every frost_candidate in order,
//       the flush's included.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "frost_b200.hpp"

namespace fb = frost::b200;

static frost_dedisp_plan_config plan_for(uint64_t nchans, uint64_t gulp, double tsamp, double f0,
                                         double df, float dm_max, uint64_t depth) {
    frost_dedisp_plan_config p{};
    p.nchans         = nchans;
    p.dt             = static_cast<float>(tsamp);
    p.f0             = static_cast<float>(f0);
    p.df             = static_cast<float>(df);
    p.dm_min         = 0.0F;
    p.dm_max         = dm_max;
    p.dm_pulse_width = 40.0F;
    p.dm_tol         = 1.25F;
    p.dm_dtype       = FROST_FLOAT32;
    p.block_nsamps   = gulp;
    p.subband_depth  = depth;
    return p;
}

static int cpu_mode() {
    const auto p    = plan_for(1024, 65536, 64e-6, 1500.0, -0.29296875, 500.0F, 0);
    const auto dms  = fb::generate_dm_list(p);
    std::cout << "ndm " << dms.size() << " first " << dms.front() << " last " << dms.back() << "\n";
    auto bad   = p;
    bad.dm_tol = 1.0F; // generate_dm_list requires dm_tol > 1
    try {
        (void)fb::generate_dm_list(bad);
        std::cout << "no-throw\n";
        return 1;
    } catch (const std::invalid_argument& e) {
        std::cout << "invalid_argument\n";
    }
    auto cfg                  = fb::default_rfi_config();
    cfg.narrow_threshold      = -1.0F;
    if (frost_rfi_config_validate(&cfg) != FROST_ERR_INVALID_ARGUMENT) {
        std::cout << "validate accepted a bad config\n";
        return 1;
    }
    // post-processing host helpers (candidate_test.cpp:14-30)
    frost_giant a{}, b{};
    a.samp_idx = 1000, a.filter_idx = 3, a.dm_idx = 10, a.members = b.members = 1;
    b            = a;
    b.samp_idx   = 1040;
    const bool in = fb::are_coincident(a, b, 5, 1, 2);
    b.samp_idx    = 1048;
    const bool out = fb::are_coincident(a, b, 5, 1, 2);
    if (!in || out) {
        std::cout << "are_coincident wrong\n";
        return 1;
    }
    if (!(fb::subband_dm_step(1000.0F, 1256.0F, 0.001F) > 0.0) ||
        !(fb::subband_time_shift_samples(100.0F, 1000.0F, 1100.0F, 0.001F) > 13.0)) {
        std::cout << "dispersion helpers wrong\n";
        return 1;
    }
    const auto ppc = fb::default_postprocess_config();
    if (fb::CandidatePostprocessPlan::estimate_memory(ppc) == 0) {
        std::cout << "estimate_memory zero\n";
        return 1;
    }
    try {
        frost_postprocess_layout bad_layout{8, 0.0, 1.0};
        fb::CandidatePostprocessPlan plan(ppc, bad_layout);
        std::cout << "bad layout accepted\n";
        return 1;
    } catch (const std::invalid_argument&) {
        std::cout << "postprocess invalid_argument\n";
    }
    // memory planning: a beam that needs more than 90 % of the budget has
    // its default gulp lowered to a multiple of 1024 samples that fits
    {
        frost_block_layout lay{1024, 65536, FROST_UINT8, 64e-6, 1500.0, -0.29296875};
        auto dd = plan_for(1024, 65536, 64e-6, 1500.0, -0.29296875, 500.0F, 1);
        frost_boxcar_config sc{};
        sc.max_boxcar = 64, sc.wtsp = 2.0F, sc.detect_thresh = 6.0F, sc.noise_sigma = 1.0F;
        sc.peak_mode = FROST_PEAK_PER_WIDTH, sc.max_candidates = 1 << 16, sc.skip_cold_prefix = 1;
        sc.input_nbits = 32, sc.storage = FROST_STORAGE_FP16;
        const auto rc = fb::default_rfi_config();
        const auto e  = fb::estimate_memory(rc, lay, 1.0F, dd, sc);
        const auto c  = fb::check_memory(rc, lay, 1.0F, dd, sc, true, e.total_bytes / 2);
        if (!c.lowered || c.gulp_used % 1024 != 0 || lay.max_nsamps != c.gulp_used || dd.block_nsamps != c.gulp_used ||
            c.estimate.total_bytes > e.total_bytes / 2 - e.total_bytes / 20) {
            std::cout << "check_memory wrong\n";
            return 1;
        }
        std::cout << "memory lowered " << c.gulp_used << "\n";
    }
    std::cout << "ok\n";
    return 0;
}

static int gpu_mode(char** argv) {
    const std::string in = argv[2];
    const uint64_t nchans = std::stoull(argv[3]), gulp = std::stoull(argv[4]);
    const int ngulps = std::stoi(argv[5]);
    std::ifstream f(in, std::ios::binary);
    std::vector<uint8_t> data(nchans * gulp * ngulps);
    f.read(reinterpret_cast<char*>(data.data()), static_cast<std::streamsize>(data.size()));
    if (!f)
        return 2;
    frost_block_layout lay{nchans, gulp, FROST_UINT8, 1e-3, 1500.0, -1.0};
    const auto plan = plan_for(nchans, gulp, 1e-3, 1500.0, -1.0, 80.0F, 1);
    frost_boxcar_config bc{};
    bc.max_boxcar       = 32;
    bc.wtsp             = 2.0F;
    bc.use_trapezoid    = 0;
    bc.detect_thresh    = 7.0F;
    bc.noise_sigma      = 1.0F;
    bc.peak_mode        = FROST_PEAK_PER_WIDTH;
    bc.max_candidates   = 1 << 16;
    bc.max_cands_per_dm = 0;
    bc.skip_cold_prefix = 1;
    bc.input_nbits      = 32;
    bc.input_mean       = 0.0F;
    bc.storage          = FROST_STORAGE_FP32;
    bc.tile_nsamps      = 0;
    fb::GulpPipeline pipe(fb::default_rfi_config(), lay, 1.0F, plan, bc);
    std::vector<frost_candidate> all;
    for (int g = 0; g < ngulps; ++g) {
        const std::span<const uint8_t> block(data.data() + g * nchans * gulp, nchans * gulp);
        auto r = pipe.execute(block, gulp);
        all.insert(all.end(), r.candidates.begin(), r.candidates.end());
    }
    auto r = pipe.flush();
    all.insert(all.end(), r.candidates.begin(), r.candidates.end());
    std::ofstream o(argv[6], std::ios::binary);
    o.write(reinterpret_cast<const char*>(all.data()),
            static_cast<std::streamsize>(all.size() * sizeof(frost_candidate)));
    std::cout << "candidates " << all.size() << " searched " << pipe.nsamps_processed() << "\n";
    return 0;
}

int main(int argc, char** argv) {
    try {
        if (argc >= 2 && std::strcmp(argv[1], "cpu") == 0)
            return cpu_mode();
        if (argc >= 7 && std::strcmp(argv[1], "gpu") == 0)
            return gpu_mode(argv);
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 3;
    }
    std::cerr << "usage: wrapper_test cpu | gpu <block.bin> <nchans> <gulp> <ngulps> <out.bin>\n";
    return 2;
}
