// TEST INFRASTRUCTURE ONLY — extern "C" entry points over the reference's
// own candidate post-processing (lib/search/postprocess.cpp, clustering.cpp,
// merge.cpp, subband_dedup.cpp, rate_limiter.cpp), compiled from its sources
// by oracle/Makefile into _ref/libfrost_ref_search.so. Converts between the
// plain C records of include/frost_b200.h and frost::search::Giant /
// dmt::RawCandidate (the stand-in of oracle/stubs/dmt/common/candidate.hpp).

#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include <frost/config/config.hpp>
#include <frost/output/cand_writer.hpp>
#include <frost/search/candidate.hpp>
#include <frost/search/clustering.hpp>
#include <frost/search/merge.hpp>
#include <frost/search/postprocess.hpp>
#include <frost/search/subband_dedup.hpp>

#include "frost_b200.h"

namespace fs = frost::search;

namespace {
thread_local std::string g_error;

fs::Giant to_giant(const frost_giant& c) {
    fs::Giant g;
    g.snr             = c.snr;
    g.dm              = c.dm;
    g.samp_idx        = c.samp_idx;
    g.filter_idx      = c.filter_idx;
    g.filter_width    = c.filter_width;
    g.dm_idx          = c.dm_idx;
    g.begin           = c.begin;
    g.end             = c.end;
    g.members         = c.members;
    g.f_low           = c.f_low;
    g.f_high          = c.f_high;
    g.chan_begin      = c.chan_begin;
    g.chan_end        = c.chan_end;
    g.plane           = c.plane;
    g.snr_best        = c.snr_best;
    g.best_chan_begin = c.best_chan_begin;
    g.best_chan_end   = c.best_chan_end;
    g.n_extents       = c.n_extents;
    if (c.has_location_best != 0) {
        g.location_best = fs::CandidateLocation{c.loc_samp_idx, c.loc_dm, c.loc_filter_width,
                                                c.loc_f_low, c.loc_f_high};
    }
    return g;
}

frost_giant from_giant(const fs::Giant& g) {
    frost_giant c;
    std::memset(&c, 0, sizeof(c));
    c.snr             = g.snr;
    c.dm              = g.dm;
    c.samp_idx        = g.samp_idx;
    c.filter_idx      = g.filter_idx;
    c.filter_width    = g.filter_width;
    c.dm_idx          = g.dm_idx;
    c.begin           = g.begin;
    c.end             = g.end;
    c.members         = g.members;
    c.f_low           = g.f_low;
    c.f_high          = g.f_high;
    c.chan_begin      = g.chan_begin;
    c.chan_end        = g.chan_end;
    c.plane           = g.plane;
    c.snr_best        = g.snr_best;
    c.best_chan_begin = g.best_chan_begin;
    c.best_chan_end   = g.best_chan_end;
    c.n_extents       = g.n_extents;
    if (g.location_best.has_value()) {
        c.has_location_best = 1;
        c.loc_samp_idx      = g.location_best->samp_idx;
        c.loc_dm            = g.location_best->dm;
        c.loc_filter_width  = g.location_best->filter_width;
        c.loc_f_low         = g.location_best->f_low;
        c.loc_f_high        = g.location_best->f_high;
    }
    return c;
}

fs::ClusterTolerances to_tol(const frost_cluster_tolerances& t) {
    return fs::ClusterTolerances{t.time_tol, t.filter_tol, t.dm_tol, t.dm_smear, t.tsamp, t.snr_floor};
}

std::vector<fs::Giant> giants(const frost_giant* g, size_t n) {
    std::vector<fs::Giant> v;
    v.reserve(n);
    for (size_t i = 0; i < n; ++i)
        v.push_back(to_giant(g[i]));
    return v;
}

struct Plan {
    fs::CandidatePostprocessPlan plan;
    std::vector<fs::Giant> last;
};
} // namespace

extern "C" {

const char* refs_last_error() { return g_error.c_str(); }

void* refs_pp_create(const frost_postprocess_config* c, const frost_postprocess_layout* l) {
    try {
        frost::config::SearchConfig cfg;
        cfg.boxcar_max             = c->boxcar_max;
        cfg.max_candidates         = c->max_candidates;
        cfg.max_pending_candidates = c->max_pending_candidates;
        cfg.detect_thresh          = c->detect_thresh;
        cfg.cand_sep_time          = c->cand_sep_time;
        cfg.cand_sep_filter        = c->cand_sep_filter;
        cfg.cand_sep_dm            = c->cand_sep_dm;
        cfg.cand_sep_dm_smear      = c->cand_sep_dm_smear;
        cfg.max_giant_rate         = c->max_giant_rate;
        cfg.cluster                = c->cluster != 0;
        cfg.subband_dedup = c->subband_dedup == FROST_DEDUP_SEEDED ? fs::SubbandDedupMode::kSeeded
                                                                    : fs::SubbandDedupMode::kTransitive;
        return new Plan{fs::CandidatePostprocessPlan(cfg, {l->nchans, l->tsamp, l->frequency_step}), {}};
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    }
}

void refs_pp_destroy(void* h) { delete static_cast<Plan*>(h); }

// 0 ok, -1 invalid_argument, -2 other exception.
int refs_pp_execute(void* h, const frost_candidate* raw, size_t n, uint64_t samples_read,
                    uint64_t duration, int final_call, uint64_t frontier, uint64_t* pending) {
    auto* p = static_cast<Plan*>(h);
    std::vector<dmt::RawCandidate> rows(n);
    for (size_t i = 0; i < n; ++i) {
        auto& r         = rows[i];
        r.snr           = raw[i].snr;
        r.peak_sample   = raw[i].peak_sample;
        r.begin_sample  = raw[i].begin_sample;
        r.end_sample    = raw[i].end_sample;
        r.filter_idx    = raw[i].filter_idx;
        r.width         = raw[i].width;
        r.dm_idx        = raw[i].dm_idx;
        r.dm            = raw[i].dm;
        r.f_low_mhz     = raw[i].f_low_mhz;
        r.f_high_mhz    = raw[i].f_high_mhz;
        r.chan_begin    = raw[i].chan_begin;
        r.chan_end      = raw[i].chan_end;
        r.beam_idx      = raw[i].beam_idx;
        r.subband_level = raw[i].subband_level;
        r.subband_idx   = raw[i].subband_idx;
    }
    dmt::CandidateResultView view;
    view.candidates = rows;
    try {
        const auto res = p->plan.execute(view, samples_read, duration, final_call != 0, frontier);
        p->last.assign(res.candidates.begin(), res.candidates.end());
        *pending = res.pending_candidates;
        return 0;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        p->last.clear();
        return -1;
    } catch (const std::exception& e) {
        g_error = e.what();
        p->last.clear();
        return -2;
    }
}

size_t refs_pp_results(void* h, frost_giant* out, size_t cap) {
    auto* p = static_cast<Plan*>(h);
    for (size_t i = 0; i < p->last.size() && i < cap; ++i)
        out[i] = from_giant(p->last[i]);
    return p->last.size();
}

uint64_t refs_pp_memory_usage(void* h) { return static_cast<Plan*>(h)->plan.memory_usage(); }

void refs_cluster_labels(const frost_giant* g, size_t n, const frost_cluster_tolerances* t, int mode,
                         uint64_t* labels) {
    const auto v = giants(g, n);
    const auto l = fs::ClusterLabelPlan(mode == FROST_CLUSTER_SEEDED ? fs::ClusterMode::kSeeded
                                                                      : fs::ClusterMode::kChain)
                       .execute(v, to_tol(*t));
    for (size_t i = 0; i < n; ++i)
        labels[i] = l[i];
}

size_t refs_merge(const frost_giant* g, const uint64_t* labels, size_t n, frost_giant* out) {
    const auto v = giants(g, n);
    std::vector<frost::SizeType> l(labels, labels + n);
    const auto m = fs::MergeCandidatesPlan{}.execute(v, l);
    for (size_t i = 0; i < m.size(); ++i)
        out[i] = from_giant(m[i]);
    return m.size();
}

long refs_subband_dedup(const frost_giant* g, size_t n, const frost_cluster_tolerances* t, float tsamp,
                        int mode, frost_giant* out) {
    try {
        const auto v = giants(g, n);
        const auto m = fs::SubbandDedupPlan(mode == FROST_DEDUP_SEEDED ? fs::SubbandDedupMode::kSeeded
                                                                        : fs::SubbandDedupMode::kTransitive)
                           .execute(v, to_tol(*t), tsamp);
        for (size_t i = 0; i < m.size(); ++i)
            out[i] = from_giant(m[i]);
        return static_cast<long>(m.size());
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int refs_are_coincident(const frost_giant* a, const frost_giant* b, const frost_cluster_tolerances* t,
                        int physical) {
    const auto ga = to_giant(*a), gb = to_giant(*b);
    if (physical != 0)
        return fs::are_coincident(ga, gb, to_tol(*t)) ? 1 : 0;
    return fs::are_coincident(ga, gb, t->time_tol, t->filter_tol, t->dm_tol) ? 1 : 0;
}

double refs_time_shift(float dm, float f_wide, float f_narrow, float tsamp) {
    return fs::subband_time_shift_samples(dm, f_wide, f_narrow, tsamp);
}

double refs_dm_step(float f_low, float f_high, float tsamp) {
    return fs::subband_dm_step(f_low, f_high, tsamp);
}

// CandWriter (lib/output/cand_writer.cpp): 0 ok, -2 on an exception.
int refs_cand_write(const char* path, double dt, int append, const frost_giant* g, size_t n,
                    uint64_t first_samp_idx) {
    try {
        frost::output::CandWriter w(path, dt,
                                    append != 0 ? frost::output::CandWriter::OpenMode::kAppend
                                                : frost::output::CandWriter::OpenMode::kTruncate);
        w.write(giants(g, n), first_samp_idx);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -2;
    }
}

int refs_cand_filename(int64_t utc, uint64_t beam, char* out, size_t cap) {
    try {
        const std::string s = frost::output::cand_filename(static_cast<std::time_t>(utc), beam);
        std::snprintf(out, cap, "%s", s.c_str());
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

} // extern "C"
