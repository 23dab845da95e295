/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle of frost's candidate
 * post-processing. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it, as the checker; the product (frost_b200) never
 * links or calls it.
 *
 * A sequential restatement of:
 *   CandidatePostprocessPlan::execute   lib/search/postprocess.cpp:67-241
 *   are_coincident (both overloads)     lib/search/clustering.cpp:24-67
 *   ClusterLabelPlan::execute           lib/search/clustering.cpp:107-226
 *   MergeCandidatesPlan::execute        lib/search/merge.cpp:8-37
 *   RateLimiter                         lib/search/rate_limiter.cpp:5-30
 *   subband_time_shift_samples,
 *   subband_dm_step, on_same_curve,
 *   SubbandDedupPlan::execute           lib/search/subband_dedup.cpp:43-315
 * Pinned two ways: the known-answer cases of the reference's own tests
 * (tests/cpp/api/{clustering,clustering_boundary,merge,candidate,
 * subband_dedup,postprocess}_test.cpp, restated in
 * tests/test_postprocess_oracle.py) and the reference's sources themselves,
 * compiled into oracle/_ref/libfrost_ref_search.so by oracle/Makefile and
 * compared row for row on seeded candidate streams.
 *
 * dmt::kDispConst (dmt v0.8.0, not vendored) enters only the sub-band time
 * shift and DM step; this oracle and the stand-in header the reference build
 * uses both take 4.148808e3 s MHz^2 cm^3 / pc as a double.
 *
 * Floating-point expressions keep the reference's operation order; the
 * Makefile builds with -ffp-contract=off so none is fused.
 */

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "frost_b200.h"

#define PP_KDISP 4.148808e3

typedef uint64_t u64;

static char g_err[256];

const char* oracle_pp_last_error(void) { return g_err; }

static void set_err(const char* m) {
    strncpy(g_err, m, sizeof(g_err) - 1);
    g_err[sizeof(g_err) - 1] = 0;
}

/* ---- scalar helpers ---------------------------------------------------- */

static u64 absdiff(u64 a, u64 b) { return a > b ? a - b : b - a; }

/* giant_boxcar_width (include/frost/search/candidate.hpp:75-81). */
static u64 box_width(const frost_giant* g) {
    if (g->filter_width > 0)
        return g->filter_width;
    return (u64)1 << (g->filter_idx < 63 ? g->filter_idx : 63);
}

/* time_reach (clustering.cpp:18-21): saturates instead of wrapping. */
static u64 time_reach(u64 width, u64 tol) {
    return (tol != 0 && width > UINT64_MAX / tol) ? UINT64_MAX : width * tol;
}

static int posfin_f(float x) { return isfinite(x) && x > 0.0f; }
static int posfin_d(double x) { return isfinite(x) && x > 0.0; }
/* std::max(a, b) = (a < b) ? b : a, NaN-propagation included. */
static double max_d(double a, double b) { return (a < b) ? b : a; }
static float max_f(float a, float b) { return (a < b) ? b : a; }
static u64 max_u(u64 a, u64 b) { return (a < b) ? b : a; }

double oracle_dm_step(float f_low, float f_high, float tsamp) {
    if (!posfin_f(tsamp) || !posfin_f(f_low) || !isfinite(f_high) || !(f_high > f_low))
        return 0.0;
    const double lo    = (double)f_low;
    const double hi    = (double)f_high;
    const double denom = (1.0 / (lo * lo)) - (1.0 / (hi * hi));
    if (!posfin_d(denom))
        return 0.0;
    return (double)tsamp / (PP_KDISP * denom);
}

double oracle_time_shift(float dm, float f_wide, float f_narrow, float tsamp) {
    if (!posfin_f(tsamp) || !posfin_f(f_wide) || !posfin_f(f_narrow))
        return 0.0;
    const double w   = (double)f_wide;
    const double n   = (double)f_narrow;
    const double inv = (1.0 / (w * w)) - (1.0 / (n * n));
    return ((double)dm * PP_KDISP * inv) / (double)tsamp;
}

int oracle_coincident_basic(const frost_giant* a, const frost_giant* b, u64 time_tol, u64 filter_tol,
                            u64 dm_tol) {
    if (a->plane != b->plane || a->chan_begin != b->chan_begin || a->chan_end != b->chan_end)
        return 0;
    const u64 widest = max_u(box_width(a), box_width(b));
    return absdiff(a->samp_idx, b->samp_idx) <= time_reach(widest, time_tol) &&
           absdiff(a->filter_idx, b->filter_idx) <= filter_tol &&
           absdiff(a->dm_idx, b->dm_idx) <= dm_tol;
}

int oracle_coincident(const frost_giant* a, const frost_giant* b, const frost_cluster_tolerances* t) {
    if (!oracle_coincident_basic(a, b, t->time_tol, t->filter_tol, t->dm_tol))
        return 0;
    if (!(t->dm_smear > 0.0) || !(t->tsamp > 0.0) || absdiff(a->dm_idx, b->dm_idx) <= 1)
        return 1;
    const double step = oracle_dm_step(a->f_low, a->f_high, (float)t->tsamp);
    if (!(step > 0.0))
        return 1;
    const double widest = (double)max_u(box_width(a), box_width(b));
    const double ddm    = fabs((double)a->dm - (double)b->dm);
    double growth       = 1.0;
    if (t->snr_floor > 0.0) {
        const double ratio = (double)max_f(a->snr, b->snr) / t->snr_floor;
        growth             = max_d(1.0, sqrt(max_d(0.0, (ratio * ratio) - 1.0)));
    }
    return ddm <= t->dm_smear * widest * step * growth;
}

/* ---- stable sort of index arrays ---------------------------------------- */

typedef int (*less_fn)(u64 a, u64 b, const void* ctx);

static void msort_rec(u64* v, u64* tmp, size_t n, less_fn less, const void* ctx) {
    if (n < 2)
        return;
    const size_t h = n / 2;
    msort_rec(v, tmp, h, less, ctx);
    msort_rec(v + h, tmp, n - h, less, ctx);
    size_t i = 0, j = h, k = 0;
    while (i < h && j < n)
        tmp[k++] = less(v[j], v[i], ctx) ? v[j++] : v[i++];
    while (i < h)
        tmp[k++] = v[i++];
    while (j < n)
        tmp[k++] = v[j++];
    memcpy(v, tmp, n * sizeof(u64));
}

static void stable_sort(u64* v, size_t n, less_fn less, const void* ctx) {
    u64* tmp = (u64*)malloc((n ? n : 1) * sizeof(u64));
    msort_rec(v, tmp, n, less, ctx);
    free(tmp);
}

static int less_samp(u64 a, u64 b, const void* ctx) {
    const frost_giant* c = (const frost_giant*)ctx;
    return c[a].samp_idx < c[b].samp_idx;
}

static int greater_snr(u64 a, u64 b, const void* ctx) {
    const frost_giant* c = (const frost_giant*)ctx;
    return c[a].snr > c[b].snr;
}

static int less_label(u64 a, u64 b, const void* ctx) {
    const u64* l = (const u64*)ctx;
    return l[a] < l[b];
}

/* ---- union-find with the smaller index as root -------------------------- */

static u64 find_root(u64* parent, u64 x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x         = parent[x];
    }
    return x;
}

static void unite(u64* parent, u64 a, u64 b) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a == b)
        return;
    if (a < b)
        parent[b] = a;
    else
        parent[a] = b;
}

/* ---- ClusterLabelPlan ---------------------------------------------------- */

void oracle_cluster_labels(const frost_giant* c, size_t n, const frost_cluster_tolerances* t, int mode,
                           u64* labels) {
    for (size_t i = 0; i < n; ++i)
        labels[i] = i;
    if (n < 2)
        return;
    u64 widest = 1;
    for (size_t i = 0; i < n; ++i)
        widest = max_u(widest, box_width(&c[i]));
    const u64 reach = time_reach(widest, t->time_tol);
    u64* by_time    = (u64*)malloc(n * sizeof(u64));
    for (size_t i = 0; i < n; ++i)
        by_time[i] = i;
    stable_sort(by_time, n, less_samp, c);

    if (mode == FROST_CLUSTER_CHAIN) {
        /* Every pair within the wider giant's time reach is tested once, from
         * the wider giant (equal widths: the earlier in time order). */
        u64* parent = (u64*)malloc(n * sizeof(u64));
        for (size_t i = 0; i < n; ++i)
            parent[i] = i;
        for (size_t r = 0; r < n; ++r) {
            const frost_giant* gr = &c[by_time[r]];
            const u64 w           = box_width(gr);
            u64 reach_r           = time_reach(w, t->time_tol);
            if (reach_r > reach)
                reach_r = reach;
            for (int dir = 0; dir < 2; ++dir) {
                for (size_t step = 1;; ++step) {
                    size_t q;
                    if (dir == 0) {
                        q = r + step;
                        if (q >= n || c[by_time[q]].samp_idx - gr->samp_idx > reach_r)
                            break;
                    } else {
                        if (step > r)
                            break;
                        q = r - step;
                        if (gr->samp_idx - c[by_time[q]].samp_idx > reach_r)
                            break;
                    }
                    const frost_giant* gq = &c[by_time[q]];
                    const u64 wq          = box_width(gq);
                    if (dir == 0 ? wq > w : wq >= w)
                        continue;
                    if (absdiff(gr->dm_idx, gq->dm_idx) > t->dm_tol ||
                        absdiff(gr->filter_idx, gq->filter_idx) > t->filter_tol)
                        continue;
                    const u64 i = by_time[r], j = by_time[q];
                    if (find_root(parent, i) != find_root(parent, j) && oracle_coincident(&c[i], &c[j], t))
                        unite(parent, i, j);
                }
            }
        }
        for (size_t i = 0; i < n; ++i)
            labels[i] = find_root(parent, i);
        free(parent);
        free(by_time);
        return;
    }

    /* Seeded: brightest first (ties by index); each unassigned giant claims
     * every unassigned giant coincident with it inside the time reach. */
    u64* by_snr      = (u64*)malloc(n * sizeof(u64));
    u64* rank_of     = (u64*)malloc(n * sizeof(u64));
    uint8_t* assigned = (uint8_t*)calloc(n, 1);
    for (size_t i = 0; i < n; ++i)
        by_snr[i] = i;
    stable_sort(by_snr, n, greater_snr, c);
    for (size_t r = 0; r < n; ++r)
        rank_of[by_time[r]] = r;
    for (size_t k = 0; k < n; ++k) {
        const u64 seed = by_snr[k];
        if (assigned[seed])
            continue;
        assigned[seed]  = 1;
        labels[seed]    = seed;
        const u64 rank  = rank_of[seed];
        const u64 s0    = c[seed].samp_idx;
        for (u64 q = rank + 1; q < n && c[by_time[q]].samp_idx - s0 <= reach; ++q) {
            const u64 j = by_time[q];
            if (!assigned[j] && oracle_coincident(&c[seed], &c[j], t)) {
                assigned[j] = 1;
                labels[j]   = seed;
            }
        }
        for (u64 q = rank; q-- > 0 && s0 - c[by_time[q]].samp_idx <= reach;) {
            const u64 j = by_time[q];
            if (!assigned[j] && oracle_coincident(&c[seed], &c[j], t)) {
                assigned[j] = 1;
                labels[j]   = seed;
            }
        }
    }
    free(by_snr);
    free(rank_of);
    free(assigned);
    free(by_time);
}

/* ---- MergeCandidatesPlan -------------------------------------------------- */

size_t oracle_merge(const frost_giant* c, const u64* labels, size_t n, frost_giant* out) {
    u64* order = (u64*)malloc((n ? n : 1) * sizeof(u64));
    for (size_t i = 0; i < n; ++i)
        order[i] = i;
    stable_sort(order, n, less_label, labels);
    size_t m = 0;
    for (size_t k = 0; k < n;) {
        const u64 label = labels[order[k]];
        frost_giant best = c[order[k]];
        size_t e         = k + 1;
        for (; e < n && labels[order[e]] == label; ++e) {
            const frost_giant* g = &c[order[e]];
            const u64 sum        = best.members + g->members;
            if (g->snr > best.snr)
                best = *g;
            best.members = sum;
        }
        out[m++] = best;
        k        = e;
    }
    free(order);
    return m;
}

/* ---- sub-band dedup -------------------------------------------------------- */

static u64 span_of(const frost_giant* g) {
    return g->chan_end < g->chan_begin ? 0 : (g->chan_end - g->chan_begin) + 1;
}

static int contains(const frost_giant* o, const frost_giant* i) {
    return o->chan_begin <= i->chan_begin && o->chan_end >= i->chan_end;
}

static int dm_within_smear(const frost_giant* a, const frost_giant* b, const frost_cluster_tolerances* t,
                           double widest, double step) {
    const double smear = t->dm_smear > 0.0 ? t->dm_smear : 1.0;
    const double delay = max_d(2.0, widest);
    const double delta = fabs((double)a->dm - (double)b->dm);
    return delta <= (smear * delay * step);
}

int oracle_on_same_curve(const frost_giant* a, const frost_giant* b, const frost_cluster_tolerances* t,
                         float tsamp) {
    const u64 sa = span_of(a), sb = span_of(b);
    if (sa == 0 || sb == 0)
        return 0;
    if (sa == sb) {
        if (a->plane == b->plane || a->chan_begin != b->chan_begin || a->chan_end != b->chan_end ||
            absdiff(a->filter_idx, b->filter_idx) > t->filter_tol)
            return 0;
        const double step   = oracle_dm_step(a->f_low, a->f_high, tsamp);
        const double widest = (double)max_u(box_width(a), box_width(b));
        return posfin_d(step) && dm_within_smear(a, b, t, widest, step) &&
               (double)absdiff(a->samp_idx, b->samp_idx) <= (double)t->time_tol * widest;
    }
    if (!contains(a, b) && !contains(b, a))
        return 0;
    const frost_giant* wide   = sa > sb ? a : b;
    const frost_giant* narrow = sa > sb ? b : a;
    if (absdiff(wide->filter_idx, narrow->filter_idx) > t->filter_tol)
        return 0;
    const double step = oracle_dm_step(narrow->f_low, narrow->f_high, tsamp);
    if (!posfin_d(step))
        return 0;
    if (!dm_within_smear(wide, narrow, t, (double)max_u(box_width(wide), box_width(narrow)), step))
        return 0;
    const double wide_step = oracle_dm_step(wide->f_low, wide->f_high, tsamp);
    if (posfin_d(wide_step) && step > 4.0 * wide_step) {
        const double expected =
            (double)wide->snr * sqrt((double)(sa < sb ? sa : sb) / (double)max_u(sa, sb));
        if ((double)narrow->snr > (2.0 * expected) + 3.0)
            return 0;
    }
    const double shift   = oracle_time_shift(wide->dm, wide->f_low, narrow->f_low, tsamp);
    const double aligned = (double)narrow->samp_idx + shift;
    const double delta   = fabs(aligned - (double)wide->samp_idx);
    const double widest  = (double)max_u(box_width(wide), box_width(narrow));
    return delta <= (double)t->time_tol * widest;
}

static float best_snr(const frost_giant* g) { return g->snr_best > g->snr ? g->snr_best : g->snr; }

static int has_best_extent(const frost_giant* g) { return g->has_location_best || g->snr_best > g->snr; }

static void strongest_location(const frost_giant* g, frost_giant* dst) {
    if (g->has_location_best) {
        dst->loc_samp_idx     = g->loc_samp_idx;
        dst->loc_dm           = g->loc_dm;
        dst->loc_filter_width = g->loc_filter_width;
        dst->loc_f_low        = g->loc_f_low;
        dst->loc_f_high       = g->loc_f_high;
    } else {
        dst->loc_samp_idx     = g->samp_idx;
        dst->loc_dm           = g->dm;
        dst->loc_filter_width = box_width(g);
        dst->loc_f_low        = g->f_low;
        dst->loc_f_high       = g->f_high;
    }
}

typedef struct {
    const frost_giant* c;
} span_ctx;

static int seeded_order_less(u64 x, u64 y, const void* ctx) {
    const frost_giant* c = ((const span_ctx*)ctx)->c;
    const u64 sx = span_of(&c[x]), sy = span_of(&c[y]);
    if (sx != sy)
        return sx > sy;
    return c[x].snr > c[y].snr;
}

/* Returns the row count, or -1 (invalid tsamp). */
long oracle_subband_dedup(const frost_giant* c, size_t n, const frost_cluster_tolerances* t, float tsamp,
                          int mode, frost_giant* out) {
    if (n == 0)
        return 0;
    if (!posfin_f(tsamp)) {
        set_err("sub-band dedup requires tsamp > 0");
        return -1;
    }
    u64* group_of = (u64*)malloc(n * sizeof(u64));
    if (mode == FROST_DEDUP_TRANSITIVE) {
        u64* parent = (u64*)malloc(n * sizeof(u64));
        for (size_t i = 0; i < n; ++i)
            parent[i] = i;
        for (size_t i = 0; i < n; ++i)
            for (size_t j = i + 1; j < n; ++j)
                if (oracle_on_same_curve(&c[i], &c[j], t, tsamp))
                    unite(parent, i, j);
        for (size_t i = 0; i < n; ++i)
            group_of[i] = find_root(parent, i);
        free(parent);
    } else {
        u64* order = (u64*)malloc(n * sizeof(u64));
        for (size_t i = 0; i < n; ++i)
            order[i] = i;
        span_ctx ctx = {c};
        stable_sort(order, n, seeded_order_less, &ctx);
        for (size_t k = 0; k < n; ++k) {
            const u64 i = order[k];
            group_of[i] = i;
            for (size_t m = 0; m < k; ++m) {
                const u64 j = order[m];
                if (oracle_on_same_curve(&c[j], &c[i], t, tsamp)) {
                    group_of[i] = group_of[j];
                    break;
                }
            }
        }
        free(order);
    }
    /* Group label = lowest member index; rows come out in label order. */
    u64* first = (u64*)malloc(n * sizeof(u64));
    for (size_t i = 0; i < n; ++i)
        first[i] = n;
    for (size_t i = 0; i < n; ++i)
        if (i < first[group_of[i]])
            first[group_of[i]] = i;
    u64* label = (u64*)malloc(n * sizeof(u64));
    for (size_t i = 0; i < n; ++i)
        label[i] = first[group_of[i]];
    u64* order = (u64*)malloc(n * sizeof(u64));
    for (size_t i = 0; i < n; ++i)
        order[i] = i;
    stable_sort(order, n, less_label, label);
    long m = 0;
    for (size_t k = 0; k < n;) {
        size_t e = k + 1;
        while (e < n && label[order[e]] == label[order[k]])
            ++e;
        frost_giant winner = c[order[k]];
        frost_giant loc;
        memset(&loc, 0, sizeof(loc));
        float bsnr       = best_snr(&c[order[k]]);
        u64 bbeg         = has_best_extent(&c[order[k]]) ? c[order[k]].best_chan_begin : c[order[k]].chan_begin;
        u64 bend         = has_best_extent(&c[order[k]]) ? c[order[k]].best_chan_end : c[order[k]].chan_end;
        strongest_location(&c[order[k]], &loc);
        for (size_t q = k + 1; q < e; ++q) {
            const frost_giant* g = &c[order[q]];
            const u64 sum        = winner.members + g->members;
            const u64 sg = span_of(g), sw = span_of(&winner);
            if (sg != sw ? sg > sw : g->snr > winner.snr)
                winner = *g;
            winner.members = sum;
            const float gb = best_snr(g);
            if (gb > bsnr) {
                bsnr = gb;
                bbeg = has_best_extent(g) ? g->best_chan_begin : g->chan_begin;
                bend = has_best_extent(g) ? g->best_chan_end : g->chan_end;
                strongest_location(g, &loc);
            }
        }
        u64 n_ext = 0;
        for (size_t q = k; q < e; ++q) {
            int seen = 0;
            for (size_t p = k; p < q && !seen; ++p)
                seen = c[order[p]].chan_begin == c[order[q]].chan_begin &&
                       c[order[p]].chan_end == c[order[q]].chan_end;
            n_ext += !seen;
        }
        winner.n_extents         = n_ext;
        winner.snr_best          = bsnr;
        winner.best_chan_begin   = bbeg;
        winner.best_chan_end     = bend;
        winner.has_location_best = 1;
        winner.loc_samp_idx      = loc.loc_samp_idx;
        winner.loc_dm            = loc.loc_dm;
        winner.loc_filter_width  = loc.loc_filter_width;
        winner.loc_f_low         = loc.loc_f_low;
        winner.loc_f_high        = loc.loc_f_high;
        out[m++]                 = winner;
        k                        = e;
    }
    free(order);
    free(label);
    free(first);
    free(group_of);
    return m;
}

/* ---- CandidatePostprocessPlan ---------------------------------------------- */

typedef struct {
    frost_postprocess_config cfg;
    frost_postprocess_layout lay;
    frost_giant* pending;
    size_t npending;
    frost_giant* ready;
    size_t nready, ready_cap;
} oracle_pp;

static u64 pending_limit(const frost_postprocess_config* c) {
    return c->max_pending_candidates != 0 ? c->max_pending_candidates : c->max_candidates;
}

void* oracle_pp_create(const frost_postprocess_config* cfg, const frost_postprocess_layout* lay) {
    if (lay->nchans < 2 || !posfin_d(lay->tsamp) || !isfinite(lay->frequency_step) ||
        lay->frequency_step == 0 || cfg->boxcar_max == 0) {
        set_err("Invalid candidate post-processing layout");
        return NULL;
    }
    if (cfg->max_candidates == 0 || pending_limit(cfg) > UINT64_MAX - cfg->max_candidates) {
        set_err("Invalid candidate post-processing capacity");
        return NULL;
    }
    oracle_pp* p = (oracle_pp*)calloc(1, sizeof(oracle_pp));
    p->cfg       = *cfg;
    p->lay       = *lay;
    return p;
}

void oracle_pp_destroy(void* h) {
    oracle_pp* p = (oracle_pp*)h;
    if (!p)
        return;
    free(p->pending);
    free(p->ready);
    free(p);
}

static void push_ready(oracle_pp* p, const frost_giant* g) {
    if (p->nready == p->ready_cap) {
        p->ready_cap = p->ready_cap ? 2 * p->ready_cap : 64;
        p->ready     = (frost_giant*)realloc(p->ready, p->ready_cap * sizeof(frost_giant));
    }
    p->ready[p->nready++] = *g;
}

static int less_incoming(u64 a, u64 b, const void* ctx) {
    const frost_giant* c = (const frost_giant*)ctx;
    if (c[a].plane != c[b].plane)
        return c[a].plane < c[b].plane;
    if (c[a].dm_idx != c[b].dm_idx)
        return c[a].dm_idx < c[b].dm_idx;
    if (c[a].filter_idx != c[b].filter_idx)
        return c[a].filter_idx < c[b].filter_idx;
    return c[a].samp_idx < c[b].samp_idx;
}

static frost_cluster_tolerances pp_tol(const oracle_pp* p) {
    frost_cluster_tolerances t;
    t.time_tol   = p->cfg.cand_sep_time;
    t.filter_tol = p->cfg.cand_sep_filter;
    t.dm_tol     = p->cfg.cand_sep_dm;
    t.dm_smear   = (double)p->cfg.cand_sep_dm_smear;
    t.tsamp      = p->lay.tsamp;
    t.snr_floor  = (double)p->cfg.detect_thresh;
    return t;
}

/* reduce_plane (postprocess.cpp:188-241). Appends carried rows to *next and
 * finished winners to ready. Returns 0, or -2 on pending overflow. */
static int reduce_plane(oracle_pp* p, const frost_giant* work, size_t n, u64 watermark, int final_call,
                        frost_giant* next, size_t* nnext) {
    frost_cluster_tolerances tol = pp_tol(p);
    tol.snr_floor                = 0.0;
    u64* labels                  = (u64*)malloc(n * sizeof(u64));
    oracle_cluster_labels(work, n, &tol, FROST_CLUSTER_CHAIN, labels);
    frost_giant* merged = (frost_giant*)malloc(n * sizeof(frost_giant));
    const size_t nm     = oracle_merge(work, labels, n, merged);
    u64* merged_index   = (u64*)malloc(n * sizeof(u64));
    u64 rank            = 0;
    for (size_t i = 0; i < n; ++i)
        if (labels[i] == i)
            merged_index[i] = rank++;
    u64* groups = (u64*)malloc(nm * sizeof(u64));
    for (size_t g = 0; g < nm; ++g)
        groups[g] = g;
    const int wings = tol.dm_smear > 0.0 && nm > 1;
    frost_giant* reduced = merged;
    size_t nr            = nm;
    if (wings) {
        const frost_cluster_tolerances full = pp_tol(p);
        oracle_cluster_labels(merged, nm, &full, FROST_CLUSTER_SEEDED, groups);
        reduced = (frost_giant*)malloc(nm * sizeof(frost_giant));
        nr      = oracle_merge(merged, groups, nm, reduced);
    }
    int rc = 0;
    if (final_call) {
        for (size_t k = 0; k < nr; ++k)
            push_ready(p, &reduced[k]);
    } else {
        uint8_t* recent = (uint8_t*)calloc(nm ? nm : 1, 1);
        for (size_t i = 0; i < n; ++i)
            if (work[i].end >= watermark)
                recent[groups[merged_index[labels[i]]]] = 1;
        for (size_t i = 0; i < n && rc == 0; ++i) {
            if (!recent[groups[merged_index[labels[i]]]])
                continue;
            if (*nnext == pending_limit(&p->cfg)) {
                set_err("Pending candidate capacity exceeded; increase max_pending_candidates or reduce "
                        "candidate production");
                rc = -2;
                break;
            }
            next[(*nnext)++] = work[i];
        }
        if (rc == 0) {
            rank = 0;
            for (size_t g = 0; g < nm; ++g) {
                if (groups[g] != g)
                    continue;
                if (!recent[g])
                    push_ready(p, &reduced[rank]);
                ++rank;
            }
        }
        free(recent);
    }
    if (reduced != merged)
        free(reduced);
    free(groups);
    free(merged_index);
    free(merged);
    free(labels);
    return rc;
}

/* Kept incoming rows of one plane under the rate limiter
 * (postprocess.cpp:143-152, rate_limiter.cpp:13-24). */
static size_t rate_limited(float max_rate, double seconds, size_t n) {
    size_t count = 0;
    for (size_t i = 0; i < n; ++i) {
        int exceeded = 0;
        if (!(max_rate <= 0.0f) && !(seconds <= 0.0)) {
            const double minutes = seconds / 60.0;
            const double rate    = (double)count / minutes;
            exceeded             = rate > (double)max_rate;
        }
        if (exceeded)
            break;
        ++count;
    }
    return count;
}

/* Returns 0 (ok), -1 (invalid argument) or -2 (runtime error). */
int oracle_pp_execute(void* h, const frost_candidate* raw, size_t n, u64 samples_read, u64 duration_samples,
                      int final_call, u64 frontier, u64* pending_out) {
    oracle_pp* p = (oracle_pp*)h;
    if (n > p->cfg.max_candidates) {
        set_err("Post-processing input exceeds max_candidates");
        return -2;
    }
    p->nready        = 0;
    frost_giant* inc = (frost_giant*)calloc(n ? n : 1, sizeof(frost_giant));
    size_t ni        = 0;
    for (size_t k = 0; k < n; ++k) {
        const frost_candidate* r = &raw[k];
        if (r->peak_sample >= samples_read)
            continue;
        if (r->chan_begin >= r->chan_end || r->chan_end > p->lay.nchans) {
            set_err("Invalid raw candidate channel extent");
            free(inc);
            return -1;
        }
        if (r->beam_idx != 0 || r->width == 0 || r->width > p->cfg.boxcar_max ||
            r->begin_sample > r->peak_sample || r->end_sample < r->peak_sample) {
            set_err("Invalid raw candidate beam, width or sample interval");
            free(inc);
            return -1;
        }
        frost_giant* g  = &inc[ni++];
        g->snr          = r->snr;
        g->samp_idx     = r->peak_sample;
        g->begin        = r->begin_sample;
        g->end          = r->end_sample < samples_read - 1 ? r->end_sample : samples_read - 1;
        g->filter_idx   = r->filter_idx;
        g->filter_width = r->width;
        g->dm_idx       = r->dm_idx;
        g->dm           = r->dm;
        g->f_low        = r->f_low_mhz;
        g->f_high       = r->f_high_mhz;
        g->chan_begin   = p->lay.frequency_step < 0 ? p->lay.nchans - r->chan_end : r->chan_begin;
        g->chan_end     = p->lay.frequency_step < 0 ? p->lay.nchans - 1 - r->chan_begin : (u64)r->chan_end - 1;
        g->plane        = (u64)r->subband_level * p->lay.nchans + r->subband_idx;
        g->members      = 1;
        g->n_extents    = 1;
    }
    u64* order = (u64*)malloc((ni ? ni : 1) * sizeof(u64));
    for (size_t i = 0; i < ni; ++i)
        order[i] = i;
    stable_sort(order, ni, less_incoming, inc);

    const u64 width = p->cfg.boxcar_max;
    const u64 reach = p->cfg.cand_sep_time >= (UINT64_MAX / width) - 1 ? UINT64_MAX
                                                                       : (p->cfg.cand_sep_time + 1) * width;
    const u64 watermark = frontier > reach ? frontier - reach : 0;
    const double seconds = (double)duration_samples * p->lay.tsamp;

    const size_t cap   = ni + p->npending;
    frost_giant* next  = (frost_giant*)malloc((cap ? cap : 1) * sizeof(frost_giant));
    frost_giant* work  = (frost_giant*)malloc((cap ? cap : 1) * sizeof(frost_giant));
    size_t nnext = 0, i = 0, j = 0;
    int rc = 0;
    while (rc == 0 && (i < ni || j < p->npending)) {
        u64 plane;
        if (i == ni)
            plane = p->pending[j].plane;
        else if (j == p->npending)
            plane = inc[order[i]].plane;
        else
            plane = inc[order[i]].plane < p->pending[j].plane ? inc[order[i]].plane : p->pending[j].plane;
        size_t e = i;
        while (e < ni && inc[order[e]].plane == plane)
            ++e;
        const size_t keep = rate_limited(p->cfg.max_giant_rate, seconds, e - i);
        size_t nw         = 0;
        for (size_t k = 0; k < keep; ++k)
            work[nw++] = inc[order[i + k]];
        i = e;
        while (j < p->npending && p->pending[j].plane == plane)
            work[nw++] = p->pending[j++];
        if (p->cfg.cluster && nw > 0)
            rc = reduce_plane(p, work, nw, watermark, final_call, next, &nnext);
        else
            for (size_t k = 0; k < nw; ++k)
                push_ready(p, &work[k]);
    }
    free(work);
    free(order);
    free(inc);
    if (rc != 0) {
        free(next);
        p->nready = 0;
        return rc;
    }
    free(p->pending);
    p->pending  = next;
    p->npending = nnext;
    if (p->cfg.cluster && p->nready > 0) {
        const frost_cluster_tolerances tol = pp_tol(p);
        frost_giant* out = (frost_giant*)malloc(p->nready * sizeof(frost_giant));
        const long m     = oracle_subband_dedup(p->ready, p->nready, &tol, (float)p->lay.tsamp,
                                                p->cfg.subband_dedup, out);
        if (m < 0) {
            free(out);
            return -1;
        }
        memcpy(p->ready, out, (size_t)m * sizeof(frost_giant));
        p->nready = (size_t)m;
        free(out);
    }
    *pending_out = p->npending;
    return 0;
}

size_t oracle_pp_results(void* h, frost_giant* out, size_t cap) {
    oracle_pp* p = (oracle_pp*)h;
    const size_t m = p->nready < cap ? p->nready : cap;
    if (m)
        memcpy(out, p->ready, m * sizeof(frost_giant));
    return p->nready;
}
