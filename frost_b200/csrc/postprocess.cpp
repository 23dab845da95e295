// Host orchestration of the device post-processing passes.
//
// CandidatePostprocessPlan::execute (lib/search/postprocess.cpp:67-180) as
// a sequence of device passes on the plan's stream:
//   ingest      raw rows -> giants, validation, value ranges      (sync 1)
//   sort        incoming by (plane, dm_idx, filter_idx, samp_idx)
//   segments    plane runs of incoming + carried rows             (sync 2)
//               -> per plane: rate limiter, work = kept incoming + carried
//   chain       friends-of-friends over each plane's work rows
//   merge       one winner per chain cluster                      (sync 3)
//   wings       seeded clustering of the winners (dm_smear > 0)
//   merge       one winner per wing group                         (sync 4)
//   retention   carry every member of a group with a recent
//               excursion; the rest become ready rows            (sync 5)
//   dedup       sub-band dedup of the ready rows across planes
// Small host reads between passes size the next launches; row data never
// leaves the device until the final rows are copied out.

#include "postprocess.hpp"

#include <algorithm>
#include <bit>
#include <chrono>
#include <cstring>
#include <limits>

#include "pp_math.cuh"

namespace fb::pp {

namespace {

constexpr size_t kGiant = sizeof(frost_giant);
constexpr size_t kRunsInline = 4096;

int bit_width_of(u64 lo, u64 hi) { return hi > lo ? 64 - std::countl_zero(hi - lo) : 0; }

void d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    FB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
}
void h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    FB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}
void d2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    FB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
}
void sync(cudaStream_t s) { FB_CUDA(cudaStreamSynchronize(s)); }

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

/** Column arrays carved from one buffer (100 bytes a row + a flag). */
Columns columns_in(DeviceBuffer& b, size_t n) {
    const size_t a = (n + 63) / 64 * 64;
    b.reserve(a * 100 + 256);
    auto* base = static_cast<uint8_t*>(b.get());
    Columns c;
    c.key    = reinterpret_cast<uint4*>(base);
    c.samp   = reinterpret_cast<u64*>(c.key + a);
    c.width  = c.samp + a;
    c.dm_idx = c.width + a;
    c.filter = c.dm_idx + a;
    c.cb     = c.filter + a;
    c.ce     = c.cb + a;
    c.plane  = c.ce + a;
    c.dm     = reinterpret_cast<float*>(c.plane + a);
    c.snr    = c.dm + a;
    c.flo    = c.snr + a;
    c.fhi    = c.flo + a;
    c.idx     = reinterpret_cast<u32*>(c.fhi + a);
    c.seg     = c.idx + a;
    c.minidx  = c.seg + a;
    c.general = c.minidx + a;
    return c;
}

size_t columns_bytes(size_t n) { return (n + 63) / 64 * 64 * 100 + 256; }

/** First k in [0, n) at which the per-plane limiter reads exceeded, else n
 * (postprocess.cpp:143-152 with rate_limiter.cpp:17-24). */
size_t rate_limited(float max_rate, double seconds, size_t n) {
    if (max_rate <= 0.0F || seconds <= 0.0)
        return n;
    const double minutes = seconds / 60.0;
    auto exceeded        = [&](size_t count) {
        return static_cast<double>(count) / minutes > static_cast<double>(max_rate);
    };
    size_t lo = 0, hi = n; // first exceeded count in [lo, hi]
    while (lo < hi) {
        const size_t mid = lo + (hi - lo) / 2;
        if (exceeded(mid))
            hi = mid;
        else
            lo = mid + 1;
    }
    return lo;
}

/** Friends-of-friends labels of rows[0, n) split into segments
 * (seg_of/seg_lo/seg_hi null: one segment). */
void chain_labels(Workspace& ws, const frost_giant* rows, size_t n, const u32* seg_of, int nseg,
                  const u32* seg_lo, const u32* seg_hi, u64 samp_lo, u64 samp_hi,
                  const frost_cluster_tolerances& tol, DeviceBuffer& cols, u32* parent, u32* label,
                  cudaStream_t s) {
    if (n == 0)
        return;
    std::vector<Workspace::Field> f{{kKeySamp, samp_lo, samp_hi}};
    if (seg_of != nullptr && nseg > 1)
        f.push_back({kKeyAux32, 0, static_cast<u64>(nseg - 1)});
    const u32* tperm = ws.sort(rows, n, f, seg_of, nullptr, nullptr, s).first;
    const Columns c  = columns_in(cols, n);
    launch_columns(rows, tperm, seg_of, seg_lo, n, samp_lo, c, s);
    launch_iota(parent, n, s);
    launch_chain(c, seg_lo, seg_hi, n, tol, parent, s);
    launch_rank_labels(parent, c, n, label, s);
}

/** Seeded clustering labels of rows[0, n) by segment (segment-major rows). */
void seeded_labels(Workspace& ws, const frost_giant* rows, size_t n, const u32* seg_of, int nseg,
                   const u32* seg_lo, const u32* seg_hi, size_t max_seg_rows, u64 samp_lo, u64 samp_hi,
                   const frost_cluster_tolerances& tol, u32* tord, u32* sord, u32* rank_of,
                   DeviceBuffer& bitmap, u32* label, cudaStream_t s) {
    if (n == 0)
        return;
    std::vector<Workspace::Field> ft{{kKeySamp, samp_lo, samp_hi}};
    std::vector<Workspace::Field> fs{{kKeySnrDesc, 0, 0xFFFFFFFFull}};
    if (seg_of != nullptr && nseg > 1) {
        ft.push_back({kKeyAux32, 0, static_cast<u64>(nseg - 1)});
        fs.push_back({kKeyAux32, 0, static_cast<u64>(nseg - 1)});
    }
    d2d(tord, ws.sort(rows, n, ft, seg_of, nullptr, nullptr, s).first, n * sizeof(u32), s);
    d2d(sord, ws.sort(rows, n, fs, seg_of, nullptr, nullptr, s).first, n * sizeof(u32), s);
    launch_invert(tord, n, rank_of, s);
    const size_t words = (max_seg_rows + 31) / 32;
    if (words * sizeof(u32) > 200 * 1024)
        bitmap.reserve(words * sizeof(u32) * static_cast<size_t>(nseg));
    launch_seeded(rows, tord, sord, rank_of, seg_lo, seg_hi, nseg, tol, label, static_cast<u32*>(bitmap.get()),
                  words, s);
}

} // namespace

// ---- Workspace -----------------------------------------------------------------

void Workspace::reserve(size_t rows) {
    if (rows <= m_rows)
        return;
    const size_t tiles = rows / kTile + 2;
    for (auto& k : keys)
        k.reserve(rows * sizeof(u64));
    for (auto& p : perm)
        p.reserve(rows * sizeof(u32));
    hist.reserve(256 * tiles * sizeof(u32));
    tile_sums.reserve(tiles * sizeof(u32));
    for (DeviceBuffer* b : {&u32a, &u32b, &u32c, &u32d, &u32e, &u32f})
        b->reserve(rows * sizeof(u32));
    u64a.reserve(rows * sizeof(u64));
    u64b.reserve(rows * sizeof(u64));
    small.reserve(4096);
    host_small.reserve(4096);
    m_rows = rows;
}

SizeType Workspace::bytes() const {
    SizeType b = hist.bytes() + tile_sums.bytes() + u32a.bytes() + u32b.bytes() + u32c.bytes() + u32d.bytes() +
                 u32e.bytes() + u32f.bytes() + u64a.bytes() + u64b.bytes() + small.bytes();
    for (const auto& k : keys)
        b += k.bytes();
    for (const auto& p : perm)
        b += p.bytes();
    return b;
}

std::pair<const u32*, const u64*> Workspace::sort(const frost_giant* rows, size_t n,
                                                   const std::vector<Field>& fields, const u32* aux32,
                                                   const u64* aux64, const u32* keep, cudaStream_t s) {
    u32* p  = perm[0].as<u32>();
    u32* pa = perm[1].as<u32>();
    u64* k  = keys[0].as<u64>();
    u64* ka = keys[1].as<u64>();
    launch_iota(p, n, s);
    std::vector<std::pair<KeySpec, int>> groups;
    KeySpec cur{};
    int shift = 0;
    for (const Field& f : fields) {
        const int b = bit_width_of(f.lo, f.hi);
        if (b == 0)
            continue;
        if (shift + b > 64 || cur.n == 4) {
            groups.push_back({cur, shift});
            cur   = KeySpec{};
            shift = 0;
        }
        cur.f[cur.n++] = KeyField{f.kind, shift, f.lo};
        shift += b;
    }
    if (cur.n > 0)
        groups.push_back({cur, shift});
    if (groups.empty()) {
        if (n > 0)
            FB_CUDA(cudaMemsetAsync(k, 0, n * sizeof(u64), s));
        return {p, k};
    }
    for (const auto& [spec, bits] : groups) {
        launch_keys(rows, p, n, spec, aux32, aux64, keep, k, s);
        radix_sort(k, p, ka, pa, n, bits, hist.as<u32>(), s);
    }
    return {p, k};
}

std::vector<std::pair<u64, u64>> Workspace::ranges(const frost_giant* rows, size_t n,
                                                   const std::vector<int>& kinds, const u32* aux32,
                                                   const u64* aux64, const u32* keep, cudaStream_t s) {
    RangeKinds rk{};
    rk.n = static_cast<int>(kinds.size());
    for (int i = 0; i < rk.n; ++i)
        rk.kind[i] = kinds[static_cast<size_t>(i)];
    auto* h = host_small.as<unsigned long long>();
    for (int i = 0; i < rk.n; ++i) {
        h[2 * i]     = ~0ull;
        h[2 * i + 1] = 0ull;
    }
    h2d(small.get(), h, 2 * rk.n * sizeof(u64), s);
    launch_ranges(rows, n, rk, aux32, aux64, keep, small.as<unsigned long long>(), s);
    d2h(h, small.get(), 2 * rk.n * sizeof(u64), s);
    sync(s);
    std::vector<std::pair<u64, u64>> out;
    for (int i = 0; i < rk.n; ++i)
        out.emplace_back(h[2 * i], h[2 * i + 1]);
    return out;
}

u32 Workspace::scan(const u32* in, u32* out, size_t n, cudaStream_t s) {
    exclusive_scan(in, out, n, tile_sums.as<u32>(), small.as<u32>(), s);
    d2h(host_small.as<u32>(), small.get(), sizeof(u32), s);
    sync(s);
    return *host_small.as<u32>();
}

// ---- standalone plans ------------------------------------------------------------

void cluster_labels(Workspace& ws, const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol,
                    int mode, u32* label, cudaStream_t s) {
    if (n == 0)
        return;
    ws.reserve(n);
    const auto r = ws.ranges(rows, n, {kKeySamp}, nullptr, nullptr, nullptr, s);
    DeviceBuffer cols, extra, bitmap;
    if (mode == FROST_CLUSTER_CHAIN) {
        chain_labels(ws, rows, n, nullptr, 1, nullptr, nullptr, r[0].first, r[0].second, tol, cols,
                     ws.u32b.as<u32>(), label, s);
        sync(s);
        return;
    }
    extra.reserve(2 * sizeof(u32));
    const u32 bounds[2] = {0, static_cast<u32>(n)};
    h2d(extra.get(), bounds, sizeof(bounds), s);
    seeded_labels(ws, rows, n, nullptr, 1, extra.as<u32>(), extra.as<u32>() + 1, n, r[0].first, r[0].second, tol,
                  ws.u32c.as<u32>(), ws.u32d.as<u32>(), ws.u32e.as<u32>(), bitmap, label, s);
    sync(s);
}

size_t merge_candidates(Workspace& ws, const frost_giant* rows, const u64* labels, size_t n, frost_giant* out,
                        cudaStream_t s) {
    if (n == 0)
        return 0;
    ws.reserve(n);
    const auto r       = ws.ranges(rows, n, {kKeyAux64}, nullptr, labels, nullptr, s);
    const auto [p, k]  = ws.sort(rows, n, {{kKeyAux64, r[0].first, r[0].second}}, nullptr, labels, nullptr, s);
    u32* heads         = ws.u32a.as<u32>();
    u32* excl          = ws.u32b.as<u32>();
    u32* ordv          = ws.u32c.as<u32>();
    u32* first         = ws.u32d.as<u32>();
    auto* best         = ws.u64a.as<unsigned long long>();
    auto* sum          = ws.u64b.as<unsigned long long>();
    launch_heads(k, n, heads, s);
    const u32 ng = ws.scan(heads, excl, n, s);
    launch_scatter_ord(p, excl, heads, n, ordv, s);
    FB_CUDA(cudaMemsetAsync(first, 0xFF, ng * sizeof(u32), s));
    FB_CUDA(cudaMemsetAsync(best, 0, ng * sizeof(u64), s));
    FB_CUDA(cudaMemsetAsync(sum, 0, ng * sizeof(u64), s));
    launch_merge_accum_ord(rows, ordv, n, best, first, sum, s);
    launch_merge_emit(rows, ng, best, first, sum, nullptr, nullptr, out, s);
    return ng;
}

size_t subband_dedup(Workspace& ws, const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol,
                     float tsamp, int mode, frost_giant* out, cudaStream_t s) {
    if (n == 0)
        return 0;
    if (!posfin_f(tsamp))
        invalid("sub-band dedup requires tsamp > 0");
    ws.reserve(n);
    u32* label = ws.u32a.as<u32>();
    if (mode == FROST_DEDUP_SEEDED) {
        const auto r   = ws.ranges(rows, n, {kKeySpanDesc}, nullptr, nullptr, nullptr, s);
        u32* order     = ws.u32c.as<u32>();
        u32* fm        = ws.u32d.as<u32>();
        u32* group_of  = ws.u32e.as<u32>();
        u32* first     = ws.u32f.as<u32>();
        d2d(order,
            ws.sort(rows, n, {{kKeySnrDesc, 0, 0xFFFFFFFFull}, {kKeySpanDesc, r[0].first, r[0].second}}, nullptr,
                    nullptr, nullptr, s)
                .first,
            n * sizeof(u32), s);
        launch_first_match(rows, order, n, tol, tsamp, fm, s);
        FB_CUDA(cudaMemsetAsync(first, 0xFF, n * sizeof(u32), s));
        launch_resolve_seeded(order, fm, n, group_of, first, s);
        launch_relabel(group_of, first, n, label, s);
    } else {
        u32* parent = ws.u32b.as<u32>();
        launch_iota(parent, n, s);
        launch_dedup_pairs(rows, n, tol, tsamp, parent, s);
        launch_find_all(parent, n, label, s);
    }
    u32* flags = ws.u32b.as<u32>();
    u32* ord   = ws.u32c.as<u32>();
    launch_root_flags(label, n, flags, s);
    const u32 ng   = ws.scan(flags, ord, n, s);
    const u32* prm = ws.sort(rows, n, {{kKeyAux32, 0, static_cast<u64>(n - 1)}}, label, nullptr, nullptr, s).first;
    u32* gstart    = ws.u32d.as<u32>();
    launch_group_starts(prm, label, ord, n, gstart, s);
    launch_dedup_emit(rows, prm, gstart, ng, n, out, s);
    return ng;
}

// ---- PostprocessPlan ----------------------------------------------------------------

namespace {

u64 pending_limit_of(const frost_postprocess_config& c) {
    return c.max_pending_candidates != 0 ? c.max_pending_candidates : c.max_candidates;
}

size_t total_rows(const frost_postprocess_config& c) {
    return static_cast<size_t>(c.max_candidates + pending_limit_of(c));
}

constexpr size_t kSegsInline = 4096;

/** Counters and ranges read back after the ingest pass. */
struct Scalars {
    unsigned long long first_err;
    u32 nkept, nruns;
    unsigned long long range[8];
};

/** Device bytes the plan reserves (row buffers, columns, scratch). */
u64 plan_bytes(const frost_postprocess_config& c) {
    const u64 mc = c.max_candidates, pl = pending_limit_of(c), t = mc + pl;
    const u64 tiles = t / kTile + 2;
    u64 b           = mc * sizeof(frost_candidate) + 2 * mc * kGiant; // raw, in, inc
    b += 5 * t * kGiant;                                               // work, merged, reduced, ready, out
    b += 2 * pl * kGiant;                                              // carried rows, double-buffered
    b += columns_bytes(static_cast<size_t>(t));
    b += 13 * t * sizeof(u32) + 2 * t * sizeof(u64);                   // per-row index arrays
    b += kSegsInline * sizeof(Seg) + 2 * kSegsInline * sizeof(u32) * 2; // segments and bounds
    // workspace
    b += 2 * t * sizeof(u64) + 2 * t * sizeof(u32) + 256 * tiles * sizeof(u32) + tiles * sizeof(u32) +
         6 * t * sizeof(u32) + 2 * t * sizeof(u64) + 4096;
    return b;
}

} // namespace

PostprocessPlan::PostprocessPlan(const frost_postprocess_config& cfg, const frost_postprocess_layout& layout,
                                 int device)
    : m_cfg(cfg), m_lay(layout), m_device(device) {
    if (layout.nchans < 2 || !is_positive_finite(layout.tsamp) || !is_finite(layout.frequency_step) ||
        layout.frequency_step == 0 || cfg.boxcar_max == 0)
        invalid("Invalid candidate post-processing layout");
    const u64 pl = pending_limit_of(cfg);
    if (cfg.max_candidates == 0 || pl > std::numeric_limits<u64>::max() - cfg.max_candidates)
        invalid("Invalid candidate post-processing capacity");
    if (cfg.max_candidates + pl >= (u64{1} << 31))
        invalid("Candidate post-processing capacity exceeds 2^31 rows");
    if (cfg.subband_dedup != FROST_DEDUP_TRANSITIVE && cfg.subband_dedup != FROST_DEDUP_SEEDED)
        invalid("Invalid sub-band dedup mode");
    DeviceGuard g(device);
    FB_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
    const size_t mc = static_cast<size_t>(cfg.max_candidates);
    m_rows          = total_rows(cfg);
    const size_t t  = m_rows;
    m_raw.reserve(mc * sizeof(frost_candidate));
    m_in.reserve(mc * kGiant);
    m_inc.reserve(mc * kGiant);
    for (DeviceBuffer* b : {&m_work, &m_merged, &m_reduced, &m_ready, &m_out})
        b->reserve(t * kGiant);
    for (auto& p : m_pend)
        p.reserve(static_cast<size_t>(pl) * kGiant);
    columns_in(m_cols, t);
    for (DeviceBuffer* b : {&m_parent, &m_label, &m_ord, &m_gmap, &m_rmap, &m_flag, &m_pos, &m_first, &m_seg_of,
                            &m_mseg, &m_tord, &m_sord, &m_rank})
        b->reserve(t * sizeof(u32));
    m_best.reserve(t * sizeof(u64));
    m_sum.reserve(t * sizeof(u64));
    m_segs.reserve(kSegsInline * sizeof(Seg));
    m_bounds.reserve(2 * kSegsInline * sizeof(u32) * 2);
    m_host_segs.reserve(kSegsInline * sizeof(Seg) + 2 * kSegsInline * sizeof(u32));
    m_host_small.reserve(sizeof(Scalars) + kRunsInline * (sizeof(u64) + sizeof(u32)));
    m_ws.reserve(t);
}

PostprocessPlan::~PostprocessPlan() {
    if (m_stream != nullptr) {
        cudaStreamSynchronize(m_stream);
        cudaStreamDestroy(m_stream);
    }
}

u64 PostprocessPlan::pending_limit() const { return pending_limit_of(m_cfg); }

frost_cluster_tolerances PostprocessPlan::tolerances() const {
    return frost_cluster_tolerances{m_cfg.cand_sep_time,
                                    m_cfg.cand_sep_filter,
                                    m_cfg.cand_sep_dm,
                                    static_cast<double>(m_cfg.cand_sep_dm_smear),
                                    m_lay.tsamp,
                                    static_cast<double>(m_cfg.detect_thresh)};
}

u64 PostprocessPlan::memory_usage() const {
    u64 b = m_raw.bytes() + m_in.bytes() + m_inc.bytes() + m_work.bytes() + m_merged.bytes() + m_reduced.bytes() +
            m_ready.bytes() + m_out.bytes() + m_pend[0].bytes() + m_pend[1].bytes() + m_segs.bytes() +
            m_cols.bytes() + m_parent.bytes() + m_label.bytes() + m_ord.bytes() + m_gmap.bytes() + m_rmap.bytes() +
            m_flag.bytes() + m_pos.bytes() + m_first.bytes() + m_best.bytes() + m_sum.bytes() + m_seg_of.bytes() +
            m_mseg.bytes() + m_tord.bytes() + m_sord.bytes() + m_rank.bytes() + m_bounds.bytes() +
            m_bitmap.bytes();
    return b + m_ws.bytes();
}

u64 PostprocessPlan::estimate_memory(const frost_postprocess_config& cfg) { return plan_bytes(cfg); }

frost_postprocess_result PostprocessPlan::execute(const frost_candidate* cands, size_t n, bool on_device,
                                                  u64 samples_read, u64 duration_samples, bool final_call,
                                                  u64 candidate_frontier) {
    if (n > m_cfg.max_candidates)
        throw Error(FROST_ERR_OVERFLOW, "Post-processing input exceeds max_candidates");
    DeviceGuard g(m_device);
    const cudaStream_t s = m_stream;
    m_results.clear();
    frost_postprocess_result res{};
    const u64 launches0 = launch_counter();

    // ---- ingest ------------------------------------------------------------
    const frost_candidate* raw = cands;
    if (!on_device && n > 0) {
        h2d(m_raw.get(), cands, n * sizeof(frost_candidate), s);
        raw = m_raw.as<frost_candidate>();
    }
    auto* hs = m_host_small.as<Scalars>();
    std::memset(hs, 0, sizeof(Scalars));
    hs->first_err = ~0ull;
    for (int k = 0; k < 4; ++k) {
        hs->range[2 * k]     = ~0ull;
        hs->range[2 * k + 1] = 0;
    }
    auto* ds = m_ws.small.as<Scalars>();
    h2d(ds, hs, sizeof(Scalars), s);
    frost_giant* in = m_in.as<frost_giant>();
    u32* keep       = m_flag.as<u32>();
    launch_ingest(raw, n, samples_read, m_lay.nchans, m_lay.frequency_step < 0 ? 1 : 0, m_cfg.boxcar_max, in,
                  keep, &ds->first_err, &ds->nkept, s);
    RangeKinds rk{4, {kKeySamp, kKeyFilter, kKeyDmIdx, kKeyPlane}};
    launch_ranges(in, n, rk, nullptr, nullptr, keep, ds->range, s);
    d2h(hs, ds, sizeof(Scalars), s);
    sync(s);
    if (hs->first_err != ~0ull) {
        if ((hs->first_err & 1ull) == 0)
            invalid("Invalid raw candidate channel extent");
        invalid("Invalid raw candidate beam, width or sample interval");
    }
    const size_t ni = hs->nkept;
    u64 rng[4][2];
    for (int k = 0; k < 4; ++k) {
        rng[k][0] = hs->range[2 * k];
        rng[k][1] = hs->range[2 * k + 1];
    }

    // ---- incoming order and plane runs -----------------------------------------
    frost_giant* inc = m_inc.as<frost_giant>();
    if (n > 0) {
        const u32* perm = m_ws.sort(in, n,
                                    {{kKeySamp, rng[0][0], rng[0][1]},
                                     {kKeyFilter, rng[1][0], rng[1][1]},
                                     {kKeyDmIdx, rng[2][0], rng[2][1]},
                                     {kKeyPlane, rng[3][0], rng[3][1]},
                                     {kKeyDropped, 0, ni < n ? 1ull : 0ull}},
                                    nullptr, nullptr, keep, s)
                              .first;
        launch_gather(in, perm, ni, inc, s);
    }
    std::vector<std::pair<u64, u32>> in_runs; // (plane, start)
    if (ni > 0) {
        u64* run_plane = m_ws.u64a.as<u64>();
        u32* run_start = m_ws.u32a.as<u32>();
        FB_CUDA(cudaMemsetAsync(&ds->nruns, 0, sizeof(u32), s));
        launch_plane_runs(inc, ni, run_plane, run_start, &ds->nruns, s);
        auto* hp          = reinterpret_cast<u64*>(hs + 1);
        auto* hq          = reinterpret_cast<u32*>(hp + kRunsInline);
        const size_t head = std::min(ni, kRunsInline);
        d2h(&hs->nruns, &ds->nruns, sizeof(u32), s);
        d2h(hp, run_plane, head * sizeof(u64), s);
        d2h(hq, run_start, head * sizeof(u32), s);
        sync(s);
        const size_t nr = hs->nruns;
        std::vector<u64> planes(nr);
        std::vector<u32> starts(nr);
        if (nr <= kRunsInline) {
            std::copy(hp, hp + nr, planes.begin());
            std::copy(hq, hq + nr, starts.begin());
        } else {
            FB_CUDA(cudaMemcpy(planes.data(), run_plane, nr * sizeof(u64), cudaMemcpyDeviceToHost));
            FB_CUDA(cudaMemcpy(starts.data(), run_start, nr * sizeof(u32), cudaMemcpyDeviceToHost));
        }
        for (size_t k = 0; k < nr; ++k)
            in_runs.emplace_back(planes[k], starts[k]);
        std::sort(in_runs.begin(), in_runs.end(), [](const auto& a, const auto& b) { return a.second < b.second; });
    }

    // ---- segments: one per plane, incoming rows rate-limited, then carried rows ----
    const double seconds = static_cast<double>(duration_samples) * m_lay.tsamp;
    std::vector<Seg> segs;
    std::vector<u32> seg_lo, seg_hi;
    {
        size_t i = 0, j = 0;
        u32 in_pos = 0, pend_pos = 0, work_pos = 0;
        while (i < in_runs.size() || j < m_pend_runs.size()) {
            u64 plane;
            if (i == in_runs.size())
                plane = m_pend_runs[j].first;
            else if (j == m_pend_runs.size())
                plane = in_runs[i].first;
            else
                plane = std::min(in_runs[i].first, m_pend_runs[j].first);
            Seg sg{};
            sg.plane    = plane;
            sg.in_start = in_pos;
            if (i < in_runs.size() && in_runs[i].first == plane) {
                const u32 end = i + 1 < in_runs.size() ? in_runs[i + 1].second : static_cast<u32>(ni);
                const u32 cnt = end - in_runs[i].second;
                sg.in_start   = in_runs[i].second;
                sg.in_keep    = static_cast<u32>(rate_limited(m_cfg.max_giant_rate, seconds, cnt));
                in_pos        = end;
                ++i;
            }
            sg.pend_start = pend_pos;
            if (j < m_pend_runs.size() && m_pend_runs[j].first == plane) {
                sg.pend_cnt = m_pend_runs[j].second;
                pend_pos += sg.pend_cnt;
                ++j;
            }
            sg.work_start = work_pos;
            sg.work_cnt   = sg.in_keep + sg.pend_cnt;
            work_pos += sg.work_cnt;
            segs.push_back(sg);
            seg_lo.push_back(sg.work_start);
            seg_hi.push_back(sg.work_start + sg.work_cnt);
        }
    }
    const int nseg     = static_cast<int>(segs.size());
    size_t nwork       = 0;
    size_t max_seg     = 0;
    for (const Seg& sg : segs) {
        nwork += sg.work_cnt;
        max_seg = std::max<size_t>(max_seg, sg.work_cnt);
    }
    const u64 bw        = m_cfg.boxcar_max;
    const u64 maxv      = std::numeric_limits<u64>::max();
    const u64 reach     = m_cfg.cand_sep_time >= (maxv / bw) - 1 ? maxv : (m_cfg.cand_sep_time + 1) * bw;
    const u64 watermark = candidate_frontier > reach ? candidate_frontier - reach : 0;
    const auto t_cluster = std::chrono::steady_clock::now();

    if (static_cast<size_t>(nseg) > kSegsInline) {
        m_segs.reserve(nseg * sizeof(Seg));
        m_bounds.reserve(4 * nseg * sizeof(u32));
        m_host_segs.reserve(nseg * sizeof(Seg) + 2 * nseg * sizeof(u32));
    }
    frost_giant* work = m_work.as<frost_giant>();
    u32* seg_of       = m_seg_of.as<u32>();
    u32* d_lo         = m_bounds.as<u32>();
    u32* d_hi         = d_lo + std::max<size_t>(nseg, 1);
    if (nwork > 0) {
        std::memcpy(m_host_segs.as<uint8_t>(), segs.data(), nseg * sizeof(Seg));
        h2d(m_segs.get(), m_host_segs.as<uint8_t>(), nseg * sizeof(Seg), s);
        auto* hb = reinterpret_cast<u32*>(m_host_segs.as<uint8_t>() + nseg * sizeof(Seg));
        std::copy(seg_lo.begin(), seg_lo.end(), hb);
        std::copy(seg_hi.begin(), seg_hi.end(), hb + nseg);
        h2d(d_lo, hb, nseg * sizeof(u32), s);
        h2d(d_hi, hb + nseg, nseg * sizeof(u32), s);
        launch_build_work(inc, m_pend[m_cur].as<frost_giant>(), m_segs.as<Seg>(), nseg, nwork, work, seg_of, s);
    }

    if (!m_cfg.cluster || nwork == 0) {
        // No clustering: every kept row is a result; nothing is carried.
        m_results.resize(nwork);
        if (nwork > 0) {
            d2h(m_results.data(), work, nwork * kGiant, s);
            sync(s);
        }
        m_npending = 0;
        m_pend_runs.clear();
        m_pend_samp_lo = ~u64{0};
        m_pend_samp_hi = 0;
        res.count      = m_results.size();
        res.launches   = launch_counter() - launches0;
        return res;
    }

    // ---- friends-of-friends within each plane ------------------------------------
    const frost_cluster_tolerances tol_full = tolerances();
    frost_cluster_tolerances tol_chain      = tol_full;
    tol_chain.snr_floor                     = 0.0;
    const u64 samp_lo = std::min(rng[0][0], m_pend_samp_lo);
    const u64 samp_hi = std::max(ni > 0 ? rng[0][1] : 0, m_npending > 0 ? m_pend_samp_hi : 0);
    u32* label        = m_label.as<u32>();
    chain_labels(m_ws, work, nwork, seg_of, nseg, d_lo, d_hi, samp_lo, samp_hi, tol_chain, m_cols,
                 m_parent.as<u32>(), label, s);

    // ---- merge per chain cluster ---------------------------------------------------
    u32* flag = m_flag.as<u32>();
    u32* ord  = m_ord.as<u32>();
    u32* gmap = m_gmap.as<u32>();
    auto* best = m_best.as<unsigned long long>();
    auto* sum  = m_sum.as<unsigned long long>();
    u32* first = m_first.as<u32>();
    launch_root_flags(label, nwork, flag, s);
    const size_t nm = m_ws.scan(flag, ord, nwork, s);
    FB_CUDA(cudaMemsetAsync(first, 0xFF, nm * sizeof(u32), s));
    FB_CUDA(cudaMemsetAsync(best, 0, nm * sizeof(u64), s));
    FB_CUDA(cudaMemsetAsync(sum, 0, nm * sizeof(u64), s));
    launch_merge_accum(work, label, ord, nwork, best, first, sum, gmap, s);
    frost_giant* merged = m_merged.as<frost_giant>();
    u32* mseg           = m_mseg.as<u32>();
    launch_merge_emit(work, nm, best, first, sum, seg_of, mseg, merged, s);

    // ---- DM wings: seeded clustering of the winners ----------------------------------
    const frost_giant* reduced = merged;
    size_t nr                  = nm;
    const u32* rmap            = nullptr;
    if (tol_full.dm_smear > 0.0 && nm > 1) {
        u32* lo2 = d_lo + 2 * std::max<size_t>(nseg, 1);
        u32* hi2 = lo2 + std::max<size_t>(nseg, 1);
        FB_CUDA(cudaMemsetAsync(lo2, 0xFF, nseg * sizeof(u32), s));
        FB_CUDA(cudaMemsetAsync(hi2, 0, nseg * sizeof(u32), s));
        launch_seg_bounds(mseg, nm, lo2, hi2, s);
        u32* glabel = m_parent.as<u32>(); // the chain's parents are no longer needed
        seeded_labels(m_ws, merged, nm, mseg, nseg, lo2, hi2, max_seg, samp_lo, samp_hi, tol_full,
                      m_tord.as<u32>(), m_sord.as<u32>(), m_rank.as<u32>(), m_bitmap, glabel, s);
        u32* ord2 = m_pos.as<u32>();
        launch_root_flags(glabel, nm, flag, s);
        nr = m_ws.scan(flag, ord2, nm, s);
        FB_CUDA(cudaMemsetAsync(first, 0xFF, nr * sizeof(u32), s));
        FB_CUDA(cudaMemsetAsync(best, 0, nr * sizeof(u64), s));
        FB_CUDA(cudaMemsetAsync(sum, 0, nr * sizeof(u64), s));
        u32* r_of_m = m_rmap.as<u32>();
        launch_merge_accum(merged, glabel, ord2, nm, best, first, sum, r_of_m, s);
        launch_merge_emit(merged, nr, best, first, sum, nullptr, nullptr, m_reduced.as<frost_giant>(), s);
        reduced = m_reduced.as<frost_giant>();
        rmap    = r_of_m;
    }

    // ---- retention: carry groups with a recent excursion -------------------------------
    frost_giant* ready = m_ready.as<frost_giant>();
    size_t nready      = 0;
    if (final_call) {
        d2d(ready, reduced, nr * kGiant, s);
        nready = nr;
        m_npending = 0;
        m_pend_runs.clear();
        m_pend_samp_lo = ~u64{0};
        m_pend_samp_hi = 0;
    } else {
        u32* recent = m_ws.u32f.as<u32>();
        FB_CUDA(cudaMemsetAsync(recent, 0, nr * sizeof(u32), s));
        launch_recent(work, nwork, gmap, rmap, watermark, recent, s);
        u32* pflag = m_flag.as<u32>();
        u32* ppos  = m_pos.as<u32>();
        launch_pending_flags(nwork, gmap, rmap, recent, 0, pflag, s);
        const size_t np = m_ws.scan(pflag, ppos, nwork, s);
        if (np > pending_limit())
            throw Error(FROST_ERR_OVERFLOW, "Pending candidate capacity exceeded; increase "
                                            "max_pending_candidates or reduce candidate production");
        const int nxt = 1 - m_cur;
        launch_compact(work, pflag, ppos, nwork, m_pend[nxt].as<frost_giant>(), s);
        // Carried rows per plane and their sample range, for the next call.
        u32* counts = m_ws.u32e.as<u32>();
        FB_CUDA(cudaMemsetAsync(counts, 0, nseg * sizeof(u32), s));
        launch_seg_counts(pflag, seg_of, nwork, counts, s);
        std::vector<u32> pc(nseg);
        d2h(pc.data(), counts, nseg * sizeof(u32), s);
        const auto pr = m_ws.ranges(work, nwork, {kKeySamp}, nullptr, nullptr, pflag, s); // synchronises
        m_pend_runs.clear();
        for (int k = 0; k < nseg; ++k)
            if (pc[k] > 0)
                m_pend_runs.emplace_back(segs[k].plane, pc[k]);
        m_pend_samp_lo = pr[0].first;
        m_pend_samp_hi = pr[0].second;
        m_npending     = np;
        m_cur          = nxt;
        u32* rflag = m_ws.u32e.as<u32>();
        u32* rpos  = m_ws.u32d.as<u32>();
        launch_ready_flags(nr, recent, 0, rflag, s);
        nready = m_ws.scan(rflag, rpos, nr, s);
        launch_compact(reduced, rflag, rpos, nr, ready, s);
    }
    sync(s);
    res.cluster_s = seconds_since(t_cluster);

    // ---- sub-band dedup across planes --------------------------------------------------
    const auto t_dedup = std::chrono::steady_clock::now();
    const size_t nout  = subband_dedup(m_ws, ready, nready, tol_full, static_cast<float>(m_lay.tsamp),
                                       m_cfg.subband_dedup, m_out.as<frost_giant>(), s);
    m_results.resize(nout);
    if (nout > 0)
        d2h(m_results.data(), m_out.get(), nout * kGiant, s);
    sync(s);
    res.dedup_s            = seconds_since(t_dedup);
    res.count              = nout;
    res.pending_candidates = m_npending;
    res.launches           = launch_counter() - launches0;
    return res;
}

} // namespace fb::pp
