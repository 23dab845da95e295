// Search engine orchestration (see search_engine.hpp).

#include "search_engine.hpp"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "dedisp.hpp"
#include "postprocess_kernels.hpp"

namespace fb::fdmt {

namespace {

template <class T> void upload(DeviceBuffer& b, const std::vector<T>& v, cudaStream_t s) {
    b.reserve(std::max<SizeType>(v.size() * sizeof(T), 16));
    if (!v.empty())
        FB_CUDA(cudaMemcpyAsync(b.get(), v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Bits that hold every value 0..v.
int bits_of(uint64_t v) {
    int b = 0;
    while (v != 0) {
        ++b;
        v >>= 1;
    }
    return b;
}

// Rows of level h that no plane searches (ascending): with the single
// level step into h fused with the search, the level kernel computes only
// these.
std::vector<int32_t> unsearched_rows(const Plan& plan, int h) {
    std::vector<char> searched(static_cast<size_t>(plan.level_rows(h)), 0);
    for (const auto& p : plan.planes())
        if (p.height == h)
            for (const auto r : p.level_row)
                searched[static_cast<size_t>(r)] = 1;
    std::vector<int32_t> out;
    for (size_t r = 0; r < searched.size(); ++r)
        if (searched[r] == 0)
            out.push_back(static_cast<int32_t>(r));
    return out;
}

// Digit histograms of the candidate radix sort for up to n keys.
SizeType sort_hist_bytes(SizeType n) { return 256 * ((n + pp::kTile - 1) / pp::kTile) * sizeof(uint32_t); }

PlanConfig plan_config(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc) {
    float f_min = 0, f_max = 0;
    dedisp::band_edges(dd, f_min, f_max);
    if (dd.block_nsamps == 0)
        invalid("search: block_nsamps must be > 0");
    PlanConfig pc;
    pc.nchans        = dd.nchans;
    pc.f_min         = f_min;
    pc.f_max         = f_max;
    pc.tsamp         = dd.dt;
    pc.block_nsamps  = dd.block_nsamps;
    pc.subband_depth = dd.subband_depth;
    pc.max_boxcar    = bc.max_boxcar;
    pc.wtsp          = bc.wtsp;
    pc.dm_list       = dedisp::generate_dm_list(dd);
    return pc;
}

} // namespace

Engine::Engine(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc,
               const uint8_t* kill_mask, SizeType memory_budget, int device)
    : m_plan(plan_config(dd, bc)), m_cfg(bc), m_device(device),
      m_fp16(bc.storage == FROST_STORAGE_FP16) {
    validate(dd, bc, m_plan);
    int ndev = 0;
    FB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        invalid("search: device " + std::to_string(device) + " does not exist");
    DeviceGuard g(device);
    FB_CUDA(cudaDeviceGetAttribute(&m_sms, cudaDevAttrMultiProcessorCount, device));
    FB_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
    FB_CUDA(cudaEventCreateWithFlags(&m_order, cudaEventDisableTiming));
    cudaStream_t s = m_stream;

    const int32_t C = m_plan.nchans();
    m_mask.assign(C, 1U);
    if (kill_mask != nullptr)
        for (int32_t c = 0; c < C; ++c)
            m_mask[c] = kill_mask[c] != 0 ? 1 : 0;
    m_kill = m_mask;

    // Level ops.
    const int L = m_plan.levels();
    std::vector<int32_t> first;
    {
        const auto& ops = m_plan.leaf_ops();
        // nodes of height 1 own contiguous op ranges with one channel pair
        first.push_back(0);
        for (size_t i = 1; i < ops.size(); ++i)
            if (ops[i].chan_lo != ops[i - 1].chan_lo || ops[i].chan_hi != ops[i - 1].chan_hi)
                first.push_back(static_cast<int32_t>(i));
        first.push_back(static_cast<int32_t>(ops.size()));
        m_node_first_op = first;
        upload(m_leaf_ops, ops, s);
        upload(m_node_first_op_d, first, s);
    }
    std::vector<RowOp> all_ops;
    m_row_op_offset.assign(L + 2, 0);
    for (int h = 2; h <= L; ++h) {
        m_row_op_offset[h] = static_cast<int64_t>(all_ops.size());
        const auto& ops    = m_plan.row_ops(h);
        all_ops.insert(all_ops.end(), ops.begin(), ops.end());
    }
    upload(m_row_ops, all_ops, s);

    build_schedule(true);

    // Searched rows, grouped by height.
    const auto& planes = m_plan.planes();
    std::vector<int32_t> order(planes.size());
    for (size_t i = 0; i < order.size(); ++i)
        order[i] = static_cast<int32_t>(i);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return planes[a].height < planes[b].height; });
    std::vector<SearchRow> rows;
    std::vector<PlaneInfo> pinfo(planes.size());
    std::vector<uint16_t> leaf;
    std::vector<int64_t> leaf_off;
    std::vector<int64_t> cap_rows;
    m_height_g0.assign(L + 1, 0);
    m_height_g1.assign(L + 1, 0);
    for (size_t i = 0; i < planes.size(); ++i) {
        const Plane& p = planes[i];
        pinfo[i]       = {static_cast<float>(p.f_lo), static_cast<float>(p.f_hi),
                          static_cast<uint32_t>(p.chan_begin), static_cast<uint32_t>(p.chan_end),
                          static_cast<uint32_t>(p.subband_level), static_cast<uint32_t>(p.subband_idx)};
    }
    int cur_h = -1;
    for (const int32_t pi : order) {
        const Plane& p = planes[pi];
        if (p.height != cur_h) {
            cur_h                = p.height;
            m_height_g0[cur_h]   = static_cast<int64_t>(rows.size());
        }
        const auto len    = m_plan.leaf_lengths(pi);
        const int32_t nch = p.chan_end - p.chan_begin;
        for (size_t r = 0; r < p.delay.size(); ++r) {
            rows.push_back({p.level_row[r], pi, static_cast<int32_t>(r), p.delay[r], p.dm[r]});
            leaf_off.push_back(static_cast<int64_t>(leaf.size()));
            leaf.insert(leaf.end(), len.begin() + r * nch, len.begin() + (r + 1) * nch);
        }
        m_height_g1[cur_h] = static_cast<int64_t>(rows.size());
    }
    m_nsearch = rows.size();
    upload(m_rows, rows, s);
    upload(m_planes, pinfo, s);
    upload(m_leaf_len, leaf, s);
    upload(m_leaf_offset, leaf_off, s);
    upload(m_widths, m_plan.widths(), s);

    // Single level steps fused with the search: the op of every searched
    // row's level row, and per searched height the rows no plane searches.
    {
        std::vector<RowOp> fs_ops(m_nsearch, RowOp{0, -1, 0, 0});
        for (SizeType g = 0; g < m_nsearch; ++g) {
            const int h = planes[static_cast<size_t>(rows[g].plane)].height;
            if (h >= 2)
                fs_ops[g] = m_plan.row_ops(h)[static_cast<size_t>(rows[g].level_row)];
        }
        upload(m_fs_ops, fs_ops, s);
        std::vector<int32_t> fs_rows;
        m_fs_rows_off.assign(L + 1, 0);
        m_fs_rows_n.assign(L + 1, 0);
        for (int h = 2; h <= L; ++h) {
            if (m_height_g1[h] <= m_height_g0[h])
                continue;
            const auto r     = unsearched_rows(m_plan, h);
            m_fs_rows_off[h] = static_cast<int64_t>(fs_rows.size());
            m_fs_rows_n[h]   = static_cast<int64_t>(r.size());
            fs_rows.insert(fs_rows.end(), r.begin(), r.end());
        }
        upload(m_fs_rows, fs_rows, s);
        // on by default, one chunk staged at once (fp16: the gulp 3.6-4.6 ms
        // shorter on the 4096-channel headline gulp; fp32: 2 ms)
        m_fs_on = true;
    }

    // Window-box variance table g[L][w].
    m_max_len          = m_plan.max_leaf_length();
    const auto& widths = m_plan.widths();
    std::vector<double> gtab((m_max_len + 1) * widths.size(), 0.0);
    for (int32_t Lc = 1; Lc <= m_max_len; ++Lc)
        for (size_t w = 0; w < widths.size(); ++w)
            gtab[Lc * widths.size() + w] =
                window_box_variance(Lc, widths[w], bc.use_trapezoid != 0);
    upload(m_gtab, gtab, s);
    const SizeType nw = widths.size();
    m_var.reserve(std::max<SizeType>(m_nsearch * nw * sizeof(double), 16));
    m_inv.reserve(std::max<SizeType>(m_nsearch * nw * sizeof(float), 16));
    m_inv_or.reserve(std::max<SizeType>(m_nsearch * nw * sizeof(float), 16));
    const SizeType nruns = bc.peak_mode == FROST_PEAK_ACROSS_WIDTHS ? 1 : nw;
    m_carry.reserve(std::max<SizeType>(m_nsearch * nruns * sizeof(RunState), 16));
    FB_CUDA(cudaMemsetAsync(m_carry.get(), 0, m_nsearch * nruns * sizeof(RunState), s));
    m_row_counts.reserve(std::max<SizeType>(m_nsearch * sizeof(uint32_t), 16));
    const SizeType maxc = std::max<uint64_t>(bc.max_candidates, 1);
    m_cands.reserve(maxc * sizeof(frost_candidate));
    for (int i = 0; i < 2; ++i) {
        m_sort_keys[i].reserve(maxc * sizeof(uint64_t));
        m_sort_vals[i].reserve(maxc * sizeof(uint32_t));
    }
    m_sort_hist.reserve(sort_hist_bytes(maxc));
    m_cands_sorted.reserve(maxc * sizeof(frost_candidate));
    m_cand_range.reserve(2 * sizeof(unsigned long long));
    {
        uint32_t max_level = 0, max_idx = 0, max_dm = 0;
        for (const PlaneInfo& pi : pinfo) {
            max_level = std::max(max_level, pi.subband_level);
            max_idx   = std::max(max_idx, pi.subband_idx);
        }
        for (const auto& p : planes)
            max_dm = std::max<uint32_t>(max_dm, static_cast<uint32_t>(std::max<size_t>(p.delay.size(), 1) - 1));
        m_key_level_bits  = bits_of(max_level);
        m_key_idx_bits    = bits_of(max_idx);
        m_key_dm_bits     = bits_of(max_dm);
        m_key_filter_bits = bits_of(static_cast<uint64_t>(std::max<SizeType>(nw, 1) - 1));
    }
    m_counters.reserve(4 * sizeof(unsigned long long));
    m_clock.reserve(sizeof(GulpClock));
    m_clock_h.reserve(sizeof(GulpClock));
    m_frontier.reserve(sizeof(unsigned long long));
    m_mask_d.reserve(C);
    m_mask_or_d.reserve(C);

    // Tile length: the whole gulp unless the budget (or the device) is short.
    int64_t tile = bc.tile_nsamps != 0 ? static_cast<int64_t>(bc.tile_nsamps)
                                       : static_cast<int64_t>(dd.block_nsamps);
    tile = round_up(std::min<int64_t>(tile, static_cast<int64_t>(dd.block_nsamps)), kTileQuantum);
    size_t free_b = 0, total_b = 0;
    FB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const SizeType limit = m_budget = memory_budget != 0 ? memory_budget
                                              : static_cast<SizeType>(0.85 * static_cast<double>(free_b));
    while (plan_bytes(tile) > limit && tile > kTileQuantum)
        tile = round_up(tile / 2, kTileQuantum);
    if (plan_bytes(tile) > limit)
        throw Error(FROST_ERR_OUT_OF_MEMORY,
                    "search: plan needs " + std::to_string(plan_bytes(tile)) +
                        " device bytes at the smallest tile; budget " + std::to_string(limit));
    allocate(tile);
    FB_CUDA(cudaStreamSynchronize(s));
}

// FDMT schedule. Levels holding searched planes, level 1 and the top are
// stored; with `fuse`, a level whose successor is not stored is computed
// straight from the one below its predecessor (two levels in one pass,
// halving that pair's HBM traffic).
void Engine::validate(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc, const Plan& plan) {
    if (bc.storage != FROST_STORAGE_FP32 && bc.storage != FROST_STORAGE_FP16)
        invalid("search: storage must be fp32 or fp16");
    if (bc.peak_mode < FROST_PEAK_PER_WIDTH || bc.peak_mode > FROST_PEAK_ALL)
        invalid("search: invalid peak_mode");
    if (!is_finite(bc.detect_thresh))
        invalid("search: detect_thresh must be finite");
    if (!(bc.noise_sigma == 1.0F) || bc.input_nbits != 32 || !(bc.input_mean == 0.0F))
        invalid("search: the engine takes calibrated float32 input (noise_sigma 1, "
                "input_nbits 32, input_mean 0)");
    if (plan.widths().size() > 32)
        invalid("search: more than 32 boxcar widths (raise wtsp)");
    if (dd.block_nsamps <= static_cast<uint64_t>(plan.dt_max()) + bc.max_boxcar)
        invalid("nsamps_gulp must exceed the dedispersion max_delay (" + std::to_string(plan.dt_max()) +
                ") plus boxcar_max (" + std::to_string(bc.max_boxcar) + ")");
    if (bc.tile_nsamps != 0 && bc.tile_nsamps % kTileQuantum != 0)
        invalid("search: tile_nsamps must be a multiple of 4096");
}

Engine::Footprint Engine::estimate(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc) {
    const Plan plan(plan_config(dd, bc));
    validate(dd, bc, plan);
    // The allocations of the constructor, allocate() for the configured tile
    // under both schedules autotune may try (buffers only grow), and
    // autotune's zero waterfall; every buffer at least 16 bytes.
    auto b16 = [](SizeType bytes) { return std::max<SizeType>(bytes, 16); };
    const SizeType es   = bc.storage == FROST_STORAGE_FP16 ? 2 : 4;
    const int L         = plan.levels();
    const int32_t C     = plan.nchans();
    const auto& widths  = plan.widths();
    const SizeType nw   = widths.size();
    Footprint f;
    // tables
    const auto& leaf = plan.leaf_ops();
    SizeType nodes   = leaf.empty() ? 0 : 1;
    for (size_t i = 1; i < leaf.size(); ++i)
        if (leaf[i].chan_lo != leaf[i - 1].chan_lo || leaf[i].chan_hi != leaf[i - 1].chan_hi)
            ++nodes;
    SizeType nrow_ops = 0;
    std::vector<int64_t> row_op_offset(L + 2, 0);
    for (int h = 2; h <= L; ++h) {
        row_op_offset[h] = static_cast<int64_t>(nrow_ops);
        nrow_ops += plan.row_ops(h).size();
    }
    SizeType nsearch = 0, nleaf = 0, nfs_rows = 0;
    std::vector<char> searched(L + 1, 0);
    for (const auto& p : plan.planes()) {
        nsearch += p.delay.size();
        nleaf += p.delay.size() * static_cast<SizeType>(p.chan_end - p.chan_begin);
        searched[p.height] = 1;
    }
    for (int h = 2; h <= L; ++h)
        if (searched[h])
            nfs_rows += unsearched_rows(plan, h).size();
    const SizeType nruns = bc.peak_mode == FROST_PEAK_ACROSS_WIDTHS ? 1 : nw;
    f.table_bytes = b16(leaf.size() * sizeof(LeafOp)) + b16((nodes + 1) * sizeof(int32_t)) +
                    b16(nrow_ops * sizeof(RowOp)) + b16(nsearch * sizeof(SearchRow)) +
                    b16(plan.planes().size() * sizeof(PlaneInfo)) + b16(nleaf * sizeof(uint16_t)) +
                    b16(nsearch * sizeof(int64_t)) + b16(nw * sizeof(int32_t)) +
                    b16(nsearch * sizeof(RowOp)) + b16(nfs_rows * sizeof(int32_t)) +
                    b16((static_cast<SizeType>(plan.max_leaf_length()) + 1) * nw * sizeof(double)) +
                    nsearch * nw * (sizeof(double) + 2 * sizeof(float)) + b16(nsearch * nruns * sizeof(RunState)) +
                    b16(nsearch * sizeof(uint32_t)) + 4 * sizeof(unsigned long long) + sizeof(GulpClock) +
                    sizeof(unsigned long long) + 2 * static_cast<SizeType>(C);
    {
        const SizeType maxc = std::max<SizeType>(bc.max_candidates, 1);
        // detections, their sorted copy, the sort's keys and positions
        // (two of each), its histograms and the peak range
        f.candidate_bytes = maxc * (2 * sizeof(frost_candidate) + 2 * sizeof(uint64_t) + 2 * sizeof(uint32_t)) +
                            sort_hist_bytes(maxc) + 2 * sizeof(unsigned long long);
    }
    // level buffers and histories of the fused and single-level schedules
    int64_t tile = bc.tile_nsamps != 0 ? static_cast<int64_t>(bc.tile_nsamps) : static_cast<int64_t>(dd.block_nsamps);
    tile                = round_up(std::min<int64_t>(tile, static_cast<int64_t>(dd.block_nsamps)), kTileQuantum);
    const int64_t ncols = round_up(tile, kTileQuantum);
    const int32_t halo  = search_halo(widths.back());
    SizeType buf[2] = {16, 16}, hist = 0, fused = 16;
    for (const bool fuse : {true, false}) {
        const Schedule sc = make_schedule(plan, row_op_offset, fuse);
        SizeType h_bytes  = 0;
        for (int h = 1; h <= L; ++h) {
            h_bytes += b16(static_cast<SizeType>(plan.level_rows(h)) * sc.hist_len[h] * es);
            if (sc.buf_of[h] < 0)
                continue;
            const int64_t need = searched[h] ? std::max<int64_t>(sc.hist_len[h], halo) : sc.hist_len[h];
            const SizeType base = static_cast<SizeType>(round_up(need, 8));
            buf[sc.buf_of[h]] = std::max<SizeType>(buf[sc.buf_of[h]],
                                                   static_cast<SizeType>(plan.level_rows(h)) * (base + ncols) * es);
        }
        hist  = std::max(hist, h_bytes);
        fused = std::max<SizeType>(fused, sc.fused.size() * sizeof(FusedOp));
    }
    const SizeType in_hist = b16(static_cast<SizeType>(C) * plan.level_history(0) * sizeof(float));
    f.table_bytes += fused;
    f.level_bytes     = buf[0] + buf[1];
    f.history_bytes   = hist + 2 * in_hist;
    f.transient_bytes = static_cast<SizeType>(C) * std::min<SizeType>(dd.block_nsamps, 4096) * sizeof(float);
    f.dt_max          = plan.dt_max();
    return f;
}

Engine::Schedule Engine::make_schedule(const Plan& plan, const std::vector<int64_t>& row_op_offset, bool fuse) {
    const int L             = plan.levels();
    const auto& plan_planes = plan.planes();
    std::vector<char> keep(L + 1, 0);
    keep[1] = 1;
    keep[L] = 1;
    for (const auto& p : plan_planes)
        keep[p.height] = 1;
    Schedule sc;
    sc.buf_of.assign(L + 1, -1);
    sc.hist_len.assign(L + 1, 0);
    sc.hist_len[0] = plan.level_history(0);
    sc.steps.push_back({1, 0, false, 0});
    sc.buf_of[1] = 0;
    for (int h = 1; h < L;) {
        Step st{};
        if (fuse && h + 2 <= L && !keep[h + 1]) {
            st = {h + 2, h, true, static_cast<int64_t>(sc.fused.size())};
            const auto& mid = plan.row_ops(h + 1);
            for (const RowOp& op : plan.row_ops(h + 2)) {
                const RowOp& a = mid[op.lo_row];
                FusedOp f{{a.lo_row, a.hi_row, -1, -1}, {0, a.hi_row >= 0 ? a.shift : 0, 0, 0}};
                if (op.hi_row >= 0) {
                    const RowOp& b = mid[op.hi_row];
                    f.row[2]       = b.lo_row;
                    f.shift[2]     = op.shift;
                    f.row[3]       = b.hi_row;
                    f.shift[3]     = b.hi_row >= 0 ? op.shift + b.shift : 0;
                }
                for (int j = 1; j < 4; ++j)
                    if (f.row[j] >= 0)
                        sc.hist_len[h] = std::max(sc.hist_len[h], f.shift[j]);
                sc.fused.push_back(f);
            }
            h += 2;
        } else {
            st = {h + 1, h, false, row_op_offset[h + 1]};
            for (const RowOp& op : plan.row_ops(h + 1))
                if (op.hi_row >= 0)
                    sc.hist_len[h] = std::max(sc.hist_len[h], op.shift);
            h += 1;
        }
        sc.buf_of[st.out] = static_cast<int>(sc.steps.size() % 2);
        sc.steps.push_back(st);
    }
    for (const auto& p : plan_planes)
        sc.hist_len[p.height] = std::max(sc.hist_len[p.height], plan.widths().back() - 1);
    // whole 16-byte vectors of fp16 (and fp32) columns, so that the history
    // copies move aligned vectors (a longer history is a superset)
    for (int h = 1; h <= L; ++h)
        sc.hist_len[h] = static_cast<int32_t>(round_up(sc.hist_len[h], 8));
    return sc;
}

void Engine::build_schedule(bool fuse) {
    Schedule sc = make_schedule(m_plan, m_row_op_offset, fuse);
    m_steps     = std::move(sc.steps);
    m_buf_of    = std::move(sc.buf_of);
    m_hist_len  = std::move(sc.hist_len);
    upload(m_fused_ops, sc.fused, m_stream);
    m_fuse = fuse;
    if (m_graph != nullptr) {
        cudaGraphExecDestroy(m_graph);
        m_graph = nullptr;
    }
}

// ---- autotuning -----------------------------------------------------------
//
// The FDMT launch shape is measured, not assumed: for this plan's geometry
// the engine times one tile pass for every candidate (fused two-level steps
// with 2, 3 or 4 bulk-copy stages, or single levels; 4 to 128 tiles
// of 2048 columns per level-kernel CTA) on a zero waterfall (the level
// kernels always process the tile's full width), keeps the fastest and
// caches it for the process by geometry, then restores a fresh stream state.
// The search chunk stays at 4096 samples: a zero waterfall exercises only
// the search's no-detection path, where 2048-sample chunks look faster, but
// on real detections (4096 channels, DM 0-2000) they are slower (38 vs 32 ms
// per gulp), so it is a manual option (set_launch_shape), not a tuned one.
namespace {
struct TuneChoice {
    bool fuse;
    int32_t tpc;
    int32_t stages;
    int32_t chunk;
    double ms;
};
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tune_cache;
} // namespace

Engine::Tuned Engine::autotune() {
    DeviceGuard g(m_device);
    const bool timing_was = m_timing_on;
    m_timing_on           = false;
    cudaStream_t s = m_stream;
    std::string key = std::to_string(m_plan.nchans()) + "|" + std::to_string(m_ncols) + "|" +
                      std::to_string(m_fp16) + "|" + std::to_string(m_plan.widths().back()) + "|" +
                      std::to_string(fused_search_mode());
    for (int h = 1; h <= m_plan.levels(); ++h)
        key += "|" + std::to_string(m_plan.level_rows(h));
    for (const auto& p : m_plan.planes())
        key += "|p" + std::to_string(p.height);
    TuneChoice best{true, 16, 0, kSearchChunk, 0.0};
    bool cached = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            best   = it->second;
            cached = true;
        }
    }
    if (!cached) {
        const int32_t C      = m_plan.nchans();
        const SizeType ncols = std::min<SizeType>(m_plan.config().block_nsamps, 4096);
        DeviceBuffer wf;
        wf.reserve(static_cast<SizeType>(C) * ncols * sizeof(float));
        FB_CUDA(cudaMemsetAsync(wf.get(), 0, static_cast<SizeType>(C) * ncols * sizeof(float), s));
        FB_CUDA(cudaMemsetAsync(m_inv.get(), 0, m_inv.bytes(), s));
        FB_CUDA(cudaMemsetAsync(m_inv_or.get(), 0, m_inv_or.bytes(), s));
        auto* ck = m_clock_h.as<GulpClock>();
        *ck      = GulpClock{0, 0, 0};
        FB_CUDA(cudaMemcpyAsync(m_clock.get(), ck, sizeof(GulpClock), cudaMemcpyHostToDevice, s));
        cudaEvent_t a, b;
        FB_CUDA(cudaEventCreate(&a));
        FB_CUDA(cudaEventCreate(&b));
        best.ms = -1.0;
        for (const bool fuse : {true, false}) {
            build_schedule(fuse);
            if (plan_bytes(m_tile) > m_budget)
                continue;
            allocate(m_tile);
            std::vector<int32_t> stage_options{0};
            if (fuse)
                stage_options = m_fp16 ? std::vector<int32_t>{2, 3, 4} : std::vector<int32_t>{2, 3};
            for (const int32_t stages : stage_options) {
                for (const int32_t tpc : {4, 8, 16, 32, 64, 128}) {
                    m_level_tpc     = tpc;
                    m_level2_stages = stages;
                    run_tiles(wf.as<float>(), ncols, s); // warm-up
                    FB_CUDA(cudaEventRecord(a, s));
                    run_tiles(wf.as<float>(), ncols, s);
                    FB_CUDA(cudaEventRecord(b, s));
                    FB_CUDA(cudaEventSynchronize(b));
                    float ms = 0.0F;
                    FB_CUDA(cudaEventElapsedTime(&ms, a, b));
                    if (best.ms < 0.0 || ms < best.ms)
                        best = {fuse, tpc, stages, kSearchChunk, ms};
                }
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
    }
    // apply the choice and start the stream afresh
    apply_shape(best.fuse, best.tpc, best.stages, best.chunk);
    m_timing_on = timing_was;
    return Tuned{best.fuse, best.tpc, best.stages, best.chunk, best.ms, cached};
}

void Engine::apply_shape(bool fuse, int32_t tpc, int32_t stages, int32_t chunk) {
    cudaStream_t s = m_stream;
    build_schedule(fuse);
    allocate(m_tile);
    m_level_tpc     = tpc;
    m_level2_stages = stages;
    m_search_chunk  = chunk;
    m_samples       = 0;
    m_var_ready     = false;
    const SizeType nruns = m_cfg.peak_mode == FROST_PEAK_ACROSS_WIDTHS ? 1 : m_plan.widths().size();
    FB_CUDA(cudaMemsetAsync(m_carry.get(), 0, m_nsearch * nruns * sizeof(RunState), s));
    FB_CUDA(cudaStreamSynchronize(s));
}

void Engine::set_launch_shape(bool fuse, int32_t tpc, int32_t stages, int32_t chunk) {
    if (tpc < 1 || tpc > 128)
        invalid("search: tiles per CTA must be in [1, 128]");
    if (stages != 0 && stages != 2 && stages != 3 && !(stages == 4 && m_fp16))
        invalid("search: fused stages must be 0, 2, 3 (or 4 with fp16 storage)");
    if (chunk != 2048 && chunk != 4096)
        invalid("search: the search chunk must be 2048 or 4096 samples");
    DeviceGuard g(m_device);
    const bool was = m_fuse;
    build_schedule(fuse);
    if (plan_bytes(m_tile) > m_budget) {
        build_schedule(was);
        throw Error(FROST_ERR_OUT_OF_MEMORY, "search: the launch shape does not fit the memory budget");
    }
    apply_shape(fuse, tpc, stages, chunk);
}

void Engine::set_residency(int32_t ctas_per_sm) {
    if (ctas_per_sm < 0 || ctas_per_sm > 64)
        invalid("search: CTAs per SM must be in [0, 64]");
    DeviceGuard g(m_device);
    FB_CUDA(cudaStreamSynchronize(m_stream));
    if (m_graph != nullptr) {
        // the captured launches carry the old grids
        FB_CUDA(cudaGraphExecDestroy(m_graph));
        m_graph = nullptr;
    }
    m_ctas_per_sm = ctas_per_sm;
}

void Engine::set_fused_search(int32_t mode) {
    if (mode < 0 || mode > 2)
        invalid("search: fused search mode must be 0, 1 or 2");
    DeviceGuard g(m_device);
    FB_CUDA(cudaStreamSynchronize(m_stream));
    if (m_graph != nullptr) {
        // the captured launches follow the old schedule
        FB_CUDA(cudaGraphExecDestroy(m_graph));
        m_graph = nullptr;
    }
    m_fs_on = mode != 0;
    if (mode != 0)
        m_fs_buffers = mode;
}

void Engine::set_wait_limit(long long tries) {
    DeviceGuard g(m_device);
    FB_CUDA(cudaStreamSynchronize(m_stream));
    if (m_graph != nullptr) {
        // the captured launches carry the old limit
        FB_CUDA(cudaGraphExecDestroy(m_graph));
        m_graph = nullptr;
    }
    m_wait_limit = tries < 0 ? kDefaultWaitLimit : tries;
}

// ---- batch members ----------------------------------------------------------

void Engine::batch_begin(const float* waterfall, SizeType nsamps, const uint8_t* mask, cudaStream_t caller) {
    if (waterfall == nullptr)
        invalid("search: null waterfall");
    if (nsamps == 0 || nsamps > m_plan.config().block_nsamps)
        invalid("search: nsamps must be in [1, block_nsamps]");
    if (m_capture_on || m_timing_on)
        fail_state("search: plane capture and timing are off in a batch");
    DeviceGuard g(m_device);
    cudaStream_t s  = m_stream;
    m_launches      = 0;
    const int32_t C = m_plan.nchans();
    std::vector<uint8_t> cur = m_mask;
    if (mask != nullptr)
        for (int32_t c = 0; c < C; ++c)
            cur[c] = mask[c] != 0 ? 1 : 0;
    const bool or_active = cur != m_mask;
    std::vector<uint8_t> orm(C);
    for (int32_t c = 0; c < C; ++c)
        orm[c] = (cur[c] | m_mask[c]) ? 1 : 0;
    if (caller != nullptr && caller != s) {
        FB_CUDA(cudaEventRecord(m_order, caller));
        FB_CUDA(cudaStreamWaitEvent(s, m_order, 0));
    }
    update_variance(cur, orm);
    auto* ck      = m_clock_h.as<GulpClock>();
    ck->gulp_t0   = static_cast<int64_t>(m_samples);
    ck->or_active = or_active ? 1 : 0;
    ck->pad       = 0;
    FB_CUDA(cudaMemcpyAsync(m_clock.get(), ck, sizeof(GulpClock), cudaMemcpyHostToDevice, s));
    FB_CUDA(cudaMemsetAsync(m_counters.get(), 0, 4 * sizeof(unsigned long long), s));
    FB_CUDA(cudaMemsetAsync(m_row_counts.get(), 0, m_nsearch * sizeof(uint32_t), s));
    m_batch_wf     = waterfall;
    m_batch_nsamps = nsamps;
    m_batch_mask   = std::move(cur);
}

int64_t Engine::batch_rounds() const {
    const int64_t tiles = (static_cast<int64_t>(m_batch_nsamps) + m_tile - 1) / m_tile;
    return tiles * static_cast<int64_t>(m_steps.size());
}

int Engine::batch_pre(int64_t round, cudaStream_t s, RoundWork& w) {
    const int64_t nsteps  = static_cast<int64_t>(m_steps.size());
    const int64_t t_off   = (round / nsteps) * m_tile;
    const size_t si       = static_cast<size_t>(round % nsteps);
    const int32_t n_valid = static_cast<int32_t>(std::min<int64_t>(m_tile, static_cast<int64_t>(m_batch_nsamps) - t_off));
    const Step& st        = m_steps[si];
    const LevelView out   = view(st.out);
    unsigned* err         = reinterpret_cast<unsigned*>(m_counters.as<unsigned long long>() + 3);
    w                     = RoundWork{};
    if (si == 0) {
        const int32_t C = m_plan.nchans();
        launch_level1(m_leaf_ops.as<LeafOp>(), m_node_first_op_d.as<int32_t>(),
                      static_cast<int32_t>(m_node_first_op.size() - 1), m_plan.level_history(0), m_batch_wf,
                      static_cast<int64_t>(m_batch_nsamps), t_off, n_valid, m_in_hist.as<float>(),
                      m_plan.level_history(0), out, static_cast<int32_t>(m_ncols), s, 0);
        launch_save_input_history(m_batch_wf, static_cast<int64_t>(m_batch_nsamps), t_off, n_valid, C,
                                  m_in_hist.as<float>(), m_in_scratch.as<float>(), m_plan.level_history(0), s);
        m_launches += 1;
        return 2;
    }
    const LevelView in = view(st.in);
    w.has_level        = true;
    w.fused            = st.fused;
    w.fp16             = m_fp16;
    w.stages           = m_level2_stages;
    w.level            = LevelSeg{st.fused ? static_cast<const void*>(m_fused_ops.as<FusedOp>() + st.op_offset)
                                           : static_cast<const void*>(m_row_ops.as<RowOp>() + st.op_offset),
                                  in.data,
                                  out.data,
                                  in.pitch,
                                  out.pitch,
                                  in.base,
                                  out.base,
                                  static_cast<int32_t>(m_ncols / kTimePerCta),
                                  m_level_tpc,
                                  static_cast<int64_t>(m_plan.level_rows(st.out)),
                                  0,
                                  err,
                                  nullptr};
    m_launches += 1;
    return 0;
}

int Engine::batch_mid(int64_t round, cudaStream_t s, RoundWork& w) {
    const int64_t nsteps  = static_cast<int64_t>(m_steps.size());
    const int64_t t_off   = (round / nsteps) * m_tile;
    const Step& st        = m_steps[static_cast<size_t>(round % nsteps)];
    const int h           = st.out;
    const int32_t n_valid = static_cast<int32_t>(std::min<int64_t>(m_tile, static_cast<int64_t>(m_batch_nsamps) - t_off));
    const LevelView out   = view(h);
    launch_load_history(out, m_plan.level_rows(h), m_hist_len[h], m_hist[h].get(), s);
    if (m_height_g1[h] > m_height_g0[h]) {
        w.has_search   = true;
        w.chunk        = m_search_chunk;
        w.search       = SearchSeg{};
        w.search.p     = params(t_off, n_valid);
        w.search.level = out.data;
        w.search.pitch = out.pitch;
        w.search.base  = out.base;
        w.search.fp16  = out.fp16;
        w.search.g0    = m_height_g0[h];
        w.search.nrows = m_height_g1[h] - m_height_g0[h];
        m_launches += 1;
    }
    return 1;
}

int Engine::batch_post(int64_t round, cudaStream_t s) {
    const int64_t nsteps  = static_cast<int64_t>(m_steps.size());
    const int64_t t_off   = (round / nsteps) * m_tile;
    const size_t si       = static_cast<size_t>(round % nsteps);
    const int32_t n_valid = static_cast<int32_t>(std::min<int64_t>(m_tile, static_cast<int64_t>(m_batch_nsamps) - t_off));
    const Step& st        = m_steps[si];
    int n                 = 0;
    if (si > 0) {
        launch_save_history(view(st.in), m_plan.level_rows(st.in), m_hist_len[st.in], n_valid,
                            m_hist[st.in].get(), s);
        ++n;
    }
    if (static_cast<int64_t>(si) == nsteps - 1) {
        const int L = m_plan.levels();
        launch_save_history(view(L), m_plan.level_rows(L), m_hist_len[L], n_valid, m_hist[L].get(), s);
        ++n;
    }
    return n;
}

void Engine::batch_finish() {
    DeviceGuard g(m_device);
    m_samples += m_batch_nsamps;
    m_mask = m_batch_mask;
    collect(m_stream);
    m_timing.total_launches += m_launches;
    m_timing.executes += 1;
    m_timing.unfused_model_bytes += unfused_model_bytes(m_batch_nsamps);
    m_batch_wf     = nullptr;
    m_batch_nsamps = 0;
}

void Engine::restart() {
    DeviceGuard g(m_device);
    FB_CUDA(cudaStreamSynchronize(m_stream));
    apply_shape(m_fuse, m_level_tpc, m_level2_stages, m_search_chunk);
    m_mask = m_kill;
    m_results.clear();
    m_dropped_global = 0;
    m_dropped_per_dm = 0;
}

Engine::Tuned Engine::launch_shape() const {
    return Tuned{m_fuse, m_level_tpc, m_level2_stages, m_search_chunk, 0.0, false};
}

Engine::~Engine() {
    if (m_stream != nullptr) {
        cudaSetDevice(m_device);
        cudaStreamSynchronize(m_stream);
        if (m_graph != nullptr)
            cudaGraphExecDestroy(m_graph);
        for (auto e : m_event_pool)
            cudaEventDestroy(e);
        if (m_order != nullptr)
            cudaEventDestroy(m_order);
        cudaStreamDestroy(m_stream);
    }
}

uint64_t Engine::unfused_model_bytes(SizeType nsamps) const {
    const uint64_t s = m_fp16 ? 2 : 4;
    const uint64_t T = nsamps;
    uint64_t b      = 0;
    for (int l = 1; l <= m_plan.levels(); ++l) {
        const uint64_t below = l == 1 ? static_cast<uint64_t>(m_plan.nchans())
                                      : static_cast<uint64_t>(m_plan.level_rows(l - 1));
        const uint64_t rows  = static_cast<uint64_t>(m_plan.level_rows(l));
        b += (below + rows) * (T + static_cast<uint64_t>(m_plan.level_history(l))) * s;
    }
    for (const auto& p : m_plan.planes())
        b += static_cast<uint64_t>(p.level_row.size()) * T * s;
    return b;
}

void Engine::enable_timing(bool on) {
    m_timing_on = on;
    m_timing    = frost_search_timing{};
}

cudaEvent_t Engine::next_event() {
    if (m_events_used == m_event_pool.size()) {
        cudaEvent_t e;
        FB_CUDA(cudaEventCreate(&e));
        m_event_pool.push_back(e);
    }
    return m_event_pool[m_events_used++];
}

template <class F> void Engine::timed(Phase ph, cudaStream_t s, F&& f) {
    if (!m_timing_on) {
        f();
        return;
    }
    Mark m{ph, next_event(), next_event()};
    FB_CUDA(cudaEventRecord(m.a, s));
    f();
    FB_CUDA(cudaEventRecord(m.b, s));
    m_marks.push_back(m);
}

// Accumulates the marked phases' device time (the stream is synchronised).
void Engine::harvest() {
    for (const auto& m : m_marks) {
        float ms = 0.0F;
        FB_CUDA(cudaEventElapsedTime(&ms, m.a, m.b));
        switch (m.phase) {
        case kLevel1: m_timing.level1_ms += ms; break;
        case kLevel: m_timing.level_ms += ms; break;
        case kSearch: m_timing.search_ms += ms; break;
        case kHistory: m_timing.history_ms += ms; break;
        case kVariance: m_timing.variance_ms += ms; break;
        default: break;
        }
    }
    m_marks.clear();
    m_events_used = 0;
}

int32_t Engine::level_base(int h) const {
    int64_t need = m_hist_len[h];
    if (m_height_g1[h] > m_height_g0[h])
        need = std::max<int64_t>(need, search_halo(m_plan.widths().back()));
    return static_cast<int32_t>(round_up(need, 8));
}

SizeType Engine::plan_bytes(int64_t tile) const {
    const SizeType es   = m_fp16 ? 2 : 4;
    const int L         = m_plan.levels();
    const int64_t ncols = round_up(tile, kTileQuantum);
    SizeType buf[2]     = {0, 0};
    for (int h = 1; h <= L; ++h)
        if (m_buf_of[h] >= 0)
            buf[m_buf_of[h]] = std::max<SizeType>(
                buf[m_buf_of[h]], static_cast<SizeType>(m_plan.level_rows(h)) * (level_base(h) + ncols) * es);
    SizeType bytes = buf[0] + buf[1];
    for (int h = 1; h <= L; ++h)
        bytes += static_cast<SizeType>(m_plan.level_rows(h)) * m_hist_len[h] * es;
    bytes += 2 * static_cast<SizeType>(m_plan.nchans()) * m_plan.level_history(0) * sizeof(float);
    bytes += m_leaf_len.bytes() + m_rows.bytes() + m_var.bytes() + m_inv.bytes() * 2 +
             m_carry.bytes() + m_cands.bytes() + m_row_ops.bytes() + m_leaf_ops.bytes() +
             m_cands_sorted.bytes() + m_sort_keys[0].bytes() * 2 + m_sort_vals[0].bytes() * 2 + m_sort_hist.bytes();
    return bytes;
}

void Engine::allocate(int64_t tile) {
    const SizeType es = m_fp16 ? 2 : 4;
    const int L       = m_plan.levels();
    m_tile            = tile;
    m_ncols           = round_up(tile, kTileQuantum);
    m_base_of.assign(L + 1, 0);
    m_pitch_of.assign(L + 1, 0);
    SizeType buf[2] = {16, 16};
    for (int h = 1; h <= L; ++h) {
        if (m_buf_of[h] < 0)
            continue;
        m_base_of[h]  = level_base(h);
        m_pitch_of[h] = m_base_of[h] + m_ncols;
        buf[m_buf_of[h]] = std::max<SizeType>(buf[m_buf_of[h]],
                                              static_cast<SizeType>(m_plan.level_rows(h)) * m_pitch_of[h] * es);
    }
    for (int i = 0; i < 2; ++i) {
        m_buf[i].reserve(buf[i]);
        FB_CUDA(cudaMemsetAsync(m_buf[i].get(), 0, buf[i], m_stream));
    }
    m_hist.clear();
    m_hist.resize(L + 1);
    for (int h = 1; h <= L; ++h) {
        const SizeType bytes = static_cast<SizeType>(m_plan.level_rows(h)) * m_hist_len[h] * es;
        m_hist[h].reserve(std::max<SizeType>(bytes, 16));
        FB_CUDA(cudaMemsetAsync(m_hist[h].get(), 0, std::max<SizeType>(bytes, 16), m_stream));
    }
    const SizeType in_bytes = static_cast<SizeType>(m_plan.nchans()) * m_plan.level_history(0) * sizeof(float);
    m_in_hist.reserve(std::max<SizeType>(in_bytes, 16));
    m_in_scratch.reserve(std::max<SizeType>(in_bytes, 16));
    FB_CUDA(cudaMemsetAsync(m_in_hist.get(), 0, std::max<SizeType>(in_bytes, 16), m_stream));
}

SizeType Engine::device_bytes() const {
    SizeType total = m_buf[0].bytes() + m_buf[1].bytes();
    for (const auto& b : m_hist)
        total += b.bytes();
    const DeviceBuffer* rest[] = {&m_in_hist, &m_in_scratch, &m_wf_stage, &m_leaf_ops,
                                  &m_node_first_op_d, &m_row_ops, &m_fused_ops, &m_rows, &m_planes,
                                  &m_widths, &m_leaf_len, &m_leaf_offset, &m_gtab, &m_var, &m_inv,
                                  &m_inv_or, &m_mask_d, &m_mask_or_d, &m_carry, &m_row_counts, &m_cands,
                                  &m_counters, &m_clock, &m_frontier, &m_capture_rows,
                                  &m_sort_keys[0], &m_sort_keys[1], &m_sort_vals[0], &m_sort_vals[1],
                                  &m_sort_hist, &m_cands_sorted, &m_cand_range, &m_fs_ops, &m_fs_rows};
    for (const auto* b : rest)
        total += b->bytes();
    for (const auto& b : m_capture)
        total += b.bytes();
    return total;
}

LevelView Engine::view(int h) const {
    return LevelView{m_buf[m_buf_of[h]].get(), m_pitch_of[h], m_base_of[h], m_fp16 ? 1 : 0};
}

SearchParams Engine::params(int64_t tile_off, int32_t n_valid) const {
    SearchParams p{};
    p.rows         = m_rows.as<SearchRow>();
    p.planes       = m_planes.as<PlaneInfo>();
    p.widths       = m_widths.as<int32_t>();
    p.nwidths      = static_cast<int32_t>(m_plan.widths().size());
    p.wmax         = m_plan.widths().back();
    p.halo         = search_halo(p.wmax);
    p.err          = reinterpret_cast<unsigned*>(m_counters.as<unsigned long long>() + 3);
    p.wait_limit   = m_wait_limit;
    p.thresh       = m_cfg.detect_thresh;
    p.peak_mode    = m_cfg.peak_mode;
    p.trapezoid    = m_cfg.use_trapezoid ? 1 : 0;
    p.skip_cold    = m_cfg.skip_cold_prefix ? 1 : 0;
    p.pow2_widths  = 1;
    for (size_t w = 0; w < m_plan.widths().size(); ++w)
        if (m_plan.widths()[w] != (int32_t{1} << std::min<size_t>(w, 30)))
            p.pow2_widths = 0;
    p.clock        = m_clock.as<GulpClock>();
    p.tile_off     = tile_off;
    p.n_valid      = n_valid;
    p.inv_sigma    = m_inv.as<float>();
    p.inv_sigma_or = m_inv_or.as<float>();
    p.carry        = m_carry.as<RunState>();
    p.cands        = m_cands.as<frost_candidate>();
    p.ncands       = m_counters.as<unsigned long long>();
    p.max_cands    = m_cfg.max_candidates;
    p.row_counts   = m_row_counts.as<uint32_t>();
    p.max_per_dm   = static_cast<uint32_t>(std::min<uint64_t>(m_cfg.max_cands_per_dm, 0xFFFFFFFFULL));
    p.dropped      = m_counters.as<unsigned long long>() + 1;
    return p;
}

void Engine::update_variance(const std::vector<uint8_t>& cur, const std::vector<uint8_t>& orm) {
    if (m_var_ready && cur == m_var_mask && orm == m_var_mask_or)
        return;
    const int32_t C = m_plan.nchans();
    FB_CUDA(cudaMemcpyAsync(m_mask_d.get(), cur.data(), C, cudaMemcpyHostToDevice, m_stream));
    FB_CUDA(cudaMemcpyAsync(m_mask_or_d.get(), orm.data(), C, cudaMemcpyHostToDevice, m_stream));
    launch_variance(m_rows.as<SearchRow>(), m_planes.as<PlaneInfo>(), m_leaf_offset.as<int64_t>(),
                    m_leaf_len.as<uint16_t>(), static_cast<int64_t>(m_nsearch), m_gtab.as<double>(),
                    m_max_len, static_cast<int32_t>(m_plan.widths().size()),
                    m_mask_d.as<uint8_t>(), m_mask_or_d.as<uint8_t>(), m_var.as<double>(),
                    m_inv.as<float>(), m_inv_or.as<float>(), m_stream);
    ++m_launches;
    m_var_mask    = cur;
    m_var_mask_or = orm;
    m_var_ready   = true;
}

void Engine::execute(const float* waterfall, SizeType nsamps, bool on_device, const uint8_t* mask,
                     cudaStream_t stream) {
    if (waterfall == nullptr)
        invalid("search: null waterfall");
    if (nsamps == 0 || nsamps > m_plan.config().block_nsamps)
        invalid("search: nsamps must be in [1, block_nsamps]");
    DeviceGuard g(m_device);
    cudaStream_t s  = m_stream;
    m_launches      = 0;
    const int32_t C = m_plan.nchans();
    std::vector<uint8_t> cur = m_mask;
    if (mask != nullptr)
        for (int32_t c = 0; c < C; ++c)
            cur[c] = mask[c] != 0 ? 1 : 0;
    const bool or_active = cur != m_mask;
    std::vector<uint8_t> orm(C);
    for (int32_t c = 0; c < C; ++c)
        orm[c] = (cur[c] | m_mask[c]) ? 1 : 0;
    // Order the caller's stream before the engine's.
    if (stream != nullptr && stream != s) {
        FB_CUDA(cudaEventRecord(m_order, stream));
        FB_CUDA(cudaStreamWaitEvent(s, m_order, 0));
    }
    timed(kVariance, s, [&] { update_variance(cur, orm); });

    const float* wf = waterfall;
    if (!on_device) {
        const SizeType bytes = static_cast<SizeType>(C) * nsamps * sizeof(float);
        m_wf_stage.reserve(bytes);
        FB_CUDA(cudaMemcpyAsync(m_wf_stage.get(), waterfall, bytes, cudaMemcpyHostToDevice, s));
        wf = m_wf_stage.as<float>();
    }
    if (m_capture_on) {
        const auto& planes = m_plan.planes();
        m_capture.resize(planes.size());
        m_capture_cols = static_cast<int64_t>(nsamps);
        for (size_t p = 0; p < planes.size(); ++p)
            m_capture[p].reserve(std::max<SizeType>(planes[p].delay.size() * nsamps * sizeof(float), 16));
    }
    // The gulp's start and mask change, read by the search from device memory.
    {
        auto* ck      = m_clock_h.as<GulpClock>();
        ck->gulp_t0   = static_cast<int64_t>(m_samples);
        ck->or_active = or_active ? 1 : 0;
        ck->pad       = 0;
        FB_CUDA(cudaMemcpyAsync(m_clock.get(), ck, sizeof(GulpClock), cudaMemcpyHostToDevice, s));
    }
    const uint64_t before = m_launches; // the variance update's
    if (m_graphs_on && !m_timing_on && !m_capture_on) {
        if (m_graph == nullptr || m_graph_wf != wf || m_graph_nsamps != nsamps) {
            if (m_graph != nullptr) {
                FB_CUDA(cudaGraphExecDestroy(m_graph));
                m_graph = nullptr;
            }
            cudaGraph_t graph = nullptr;
            FB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try {
                run_tiles(wf, nsamps, s);
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph != nullptr)
                    cudaGraphDestroy(graph);
                throw;
            }
            FB_CUDA(cudaStreamEndCapture(s, &graph));
            const cudaError_t e = cudaGraphInstantiate(&m_graph, graph, 0);
            cudaGraphDestroy(graph);
            FB_CUDA(e);
            m_graph_wf       = wf;
            m_graph_nsamps   = nsamps;
            m_graph_launches = m_launches - before;
        }
        FB_CUDA(cudaGraphLaunch(m_graph, s));
        m_launches = before + m_graph_launches;
    } else {
        run_tiles(wf, nsamps, s);
    }
    m_samples += nsamps;
    m_mask = cur;
    collect(s);
    m_timing.total_launches += m_launches;
    m_timing.executes += 1;
    m_timing.unfused_model_bytes += unfused_model_bytes(nsamps);
    harvest();
}

void Engine::run_tiles(const float* wf, SizeType nsamps, cudaStream_t s) {
    FB_CUDA(cudaMemsetAsync(m_counters.get(), 0, 4 * sizeof(unsigned long long), s));
    FB_CUDA(cudaMemsetAsync(m_row_counts.get(), 0, m_nsearch * sizeof(uint32_t), s));

    const int L          = m_plan.levels();
    const int32_t C      = m_plan.nchans();
    const auto& planes   = m_plan.planes();
    const uint64_t es    = m_fp16 ? 2 : 4;
    for (int64_t t_off = 0; t_off < static_cast<int64_t>(nsamps); t_off += m_tile) {
        const int32_t n_valid = static_cast<int32_t>(std::min<int64_t>(m_tile, nsamps - t_off));
        const SearchParams sp = params(t_off, n_valid);
        for (size_t si = 0; si < m_steps.size(); ++si) {
            const Step& st      = m_steps[si];
            const int h         = st.out;
            const LevelView out = view(h);
            unsigned* err       = reinterpret_cast<unsigned*>(m_counters.as<unsigned long long>() + 3);
            if (si == 0) {
                timed(kLevel1, s, [&] {
                    launch_level1(m_leaf_ops.as<LeafOp>(), m_node_first_op_d.as<int32_t>(),
                                  static_cast<int32_t>(m_node_first_op.size() - 1),
                                  m_plan.level_history(0), wf, static_cast<int64_t>(nsamps), t_off,
                                  n_valid, m_in_hist.as<float>(), m_plan.level_history(0), out,
                                  static_cast<int32_t>(m_ncols), s, cta_cap());
                });
                timed(kHistory, s, [&] {
                    launch_save_input_history(wf, static_cast<int64_t>(nsamps), t_off, n_valid, C,
                                              m_in_hist.as<float>(), m_in_scratch.as<float>(),
                                              m_plan.level_history(0), s);
                });
                m_launches += 1;
                m_timing.algorithmic_level1_bytes +=
                    static_cast<uint64_t>(C) * m_ncols * sizeof(float) +
                    static_cast<uint64_t>(m_plan.level_rows(1)) * m_ncols * es;
            } else if (fused_search(st)) {
                // only the rows no plane searches; the search computes the rest
                const int64_t n = m_fs_rows_n[h];
                if (n > 0) {
                    timed(kLevel, s, [&] {
                        launch_level(m_row_ops.as<RowOp>() + st.op_offset, n, view(st.in), out,
                                     static_cast<int32_t>(m_ncols), err, s, m_level_tpc, cta_cap(), m_wait_limit,
                                     m_fs_rows.as<int32_t>() + m_fs_rows_off[h]);
                    });
                    m_launches += 1;
                    m_timing.level_launches += 1;
                    m_timing.algorithmic_level_bytes += static_cast<uint64_t>(3 * n) * m_ncols * es;
                }
            } else {
                timed(kLevel, s, [&] {
                    if (st.fused)
                        launch_level2(m_fused_ops.as<FusedOp>() + st.op_offset, m_plan.level_rows(h),
                                      view(st.in), out, static_cast<int32_t>(m_ncols), err, s, m_level_tpc,
                                      m_level2_stages, cta_cap(), m_wait_limit);
                    else
                        launch_level(m_row_ops.as<RowOp>() + st.op_offset, m_plan.level_rows(h),
                                     view(st.in), out, static_cast<int32_t>(m_ncols), err, s, m_level_tpc,
                                     cta_cap(), m_wait_limit);
                });
                m_launches += 1;
                m_timing.level_launches += 1;
                m_timing.algorithmic_level_bytes +=
                    static_cast<uint64_t>(m_plan.level_rows(st.in) + m_plan.level_rows(h)) * m_ncols * es;
            }
            timed(kHistory, s, [&] {
                launch_load_history(out, m_plan.level_rows(h), m_hist_len[h], m_hist[h].get(), s);
            });
            if (m_height_g1[h] > m_height_g0[h]) {
                const bool fs   = si > 0 && fused_search(st);
                const int64_t g = m_height_g1[h] - m_height_g0[h];
                timed(kSearch, s, [&] {
                    if (fs)
                        launch_search_fused(sp, view(st.in), out, m_fs_ops.as<RowOp>(), m_height_g0[h],
                                            m_height_g1[h], s, m_search_chunk, cta_cap(), m_fs_buffers);
                    else
                        launch_search(sp, out, m_height_g0[h], m_height_g1[h], s, m_search_chunk, cta_cap());
                });
                m_launches += 1;
                m_timing.search_launches += 1;
                // fused: the searched rows' children (at most two rows each) are
                // read and the rows written, instead of the rows read
                m_timing.algorithmic_search_bytes +=
                    static_cast<uint64_t>(fs ? 3 * g : g) * m_ncols * es;
                if (m_capture_on) {
                    for (size_t p = 0; p < planes.size(); ++p) {
                        if (planes[p].height != h)
                            continue;
                        std::vector<int64_t> rows(planes[p].level_row.begin(), planes[p].level_row.end());
                        upload(m_capture_rows, rows, s);
                        launch_capture_rows(out, m_capture_rows.as<int64_t>(),
                                            static_cast<int64_t>(rows.size()),
                                            m_capture[p].as<float>(), m_capture_cols, t_off,
                                            n_valid, s);
                        FB_CUDA(cudaStreamSynchronize(s));
                    }
                }
            }
            if (si > 0)
                timed(kHistory, s, [&] {
                    launch_save_history(view(st.in), m_plan.level_rows(st.in), m_hist_len[st.in],
                                        n_valid, m_hist[st.in].get(), s);
                });
        }
        timed(kHistory, s, [&] {
            launch_save_history(view(L), m_plan.level_rows(L), m_hist_len[L], n_valid, m_hist[L].get(), s);
        });
    }
}

void Engine::collect(cudaStream_t s) {
    const uint64_t cap = std::max<uint64_t>(m_cfg.max_candidates, 1);
    const frost_candidate* cands = m_cands.as<frost_candidate>();
    launch_cand_range(cands, m_counters.as<unsigned long long>(), cap, m_cand_range.as<unsigned long long>(), s);
    m_launches += 1;
    unsigned long long counters[6];
    FB_CUDA(cudaMemcpyAsync(counters, m_counters.get(), 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemcpyAsync(counters + 4, m_cand_range.get(), 2 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    if (counters[3] != 0)
        throw Error(FROST_ERR_TIMEOUT, "search: a level or search kernel's bounded wait for its bulk copies ran "
                                       "out; this call's results are incomplete");
    const uint64_t n = std::min<uint64_t>(counters[0], cap);
    m_results.resize(n);
    m_dropped_global = counters[1];
    m_dropped_per_dm = counters[2];
    if (n == 0)
        return;
    // Order (level, sub-band, DM row, peak, width): one packed key when the
    // fields fit in 64 bits (always for real plans: the peaks of one call
    // span about a gulp), else a comparison sort on the host.
    const int peak_bits = bits_of(counters[5] - counters[4]);
    const int key_bits  = m_key_level_bits + m_key_idx_bits + m_key_dm_bits + peak_bits + m_key_filter_bits;
    if (n >= 2 && key_bits <= 64) {
        const CandKeySpec spec{counters[4], m_key_idx_bits, m_key_dm_bits, peak_bits, m_key_filter_bits};
        uint64_t* keys     = m_sort_keys[0].as<uint64_t>();
        uint64_t* keys_alt = m_sort_keys[1].as<uint64_t>();
        uint32_t* vals     = m_sort_vals[0].as<uint32_t>();
        uint32_t* vals_alt = m_sort_vals[1].as<uint32_t>();
        launch_cand_keys(cands, n, spec, keys, vals, s);
        pp::radix_sort(keys, vals, keys_alt, vals_alt, n, key_bits, m_sort_hist.as<uint32_t>(), s);
        launch_cand_gather(cands, vals, n, m_cands_sorted.as<frost_candidate>(), s);
        m_launches += 2 + 3 * static_cast<uint64_t>((key_bits + 7) / 8);
        FB_CUDA(cudaMemcpyAsync(m_results.data(), m_cands_sorted.get(), n * sizeof(frost_candidate),
                                cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    FB_CUDA(cudaMemcpyAsync(m_results.data(), cands, n * sizeof(frost_candidate), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    std::sort(m_results.begin(), m_results.end(), [](const frost_candidate& a, const frost_candidate& b) {
        if (a.subband_level != b.subband_level)
            return a.subband_level < b.subband_level;
        if (a.subband_idx != b.subband_idx)
            return a.subband_idx < b.subband_idx;
        if (a.dm_idx != b.dm_idx)
            return a.dm_idx < b.dm_idx;
        if (a.peak_sample != b.peak_sample)
            return a.peak_sample < b.peak_sample;
        return a.filter_idx < b.filter_idx;
    });
}

void Engine::drain() {
    DeviceGuard g(m_device);
    cudaStream_t s = m_stream;
    FB_CUDA(cudaMemsetAsync(m_counters.get(), 0, 4 * sizeof(unsigned long long), s));
    FB_CUDA(cudaMemsetAsync(m_row_counts.get(), 0, m_nsearch * sizeof(uint32_t), s));
    const SearchParams sp = params(0, 0); // k_flush only emits the carried runs
    launch_flush_runs(sp, static_cast<int64_t>(m_nsearch), s);
    collect(s);
}

uint64_t Engine::frontier() {
    DeviceGuard g(m_device);
    // Earliest start of a still-open run, else the samples processed so far.
    const SizeType nruns = m_cfg.peak_mode == FROST_PEAK_ACROSS_WIDTHS ? 1 : m_plan.widths().size();
    if (m_cfg.peak_mode == FROST_PEAK_ALL)
        return m_samples;
    std::vector<RunState> runs(m_nsearch * nruns);
    FB_CUDA(cudaStreamSynchronize(m_stream));
    if (!runs.empty())
        FB_CUDA(cudaMemcpy(runs.data(), m_carry.get(), runs.size() * sizeof(RunState), cudaMemcpyDeviceToHost));
    uint64_t f = m_samples;
    for (const auto& r : runs)
        if (r.open)
            f = std::min<uint64_t>(f, static_cast<uint64_t>(r.start));
    return f;
}

frost_search_info Engine::info() const {
    frost_search_info i{};
    i.nchans       = static_cast<uint64_t>(m_plan.nchans());
    i.block_nsamps = m_plan.config().block_nsamps;
    i.tile_nsamps  = static_cast<uint64_t>(m_tile);
    i.dt_max       = static_cast<uint64_t>(m_plan.dt_max());
    i.ndm          = m_plan.config().dm_list.size();
    i.nplanes      = m_plan.planes().size();
    i.nwidths      = m_plan.widths().size();
    i.levels       = static_cast<uint64_t>(m_plan.levels());
    i.device_bytes = device_bytes();
    i.f_min        = m_plan.config().f_min;
    i.f_max        = m_plan.config().f_max;
    return i;
}

std::vector<double> Engine::variance_grid(SizeType plane, uint32_t width, const uint8_t* mask) const {
    const auto& planes = m_plan.planes();
    if (plane >= planes.size())
        invalid("search: plane index out of range");
    const Plane& p    = planes[plane];
    const auto len    = m_plan.leaf_lengths(static_cast<int>(plane));
    const int32_t nch = p.chan_end - p.chan_begin;
    const uint8_t* m  = mask != nullptr ? mask : m_mask.data();
    std::vector<double> g(m_plan.max_leaf_length() + 2, 0.0);
    for (int32_t L = 1; L < static_cast<int32_t>(g.size()); ++L)
        g[L] = window_box_variance(L, static_cast<int32_t>(width), m_cfg.use_trapezoid != 0);
    std::vector<double> out(p.delay.size(), 0.0);
    for (size_t r = 0; r < p.delay.size(); ++r) {
        double v = 0.0;
        for (int32_t c = 0; c < nch; ++c)
            if (m[p.chan_begin + c])
                v += g[len[r * nch + c]];
        out[r] = v;
    }
    return out;
}

void Engine::capture(bool on) {
    m_capture_on = on;
    if (!on)
        m_capture.clear();
}

void Engine::plane_data(SizeType plane, float* out, SizeType capacity) const {
    if (!m_capture_on || plane >= m_capture.size())
        fail_state("search: plane capture is off or no execute has run");
    const SizeType n = m_plan.planes()[plane].delay.size() * static_cast<SizeType>(m_capture_cols);
    if (capacity < n)
        invalid("search: plane buffer too small");
    DeviceGuard g(m_device);
    FB_CUDA(cudaMemcpy(out, m_capture[plane].get(), n * sizeof(float), cudaMemcpyDeviceToHost));
}

} // namespace fb::fdmt
