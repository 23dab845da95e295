// The search engine: a frost-owned replacement for dmt::FDMTBoxcar with its
// call shape (lib/pipeline/pipeline.cpp:346-367, 493, 517, 598-608).
// Streaming FDMT (per-level history carried across tiles and gulps) feeding
// the boxcar/trapezoid search with exact per-DM/width/mask noise.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.hpp"
#include "fdmt_plan.hpp"
#include "search_kernels.hpp"

namespace fb::fdmt {

class Engine {
public:
    Engine(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc,
           const uint8_t* kill_mask, SizeType memory_budget, int device);
    ~Engine();
    Engine(const Engine&)            = delete;
    Engine& operator=(const Engine&) = delete;

    void execute(const float* waterfall, SizeType nsamps, bool on_device, const uint8_t* mask,
                 cudaStream_t stream);
    void drain();

    const std::vector<frost_candidate>& results() const { return m_results; }
    /** The last results on the device (unsorted; results().size() rows),
     * valid until the next execute or drain. */
    const frost_candidate* device_results() const { return m_cands.as<frost_candidate>(); }
    uint64_t dropped_global() const { return m_dropped_global; }
    uint64_t dropped_per_dm() const { return m_dropped_per_dm; }
    uint64_t frontier();
    frost_search_info info() const;
    const Plan& plan() const { return m_plan; }
    std::vector<double> variance_grid(SizeType plane, uint32_t width, const uint8_t* mask) const;
    void capture(bool on);
    void plane_data(SizeType plane, float* out, SizeType capacity) const;
    int device() const { return m_device; }
    SizeType device_bytes() const;
    /** Stream of the engine's kernels (for callers timing them). */
    cudaStream_t stream() const { return m_stream; }
    /** Kernel launches of the last execute call. */
    uint64_t last_launches() const { return m_launches; }
    void enable_timing(bool on);
    const frost_search_timing& timing() const { return m_timing; }
    /** Tries of the level and search kernels' first wait on each bulk copy
     * (negative: the default; 0: give up at once); a drain after a give-up
     * always uses the default. */
    void set_wait_limit(long long tries);
    /** Bytes of the unfused FDMT + search model for a gulp of `nsamps`
     * samples (frost_search_timing.unfused_model_bytes). */
    uint64_t unfused_model_bytes(SizeType nsamps) const;

    /** The engine as one member of a multi-beam batch (serve::Batch): the
     * gulp is taken on the engine's own stream (batch_begin: mask, noise
     * tables, gulp clock, counters; ordered after `caller`), then run as
     * batch_rounds() rounds, one (tile, level step) each, whose level and
     * search launches the batch merges with the other members' into single
     * launches on its stream: batch_pre enqueues the round's own launches
     * that come before the level step (the leaf level) and describes its
     * level segment, batch_mid loads the level's history and describes its
     * search segment, batch_post saves the histories. batch_finish collects
     * the results once the engine's stream waits for the batch's. Device
     * waterfalls only; no plane capture or per-phase timing. */
    struct RoundWork {
        bool has_level  = false;
        bool fused      = false;
        bool fp16       = false;
        int32_t stages  = 0;
        LevelSeg level{};
        bool has_search = false;
        int32_t chunk   = 0;
        SearchSeg search{};
    };
    void batch_begin(const float* waterfall, SizeType nsamps, const uint8_t* mask, cudaStream_t caller);
    int64_t batch_rounds() const;
    /** Each returns the launches it enqueued itself (segments not counted). */
    int batch_pre(int64_t round, cudaStream_t s, RoundWork& w);
    int batch_mid(int64_t round, cudaStream_t s, RoundWork& w);
    int batch_post(int64_t round, cudaStream_t s);
    void batch_finish();
    /** Starts the stream afresh: histories and run states cleared, sample
     * count zero, the constructor's mask current (after a failed gulp). */
    void restart();

private:
    enum Phase { kLevel1, kLevel, kSearch, kHistory, kVariance, kPhases };
    struct Mark {
        Phase phase;
        cudaEvent_t a, b;
    };
    bool m_timing_on = false;
    frost_search_timing m_timing{};
    std::vector<cudaEvent_t> m_event_pool;
    std::vector<Mark> m_marks;
    size_t m_events_used = 0;
    cudaEvent_t next_event();
    template <class F> void timed(Phase ph, cudaStream_t s, F&& f);
    void harvest();

    Plan m_plan;
    frost_boxcar_config m_cfg;
    int m_device;
    cudaStream_t m_stream = nullptr;
    cudaEvent_t m_order   = nullptr; // orders the caller's stream before the engine's
    long long m_wait_limit = kDefaultWaitLimit;
    // the batch gulp in progress
    const float* m_batch_wf = nullptr;
    SizeType m_batch_nsamps = 0;
    std::vector<uint8_t> m_batch_mask;
    std::vector<uint8_t> m_kill; // the constructor's mask
    bool m_fp16;
    int64_t m_tile = 0, m_ncols = 0;
    // Per stored level: history columns before base (the level's own
    // history, or the search halo for searched levels) and the row pitch.
    std::vector<int32_t> m_base_of;
    std::vector<int64_t> m_pitch_of;
    /** Level h's base column for a tile of ncols columns. */
    int32_t level_base(int h) const;
    SizeType m_nsearch = 0; // searched rows over all planes
    std::vector<int64_t> m_height_g0, m_height_g1; // searched rows per height
    std::vector<int32_t> m_node_first_op;

    DeviceBuffer m_buf[2];
    std::vector<DeviceBuffer> m_hist;
    DeviceBuffer m_in_hist, m_in_scratch, m_wf_stage;
    DeviceBuffer m_leaf_ops, m_node_first_op_d, m_row_ops, m_rows, m_planes, m_widths, m_leaf_len,
        m_leaf_offset, m_gtab, m_var, m_inv, m_inv_or, m_mask_d, m_mask_or_d, m_carry,
        m_row_counts, m_cands, m_counters, m_frontier, m_capture_rows;
    // Candidate ordering: packed keys and their positions (ping-ponged by
    // the radix sort), its digit histograms, the sorted copy and the
    // smallest / largest peak sample of a call.
    DeviceBuffer m_sort_keys[2], m_sort_vals[2], m_sort_hist, m_cands_sorted, m_cand_range;
    // Single level steps fused with the search of their level: the RowOp of
    // each searched row [g], and per height the rows the level kernel still
    // computes (m_fs_rows[m_fs_rows_off[h] ..][m_fs_rows_n[h]]).
    DeviceBuffer m_fs_ops, m_fs_rows;
    std::vector<int64_t> m_fs_rows_off, m_fs_rows_n;
    bool m_fs_on = true;
    int32_t m_fs_buffers = 1;
    int m_key_level_bits = 0, m_key_idx_bits = 0, m_key_dm_bits = 0, m_key_filter_bits = 0;
    std::vector<int64_t> m_row_op_offset;
    /** One FDMT step: level `out` from level `in` = out - 1 (single) or
     * out - 2 (fused: the level between is never stored). Step 0 is level 1
     * from the input. */
    struct Step {
        int out, in;
        bool fused;
        int64_t op_offset; // into m_row_ops (single) or m_fused_ops (fused)
    };
    std::vector<Step> m_steps;
    /** The step's level is searched in the same pass (fused single step). */
    bool fused_search(const Step& st) const {
        return m_fs_on && !st.fused && st.out >= 2 && m_height_g1[st.out] > m_height_g0[st.out] &&
               search_halo(m_plan.widths().back()) <= m_search_chunk;
    }
    std::vector<int> m_buf_of;         // level -> level buffer (-1: not stored)
    std::vector<int32_t> m_hist_len;   // level -> history columns kept
    struct Schedule {
        std::vector<Step> steps;
        std::vector<int> buf_of;
        std::vector<int32_t> hist_len;
        std::vector<FusedOp> fused;
    };
    /** The FDMT schedule of `plan` (host only): steps, the buffer of every
     * stored level, history lengths and the fused ops. */
    static Schedule make_schedule(const Plan& plan, const std::vector<int64_t>& row_op_offset, bool fuse);
    static void validate(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc, const Plan& plan);
    DeviceBuffer m_fused_ops;
    bool m_fuse        = true; // fused two-level steps in the schedule
    int32_t m_level_tpc = 16;  // tiles of 2048 columns per level-kernel CTA
    int32_t m_level2_stages = 0; // bulk-copy stages of the fused kernel (0: its default)
    int32_t m_search_chunk  = kSearchChunk; // samples per search-kernel step
    void build_schedule(bool fuse);
    void apply_shape(bool fuse, int32_t tpc, int32_t stages, int32_t chunk);
    SizeType m_budget = 0; // device memory budget of the plan
  public:
    struct Tuned {
        bool fuse;
        int32_t tiles_per_cta;
        int32_t stages; // fused kernel's stages (0 = default or not fused)
        int32_t search_chunk;
        double ms;   // one tile pass with the choice (0 if taken from the cache)
        bool cached;
    };
    /** Measures the FDMT launch shapes for this geometry, applies the fastest
     * and restarts the stream (call before the first gulp). */
    Tuned autotune();
    /** Pins a launch shape (as autotune would set it) and restarts the
     * stream (call before the first gulp). */
    void set_launch_shape(bool fuse, int32_t tiles_per_cta, int32_t stages, int32_t search_chunk);
    Tuned launch_shape() const;
    /** Caps the level and search kernels at `ctas_per_sm` resident CTAs per
     * SM, each CTA looping over work items (0: one CTA per work item). The
     * rest of every SM stays free for other streams' kernels (the served
     * beams' kernels overlap); results do not depend on it. */
    void set_residency(int32_t ctas_per_sm);
    int32_t residency() const { return m_ctas_per_sm; }
    /** Fuses each single level step into a searched level with its search
     * (mode 0: off; 1 or 2: on, that many chunks staged at once); identical
     * results. Waits for the engine's stream. */
    void set_fused_search(int32_t mode);
    int32_t fused_search_mode() const { return m_fs_on ? m_fs_buffers : 0; }

    /** Device bytes an engine for (dd, bc) allocates, computed on the host
     * from its plan without allocating anything: level buffers (under
     * either schedule autotune may try), histories, tables, candidates, and
     * autotune's transient zero waterfall. Throws what the constructor
     * throws for an invalid configuration. */
    struct Footprint {
        SizeType level_bytes = 0, history_bytes = 0, table_bytes = 0, candidate_bytes = 0;
        SizeType transient_bytes = 0;
        int32_t dt_max           = 0;
        SizeType total() const { return level_bytes + history_bytes + table_bytes + candidate_bytes; }
    };
    static Footprint estimate(const frost_dedisp_plan_config& dd, const frost_boxcar_config& bc);
  private:
    int32_t m_ctas_per_sm = 0;
    int32_t m_sms         = 0;
    /** CTA cap of a launch (0: none). */
    int32_t cta_cap() const { return m_ctas_per_sm > 0 ? m_sms * m_ctas_per_sm : 0; }
    std::vector<DeviceBuffer> m_capture;
    bool m_capture_on = false;
    int64_t m_capture_cols = 0;

    std::vector<uint8_t> m_mask;     // mask of the previous gulp (FDMT order)
    std::vector<uint8_t> m_var_mask, m_var_mask_or;
    bool m_var_ready = false;
    uint64_t m_samples = 0;          // absolute samples processed
    std::vector<frost_candidate> m_results;
    uint64_t m_dropped_global = 0, m_dropped_per_dm = 0;
    uint64_t m_launches = 0;
    int32_t m_max_len = 1;

    SizeType plan_bytes(int64_t tile) const;
    void allocate(int64_t tile);
    SearchParams params(int64_t tile_off, int32_t n_valid) const;
    /** The per-gulp launch sequence (memsets, every tile's FDMT steps,
     * history copies and searches) for a waterfall at `wf`. */
    void run_tiles(const float* wf, SizeType nsamps, cudaStream_t s);
    // The sequence captured as a CUDA graph, replayed while the waterfall
    // address and length stay the same (timing and plane capture launch
    // directly).
    cudaGraphExec_t m_graph     = nullptr;
    const float* m_graph_wf     = nullptr;
    SizeType m_graph_nsamps     = 0;
    uint64_t m_graph_launches   = 0;
    bool m_graphs_on            = true;
    DeviceBuffer m_clock;       // GulpClock read by the search
    PinnedBuffer m_clock_h;
  public:
    /** Enables (default) or disables graph capture of the launch sequence. */
    void use_graphs(bool on) { m_graphs_on = on; }
  private:
    LevelView view(int h) const;
    void update_variance(const std::vector<uint8_t>& cur, const std::vector<uint8_t>& orm);
    void collect(cudaStream_t s);
};

} // namespace fb::fdmt
