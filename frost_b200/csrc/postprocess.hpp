// Candidate post-processing on the device: the state of
// CandidatePostprocessPlan (lib/search/postprocess.cpp:48-260) and the
// standalone ClusterLabelPlan / MergeCandidatesPlan / SubbandDedupPlan.
#pragma once

#include <cstdint>
#include <utility>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.hpp"
#include "frost_b200.h"
#include "postprocess_kernels.hpp"

namespace fb::pp {

/** Device scratch of the post-processing passes, sized for `rows` rows. */
class Workspace {
public:
    void reserve(size_t rows);
    size_t capacity() const { return m_rows; }
    SizeType bytes() const;

    /** Stable sort of rows[0, n) by `fields` (least significant first, each
     * with its inclusive value range); ties keep the row order. Returns the
     * sorted row permutation and the final (most significant group's) keys,
     * both in this workspace's sort buffers until the next sort. */
    struct Field {
        int kind;
        u64 lo, hi;
    };
    std::pair<const u32*, const u64*> sort(const frost_giant* rows, size_t n, const std::vector<Field>& fields,
                                           const u32* aux32, const u64* aux64, const u32* keep,
                                           cudaStream_t s);

    /** Min/max of each kind over rows[0, n) (kept rows only); synchronises. */
    std::vector<std::pair<u64, u64>> ranges(const frost_giant* rows, size_t n, const std::vector<int>& kinds,
                                            const u32* aux32, const u64* aux64, const u32* keep,
                                            cudaStream_t s);

    /** Exclusive scan; returns the total (synchronises). */
    u32 scan(const u32* in, u32* out, size_t n, cudaStream_t s);

    // Row-sized scratch.
    DeviceBuffer keys[2], perm[2], hist, tile_sums, u32a, u32b, u32c, u32d, u32e, u32f, u64a, u64b, small;
    PinnedBuffer host_small;

private:
    size_t m_rows = 0;
};

/** ClusterLabelPlan::execute on device rows (labels as u32 row indices). */
void cluster_labels(Workspace& ws, const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol,
                    int mode, u32* label, cudaStream_t s);

/** MergeCandidatesPlan::execute with arbitrary 64-bit labels; returns the
 * group count (rows written to out in ascending label order). */
size_t merge_candidates(Workspace& ws, const frost_giant* rows, const u64* labels, size_t n, frost_giant* out,
                        cudaStream_t s);

/** SubbandDedupPlan::execute; returns the row count written to out. */
size_t subband_dedup(Workspace& ws, const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol,
                     float tsamp, int mode, frost_giant* out, cudaStream_t s);

class PostprocessPlan {
public:
    PostprocessPlan(const frost_postprocess_config& cfg, const frost_postprocess_layout& layout, int device);
    ~PostprocessPlan();
    PostprocessPlan(const PostprocessPlan&)            = delete;
    PostprocessPlan& operator=(const PostprocessPlan&) = delete;

    /** CandidatePostprocessPlan::execute over n raw rows (device or host). */
    frost_postprocess_result execute(const frost_candidate* cands, size_t n, bool on_device, u64 samples_read,
                                     u64 duration_samples, bool final_call, u64 candidate_frontier);

    const std::vector<frost_giant>& results() const { return m_results; }
    u64 memory_usage() const;
    static u64 estimate_memory(const frost_postprocess_config& cfg);
    int device() const { return m_device; }
    cudaStream_t stream() const { return m_stream; }

private:
    frost_cluster_tolerances tolerances() const;
    u64 pending_limit() const;

    frost_postprocess_config m_cfg;
    frost_postprocess_layout m_lay;
    int m_device;
    cudaStream_t m_stream = nullptr;
    size_t m_rows         = 0; // max_candidates + pending limit
    Workspace m_ws;
    DeviceBuffer m_raw, m_in, m_inc, m_work, m_merged, m_reduced, m_ready, m_out, m_pend[2], m_segs;
    DeviceBuffer m_cols, m_parent, m_label, m_ord, m_gmap, m_rmap, m_flag, m_pos, m_first, m_best, m_sum,
        m_seg_of, m_mseg, m_tord, m_sord, m_rank, m_bounds, m_bitmap;
    PinnedBuffer m_host_segs, m_host_small;
    int m_cur = 0; // m_pend[m_cur] holds the carried rows
    size_t m_npending = 0;
    std::vector<std::pair<u64, u32>> m_pend_runs; // (plane, rows) in plane order
    u64 m_pend_samp_lo = ~u64{0}, m_pend_samp_hi = 0;
    std::vector<frost_giant> m_results;
};

} // namespace fb::pp
