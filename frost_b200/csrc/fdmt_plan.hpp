// Streaming FDMT plan: the sub-band tree, the delay rows each node must
// produce, the per-level merge operations, the search planes (full band,
// halves, quarters and the staggered bands across their boundaries) and the
// per-row leaf windows that give the exact noise of every DM, width and mask.
//
// Zackay & Ofek (2017) restated for frost's contracts (the dmt library frost
// links is not available, so its delay rounding is not reproduced; this plan
// fixes its own and the oracle restates the same rule independently):
//
//   * channels are the C equal bins of [f_min, f_max] (ascending);
//   * K(a, b) = a^-2 - b^-2; the delay of a band [a, b] at DM is
//     kDispConst * DM * K(a, b) / tsamp samples, rounded to nearest;
//   * a node [a, b) splits at mid = a + n/2 into low [a, mid) and high
//     [mid, b); a row of delay d takes d_hi = round(d K(f_mid, f_hi) /
//     K(f_lo, f_hi)) from the high child and d_lo = d - d_hi from the low;
//     out[d][t] = low[d_lo][t] + high[d_hi][t - d_lo] (time referenced to
//     the bottom of the node's band);
//   * a single channel c with row d is the window sum
//     sum_{j=0..d} I[c][t - j];
//   * every output row is therefore sum_c sum_{j<L_c} I[c][t - s_c - j] with
//     each input cell at most once: for unit-variance independent input its
//     width-W (boxcar or trapezoid) window has variance
//     sum_{c active} g(L_c, W), g = sum of squared window-box multiplicities.
#pragma once

#include <cstdint>
#include <vector>

#include "common.hpp"

namespace fb::fdmt {

constexpr double kDispConst = 4.148808e3; // s MHz^2 cm^3 / pc

struct Node {
    int32_t chan_begin = 0, chan_end = 0; // [begin, end) in FDMT (ascending) order
    int32_t lo = -1, hi = -1;             // children; hi = -1 with lo >= 0: pass-through
    int32_t height    = 0;                // 0 for single channels
    int32_t staggered = 0;
    double f_lo = 0, f_hi = 0, f_mid = 0;
    std::vector<int32_t> delays;          // rows, ascending distinct delays
    int64_t row_offset = 0;               // first row in its level buffer

    bool leaf() const { return lo < 0; }
    int32_t row_of(int32_t d) const;       // index of delay d in `delays`
};

/** One output row of a level >= 2: out = in[lo] + in[hi] shifted by `shift`. */
struct RowOp {
    int32_t lo_row;
    int32_t hi_row; // -1: copy of lo_row
    int32_t shift;  // d_lo
    int32_t delay;
};

/** One output row of level 1, computed from the input channels. */
struct LeafOp {
    int32_t chan_lo;
    int32_t chan_hi; // -1: single channel window
    int32_t d_lo;    // window of chan_lo: [t - d_lo, t]
    int32_t d_hi;    // window of chan_hi: [t - d_lo - d_hi, t - d_lo]
};

struct Plane {
    int32_t node           = 0;
    int32_t height         = 0;
    int32_t subband_level  = 0;
    int32_t subband_idx    = 0;
    int32_t staggered      = 0;
    int32_t chan_begin     = 0, chan_end = 0;
    double f_lo = 0, f_hi = 0;
    std::vector<int64_t> level_row; // row index in the level buffer, per searched row
    std::vector<int32_t> delay;     // per searched row (= warm-up samples)
    std::vector<float> dm;          // DM per searched row
    std::vector<int32_t> dm_index;  // first index in the DM list per searched row
};

struct PlanConfig {
    uint64_t nchans      = 0;
    double f_min         = 0, f_max = 0; // band edges, MHz
    double tsamp         = 0;            // seconds
    uint64_t block_nsamps = 0;
    uint64_t subband_depth = 0;
    uint64_t max_boxcar  = 1;
    float wtsp           = 2.0F;
    std::vector<float> dm_list;
};

class Plan {
public:
    explicit Plan(PlanConfig cfg);

    const PlanConfig& config() const { return m_cfg; }
    int32_t nchans() const { return static_cast<int32_t>(m_cfg.nchans); }
    int32_t dt_max() const { return m_dt_max; }
    int32_t levels() const { return m_levels; } // highest height
    const std::vector<Node>& nodes() const { return m_nodes; }
    int32_t root() const { return m_root; }
    const std::vector<Plane>& planes() const { return m_planes; }
    const std::vector<int32_t>& widths() const { return m_widths; }
    const std::vector<int32_t>& final_delays() const { return m_final_delays; }

    /** Rows of the level-h buffer (h >= 1). */
    int64_t level_rows(int h) const { return m_level_rows[h]; }
    /** History samples level h must keep for its consumers (h = 0: input). */
    int32_t level_history(int h) const { return m_level_hist[h]; }
    const std::vector<LeafOp>& leaf_ops() const { return m_leaf_ops; }
    const std::vector<RowOp>& row_ops(int h) const { return m_row_ops[h]; }
    int64_t max_level_rows() const;
    int32_t max_history() const;

    /** Leaf window length L_c = delay + 1 of every channel of every searched
     * row of plane p, [row][channel - chan_begin]. */
    std::vector<uint16_t> leaf_lengths(int p) const;
    int32_t max_leaf_length() const { return m_max_leaf_len; }

    /** Channel frequency edge c (0..C) in MHz. */
    double edge(int64_t c) const;
    static double K(double a, double b) { return 1.0 / (a * a) - 1.0 / (b * b); }
    int32_t band_delay(double dm, double f_lo, double f_hi) const;

private:
    PlanConfig m_cfg;
    std::vector<Node> m_nodes;
    int32_t m_root   = 0;
    int32_t m_levels = 0;
    int32_t m_dt_max = 0;
    int32_t m_max_leaf_len = 1;
    std::vector<int32_t> m_final_delays;
    std::vector<int32_t> m_widths;
    std::vector<Plane> m_planes;
    std::vector<int64_t> m_level_rows;
    std::vector<int32_t> m_level_hist;
    std::vector<LeafOp> m_leaf_ops;
    std::vector<std::vector<RowOp>> m_row_ops;

    int32_t build_tree(int32_t begin, int32_t end);
    int32_t wrap(int32_t node, int32_t height);
    void split_delay(const Node& n, int32_t d, int32_t& d_lo, int32_t& d_hi) const;
    void descend(int32_t node, int32_t d, uint16_t* out, int32_t base) const;
};

/** Widths 1, then max(ceil(wtsp * w), w + 1) up to max_boxcar. */
std::vector<int32_t> box_widths(uint64_t max_boxcar, float wtsp);

/** Sum of squared multiplicities of a width-W window (boxcar, or trapezoid
 * with half-weight edges of (W + 1) / 4 samples for W >= 3) convolved with a
 * length-L box. */
double window_box_variance(int32_t L, int32_t W, bool trapezoid);

} // namespace fb::fdmt
