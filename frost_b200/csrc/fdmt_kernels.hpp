// Launchers of the FDMT level kernels and the boxcar/trapezoid search
// (fdmt_kernels.cu, search_kernels.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime_api.h>

#include "fdmt_plan.hpp"

namespace fb::fdmt {

/** A level buffer: rows of `pitch` elements; time t of the current tile is
 * column `base + t`, its history occupies columns [base - H, base). */
struct LevelView {
    void* data;
    int64_t pitch;
    int32_t base;
    int32_t fp16; // element type: 0 float, 1 __half
};

constexpr int kTimePerCta = 2048; // samples per CTA in the level kernels

/** One level step of one engine as a segment of a pipelined level launch:
 * output rows [0, nrows) of `out` from `in` by its ops (RowOp for single
 * levels, FusedOp for fused steps), each row cut into runs of `tpc` of
 * `ntiles` time tiles. A launch covers several segments (the same step of
 * several beams) in one grid; item_end is filled by the launcher. */
struct LevelSeg {
    const void* ops;
    const void* in;
    void* out;
    int64_t in_pitch;
    int64_t out_pitch;
    int32_t in_base;
    int32_t out_base;
    int32_t ntiles;
    int32_t tpc;
    int64_t nrows;
    int64_t item_end;
    unsigned* err;
    // single levels: output rows rows[0 .. nrows) of the level (their ops
    // ops[rows[i]]); nullptr: rows 0 .. nrows - 1
    const int32_t* rows;
};
constexpr int kMaxLevelSegs = 48;
template <int K> struct LevelSegTable {
    int32_t n;
    int32_t pad;
    LevelSeg s[K];
};
/** Tries a pipelined kernel's first wait on a bulk copy makes before it
 * gives up (bulk::kSpinLimit); a drain after a give-up always uses it. */
constexpr long long kDefaultWaitLimit = 1LL << 22;

/* Residency: every level launcher takes `ctas`, the most CTAs of the launch
 * (0: one CTA per work item). With a cap each CTA loops over work items, so
 * a launch holds at most `ctas` CTAs' resources and leaves the rest of the
 * GPU to other streams' kernels; results do not depend on it. */

/** Level 1 straight from the input channels: each row is the sum of two
 * leaf windows read from the waterfall (columns t0 .. t0 + n_valid) and,
 * for times before the tile, the input history [C][hist_len]. */
void launch_level1(const LeafOp* ops, const int32_t* node_first_op, int32_t nnodes,
                   int32_t max_node_delay, const float* waterfall, int64_t waterfall_pitch,
                   int64_t t0, int32_t n_valid, const float* input_hist, int32_t hist_len,
                   LevelView out, int32_t ncols, cudaStream_t s, int32_t ctas = 0);

/** Level h >= 2: out[row] = in[lo] + in[hi] shifted (only the rows
 * row_map[0 .. nrows) when a map is given; the pipelined kernel only). With `err` non-null
 * the TMA-pipelined kernel runs (each CTA takes `tiles_per_cta` tiles of
 * 2048 columns) and sets *err if a bounded wait ran out; with `err` null
 * the direct (one CTA per row and tile) kernel runs. */
void launch_level(const RowOp* ops, int64_t nrows, LevelView in, LevelView out, int32_t ncols,
                  unsigned* err, cudaStream_t s, int32_t tiles_per_cta = 16, int32_t ctas = 0,
                  long long wait_limit = kDefaultWaitLimit, const int32_t* row_map = nullptr);

/** A row of level h+1 from four rows of level h-1: the sum of row[j] read at
 * t - shift[j] (shift[0] = 0), grouped (row0 + row1) + (row2 + row3); a
 * negative row[j] is absent (pass-through nodes). */
struct FusedOp {
    int32_t row[4];
    int32_t shift[4];
};

/** Level h+1 straight from level h-1 (TMA-pipelined; *err set if a bounded
 * wait ran out). `stages` tiles in flight per CTA (2, 3 or 4; 4 only with
 * fp16 storage; 0 = 4 for fp16, 3 for float): fewer stages leave room for
 * more CTAs per SM. */
void launch_level2(const FusedOp* ops, int64_t nrows, LevelView in, LevelView out, int32_t ncols,
                   unsigned* err, cudaStream_t s, int32_t tiles_per_cta = 16, int32_t stages = 0,
                   int32_t ctas = 0, long long wait_limit = kDefaultWaitLimit);

/** One pipelined launch over `n` level segments of the same kind (fused
 * or single), element type and stage count; more than kMaxLevelSegs
 * segments take several launches. `ctas` caps each launch's CTAs. */
void launch_level_segs(LevelSeg* segs, int n, bool fused, bool fp16, int32_t stages, cudaStream_t s,
                       int32_t ctas = 0, long long wait_limit = kDefaultWaitLimit);

/** dst[r][0 .. width) = src[r][0 .. width) for `rows` rows of pitches
 * dpitch / spitch bytes (device memory): 16-byte vectors when pointers,
 * pitches and width allow, cudaMemcpy2DAsync otherwise. */
void copy_rows(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows,
               cudaStream_t s);

/** Copies the last `hist` columns ending at column base + n_valid of every
 * row of `view` into hist_buf[rows][hist]. */
void launch_save_history(LevelView view, int64_t rows, int32_t hist, int32_t n_valid,
                         void* hist_buf, cudaStream_t s);

/** Copies hist_buf[rows][hist] into columns [base - hist, base). */
void launch_load_history(LevelView view, int64_t rows, int32_t hist, const void* hist_buf,
                         cudaStream_t s);

/** Copies level rows `rows[0..nrows)` (tile columns [0, n_valid)) to
 * out[i][t_off + k] as float. */
void launch_capture_rows(LevelView view, const int64_t* rows, int64_t nrows, float* out,
                         int64_t out_pitch, int64_t t_off, int32_t n_valid, cudaStream_t s);

/** Input history update: last hist columns of (old history ++ waterfall
 * columns [t0, t0 + n_valid)). */
void launch_save_input_history(const float* waterfall, int64_t pitch, int64_t t0, int32_t n_valid,
                               int32_t nchans, float* hist, float* scratch, int32_t hist_len,
                               cudaStream_t s);

} // namespace fb::fdmt
