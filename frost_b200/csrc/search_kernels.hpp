// Boxcar/trapezoid matched-filter search with exact per-DM/width noise and
// run-based peak finding (search_kernels.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime_api.h>

#include "fdmt_kernels.hpp"
#include "frost_b200.h"

namespace fb::fdmt {

/** Samples per search chunk; level tiles are a whole number of chunks. */
constexpr int kSearchChunk = 4096;
/** Column granularity of a level-buffer tile. */
constexpr int kTileQuantum = kSearchChunk > kTimePerCta ? kSearchChunk : kTimePerCta;

/** Columns before a search chunk that the search stages: the widest boxcar
 * rounded up to whole 256-column segments. Level buffers keep at least this
 * many history columns. */
constexpr int32_t search_halo(int32_t wmax) { return (wmax + 255) / 256 * 256; }

/** One searched row: a DM trial of one plane. */
struct SearchRow {
    int64_t level_row; // row in its level buffer
    int32_t plane;
    int32_t prow;      // index in the plane's DM grid (dm_idx)
    int32_t delay;     // warm-up samples of the row
    float dm;
};

/** Per-plane constants copied into every candidate. */
struct PlaneInfo {
    float f_low, f_high;
    uint32_t chan_begin, chan_end;
    uint32_t subband_level, subband_idx;
};

/** Open above-threshold run carried across chunks, tiles and gulps. */
struct RunState {
    int32_t open;
    int32_t best_w;
    float best;
    int32_t pad;
    int64_t start;
    int64_t best_t;
    int64_t last_t;
};

/** The per-gulp times the search reads from device memory, so that one
 * captured launch sequence (a CUDA graph) serves every gulp. */
struct GulpClock {
    int64_t gulp_t0;   // absolute sample of the gulp's first column
    int32_t or_active; // this gulp's mask differs from the previous one
    int32_t pad;
};

struct SearchParams {
    const SearchRow* rows;   // indexed by global searched-row g
    const PlaneInfo* planes;
    const int32_t* widths;
    int32_t nwidths;
    int32_t wmax;
    int32_t halo;            // search_halo(wmax)
    float thresh;
    int32_t peak_mode;       // enum frost_peak_mode
    int32_t trapezoid;
    int32_t skip_cold;
    int32_t pow2_widths;     // the widths are 1, 2, 4, ... (read by the launcher)
    const GulpClock* clock;  // gulp start and mask change (device)
    int64_t tile_off;        // tile column 0 relative to the gulp start
    int32_t n_valid;         // valid columns in this tile
    const float* inv_sigma;  // [g][nwidths]
    const float* inv_sigma_or;
    RunState* carry;         // [g][nwidths] (per width) or [g] (across widths)
    frost_candidate* cands;
    unsigned long long* ncands;
    uint64_t max_cands;
    uint32_t* row_counts;    // [g]
    uint32_t max_per_dm;     // 0 = unlimited
    unsigned long long* dropped; // [0] global, [1] per DM
    unsigned* err;           // set when a bounded wait for staged data ran out
    long long wait_limit;    // tries of a chunk's first wait (a drain uses kSpinLimit)
};

/** One engine's search of rows [g0, g0 + nrows) of one level as a segment
 * of a search launch; a launch covers the segments of several beams whose
 * search shape (widths, halo, peak mode, trapezoid, cold prefix, valid
 * columns) is the same. row_end is filled by the launcher. */
struct SearchSeg {
    SearchParams p;
    const void* level;
    int64_t pitch;
    int32_t base;
    int32_t fp16;
    int64_t g0;
    int64_t nrows;
    int64_t row_end;
    // Fused single level step (in != nullptr): each searched row of `level`
    // is computed in the same pass from the level below, out = in[lo] +
    // in[hi] shifted by its op (ops[g] for searched row g), written to
    // `level` and searched; its halo columns are already in `level`.
    const void* in;
    int64_t in_pitch;
    int32_t in_base;
    int32_t fs_buffers; // chunks staged at once: 1 or 2 (two: fewer CTAs an SM)
    const RowOp* ops;
};
constexpr int kMaxSearchSegs = 32;
template <int K> struct SearchSegTable {
    int32_t n;
    int32_t pad;
    SearchSeg s[K];
};

/** One launch (or one per kMaxSearchSegs) over `n` search segments of the
 * same shape and element type. */
void launch_search_segs(SearchSeg* segs, int n, cudaStream_t s, int32_t chunk = kSearchChunk, int32_t ctas = 0);

/** Searches rows [g0, g1) (all in `level`) over the tile's valid columns,
 * `chunk` (2048 or 4096) samples per step of a CTA: the smaller chunk needs
 * half the shared memory and fewer registers, so more CTAs fit an SM, at
 * the cost of a larger halo share. `ctas` caps the launch's CTAs, each then
 * looping over rows (0: one CTA per row). */
void launch_search(const SearchParams& p, LevelView level, int64_t g0, int64_t g1,
                   cudaStream_t s, int32_t chunk = kSearchChunk, int32_t ctas = 0);

/** launch_search with the single level step into `level` fused: searched
 * row g is first computed from `in` by ops[g] (the step's RowOp of its
 * level row) and written to `level`; `buffers` (1 or 2) chunks are staged
 * at once. The halo must not exceed the chunk. */
void launch_search_fused(const SearchParams& p, LevelView in, LevelView level, const RowOp* ops, int64_t g0,
                         int64_t g1, cudaStream_t s, int32_t chunk = kSearchChunk, int32_t ctas = 0,
                         int32_t buffers = 1);

/** Exact variance of every searched row and width for `mask` and for
 * `mask_or`: var = sum over active channels of g[L_c][w]; writes
 * inv_sigma = 1/sqrt(var) (0 where var = 0) and the FP64 variances. */
void launch_variance(const SearchRow* rows, const PlaneInfo* planes, const int64_t* leaf_offset,
                     const uint16_t* leaf_len, int64_t nrows, const double* gtab,
                     int32_t max_len, int32_t nwidths, const uint8_t* mask,
                     const uint8_t* mask_or, double* var, float* inv_sigma, float* inv_sigma_or,
                     cudaStream_t s);

/** Emits every open run as a candidate and closes it (drain). */
void launch_flush_runs(const SearchParams& p, int64_t nrows, cudaStream_t s);

/** Bit widths of the packed candidate order key (level, sub-band, DM row,
 * peak - peak_base, width index; most significant first). */
struct CandKeySpec {
    uint64_t peak_base;
    int idx_bits, dm_bits, peak_bits, filter_bits;
};

/** range[0] = smallest, range[1] = largest peak sample of the first
 * min(*count, cap) candidates (~0 and 0 when there are none). */
void launch_cand_range(const frost_candidate* c, const unsigned long long* count, uint64_t cap,
                       unsigned long long* range, cudaStream_t s);
/** keys[i] = packed order key of c[i], idx[i] = i. */
void launch_cand_keys(const frost_candidate* c, uint64_t n, const CandKeySpec& k, uint64_t* keys,
                      uint32_t* idx, cudaStream_t s);
/** out[i] = c[perm[i]]. */
void launch_cand_gather(const frost_candidate* c, const uint32_t* perm, uint64_t n, frost_candidate* out,
                        cudaStream_t s);

} // namespace fb::fdmt
