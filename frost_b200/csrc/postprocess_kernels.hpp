// Launchers of the candidate post-processing kernels
// (postprocess_kernels.cu). Every launcher is asynchronous on `s`; all
// pointers are device pointers. Row indices are 32-bit: one call handles
// fewer than 2^32 rows.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime_api.h>

#include "frost_b200.h"

namespace fb::pp {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

/** Kernels launched by this file's launchers in this process. */
u64 launch_counter();

/** Rows per radix tile (256 threads x 8 rows). */
constexpr size_t kTile = 2048;

/** Sort-key fields, read from a frost_giant row (or an auxiliary column). */
enum KeyKind : int {
    kKeyPlane    = 0,
    kKeyDmIdx    = 1,
    kKeyFilter   = 2,
    kKeySamp     = 3,
    kKeySnrDesc  = 4, // descending S/N (order-preserving float bits, inverted)
    kKeySpanDesc = 5, // descending channel span
    kKeyAux32    = 6, // aux32[row]
    kKeyAux64    = 7, // aux64[row]
    kKeyDropped  = 8, // 1 for rows with keep[row] == 0
};

struct KeyField {
    int kind;
    int shift;
    u64 lo;
};

/** Up to four fields packed into one 64-bit key: sum of
 * (value - lo) << shift. */
struct KeySpec {
    int n;
    KeyField f[4];
};

struct RangeKinds {
    int n;
    int kind[8];
};

/** Per-row columns of the friends-of-friends sweep, in time order. */
struct Columns {
    uint4* key; // (samp - samp_lo, width, dm_idx, filter_idx) when they fit 32 bits
    u64* samp;
    u64* width;
    u64* dm_idx;
    u64* filter;
    u64* cb;
    u64* ce;
    u64* plane;
    float* dm;
    float* snr;
    float* flo;
    float* fhi;
    u32* idx;     // row index in the clustered array
    u32* seg;     // segment (plane) of the row
    u32* minidx;  // per rank root: smallest row index of its component
    u32* general; // one word: set when the general sweep must run
};

/** One plane of one execute call. */
struct Seg {
    u64 plane;
    u32 in_start, in_keep, pend_start, pend_cnt, work_start, work_cnt;
};

// ---- generic pieces -------------------------------------------------------

void launch_iota(u32* v, size_t n, cudaStream_t s);

/** Stable sort of (keys, vals) by the low `bits` bits of keys; returns
 * through the references the buffers holding the result (ping-ponged with
 * the *_alt buffers). `hist` holds 256 * ceil(n / kTile) words. */
void radix_sort(u64*& keys, u32*& vals, u64*& keys_alt, u32*& vals_alt, size_t n, int bits, u32* hist,
                cudaStream_t s);

/** keys[i] = spec(rows[perm[i]]). `keep` (optional) marks kept rows: the
 * other rows take lo for every field and 1 for kKeyDropped. */
void launch_keys(const frost_giant* rows, const u32* perm, size_t n, const KeySpec& spec, const u32* aux32,
                 const u64* aux64, const u32* keep, u64* keys, cudaStream_t s);

/** Per kind: min and max over kept rows (out[2k] = min, out[2k+1] = max;
 * the caller sets them to ~0 and 0 first). */
void launch_ranges(const frost_giant* rows, size_t n, const RangeKinds& kinds, const u32* aux32,
                   const u64* aux64, const u32* keep, unsigned long long* out, cudaStream_t s);

/** Exclusive scan of n words into out; *total receives the sum.
 * `tile_sums` holds ceil(n / kTile) words. */
void exclusive_scan(const u32* in, u32* out, size_t n, u32* tile_sums, u32* total, cudaStream_t s);

/** dst[i] = src[perm[i]]. */
void launch_gather(const frost_giant* src, const u32* perm, size_t n, frost_giant* dst, cudaStream_t s);

/** dst[pos[i]] = src[i] where flag[i]. */
void launch_compact(const frost_giant* src, const u32* flag, const u32* pos, size_t n, frost_giant* dst,
                    cudaStream_t s);

// ---- ingest ----------------------------------------------------------------

/** Raw detections to giants (postprocess.cpp:79-116): keep[i] = peak inside
 * the read input; first_err = min over invalid kept rows of
 * (index << 1 | kind), kind 0 = channel extent, 1 = beam/width/interval;
 * *nkept counts kept rows. */
void launch_ingest(const frost_candidate* raw, size_t n, u64 samples_read, u64 nchans, int flip,
                   u64 boxcar_max, frost_giant* out, u32* keep, unsigned long long* first_err, u32* nkept,
                   cudaStream_t s);

/** Starts of the runs of equal plane in plane-sorted rows (unordered). */
void launch_plane_runs(const frost_giant* rows, size_t n, u64* run_plane, u32* run_start, u32* nruns,
                       cudaStream_t s);

/** work[w] from the rate-limited incoming rows and the carried rows of
 * each segment; seg_of[w] = its segment. */
void launch_build_work(const frost_giant* inc, const frost_giant* pend, const Seg* segs, int nseg,
                       size_t nwork, frost_giant* work, u32* seg_of, cudaStream_t s);

// ---- friends-of-friends (chain) --------------------------------------------

/** Columns of rows[perm[r]] for r < n (time order); seg from seg_of (or 0
 * if null); segment s starts at rank seg_lo[s] (null: 0). Sets
 * *c.general when the fast sweep cannot take the rows. */
void launch_columns(const frost_giant* rows, const u32* perm, const u32* seg_of, const u32* seg_lo, size_t n,
                    u64 samp_lo, const Columns& c, cudaStream_t s);

/** Unites every coincident pair inside the wider giant's time reach
 * (clustering.cpp:129-183). Segment s occupies ranks
 * [seg_lo[s], seg_hi[s]) (null: one segment [0, n)). parent[] starts as the
 * identity over time ranks. Launches the fast and the general sweep; the
 * one *c.general does not select returns at once. */
void launch_chain(const Columns& c, const u32* seg_lo, const u32* seg_hi, size_t n,
                  const frost_cluster_tolerances& tol, u32* parent, cudaStream_t s);

/** label[idx[r]] = the smallest row index in r's component. c.minidx must
 * hold ~0 (k_columns sets it). */
void launch_rank_labels(u32* parent, const Columns& c, size_t n, u32* label, cudaStream_t s);

/** label[i] = root of i (the smallest index of its component). */
void launch_find_all(u32* parent, size_t n, u32* label, cudaStream_t s);

// ---- seeded clustering ------------------------------------------------------

/** ClusterLabelPlan kSeeded (clustering.cpp:190-224) per segment: rows of
 * segment s are [lo[s], hi[s]), ordered by time in tord and by descending
 * S/N in sord (both segment-major); rank_of[row] = position in tord.
 * label[row] = its seed. `bitmap_words` bounds a segment's rows / 32. */
void launch_seeded(const frost_giant* rows, const u32* tord, const u32* sord, const u32* rank_of,
                   const u32* lo, const u32* hi, int nseg, const frost_cluster_tolerances& tol, u32* label,
                   u32* gbitmap, size_t bitmap_words, cudaStream_t s);

/** rank_of[perm[r]] = r. */
void launch_invert(const u32* perm, size_t n, u32* rank_of, cudaStream_t s);

/** Segment bounds of seg-major rows: lo[seg_of[i]] = min i, hi = max i + 1
 * (lo preset to ~0, hi to 0). */
void launch_seg_bounds(const u32* seg_of, size_t n, u32* lo, u32* hi, cudaStream_t s);

// ---- merge -------------------------------------------------------------------

/** flag[i] = (label[i] == i). */
void launch_root_flags(const u32* label, size_t n, u32* flag, cudaStream_t s);

/** MergeCandidatesPlan over labels that are row indices with
 * label[label[i]] == label[i]: ord[] = exclusive scan of the root flags.
 * Accumulates per group (g = ord[label[i]]) the first member, the packed
 * best (S/N, lowest index) and the member sum; gmap[i] = g. The caller
 * presets first to ~0 and best/sum to 0. */
void launch_merge_accum(const frost_giant* rows, const u32* label, const u32* ord, size_t n,
                        unsigned long long* best, u32* first, unsigned long long* sum, u32* gmap,
                        cudaStream_t s);

/** out[g] = the group's winner (merge.cpp:16-29) with members = the sum;
 * seg_out[g] = seg_of[first[g]] when both are given. */
void launch_merge_emit(const frost_giant* rows, size_t ngroups, const unsigned long long* best,
                       const u32* first, const unsigned long long* sum, const u32* seg_of, u32* seg_out,
                       frost_giant* out, cudaStream_t s);

/** Labels of arbitrary 64-bit values, sorted (perm): ordv[perm[k]] = rank
 * of its distinct value; heads[k] = 1 at the first row of each value. */
void launch_heads(const u64* sorted_keys, size_t n, u32* heads, cudaStream_t s);
void launch_scatter_ord(const u32* perm, const u32* excl, const u32* heads, size_t n, u32* ordv,
                        cudaStream_t s);
/** counts[seg_of[i]] += flag[i]. */
void launch_seg_counts(const u32* flag, const u32* seg_of, size_t n, u32* counts, cudaStream_t s);
/** label[i] = i for identity-ordinal merges over ordv: accumulates like
 * launch_merge_accum with g = ordv[i]. */
void launch_merge_accum_ord(const frost_giant* rows, const u32* ordv, size_t n, unsigned long long* best,
                            u32* first, unsigned long long* sum, cudaStream_t s);

// ---- retention ----------------------------------------------------------------

/** recent[rmap[gmap[w]]] = 1 where work[w].end >= watermark (rmap null:
 * identity). */
void launch_recent(const frost_giant* work, size_t n, const u32* gmap, const u32* rmap, u64 watermark,
                   u32* recent, cudaStream_t s);
/** pflag[w] = recent[rmap[gmap[w]]] (0 when final). */
void launch_pending_flags(size_t n, const u32* gmap, const u32* rmap, const u32* recent, int final_call,
                          u32* pflag, cudaStream_t s);
/** rflag[g] = final || !recent[g]. */
void launch_ready_flags(size_t n, const u32* recent, int final_call, u32* rflag, cudaStream_t s);

// ---- sub-band dedup -------------------------------------------------------------

/** Transitive dedup: unites every pair i < j on one dispersion curve. */
void launch_dedup_pairs(const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol, float tsamp,
                        u32* parent, cudaStream_t s);

/** Seeded dedup: fm[k] = the first m < k with on_same_curve(order[m],
 * order[k]), else k. */
void launch_first_match(const frost_giant* rows, const u32* order, size_t n,
                        const frost_cluster_tolerances& tol, float tsamp, u32* fm, cudaStream_t s);
/** group_of[order[k]] = order[root of k's match chain]; first[group] =
 * min member (preset ~0). */
void launch_resolve_seeded(const u32* order, const u32* fm, size_t n, u32* group_of, u32* first,
                           cudaStream_t s);
/** label[i] = first[group_of[i]]. */
void launch_relabel(const u32* group_of, const u32* first, size_t n, u32* label, cudaStream_t s);

/** Group starts in the label-sorted order: gstart[ord[label[perm[k]]]] = k
 * at each head. */
void launch_group_starts(const u32* perm, const u32* label, const u32* ord, size_t n, u32* gstart,
                         cudaStream_t s);

/** One giant per dedup group (subband_dedup.cpp:254-314): members
 * perm[gstart[g] .. gstart[g + 1]) in index order. */
void launch_dedup_emit(const frost_giant* rows, const u32* perm, const u32* gstart, size_t ngroups, size_t n,
                       frost_giant* out, cudaStream_t s);

} // namespace fb::pp
