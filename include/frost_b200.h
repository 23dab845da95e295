/*
 * frost_b200 — C ABI of the B200 (sm_100a) per-gulp search path of frost:
 * RFI excision and normalisation, the DM trial grid, and the streaming
 * FDMT + boxcar/trapezoid search with exact noise.
 *
 * Plain C types only: no C++ or torch types cross this boundary. Every entry
 * point returns an int status (FROST_OK == 0, negative on failure) and never
 * throws; frost_last_error() gives the calling thread's last message.
 * Arguments are validated before any state changes. Handles own their device
 * buffers; device pointers they return stay valid until the next call on the
 * same handle. Device inputs are read in the order of the caller's stream,
 * which must not be NULL (frost refuses the null stream for device input,
 * lib/cuda/device_rfi_detail.cuh:77-83); with host inputs a NULL stream
 * selects the handle's own stream.
 *
 * Reference interfaces each entry point replaces are cited as
 * file:line within pravirkr/frost.
 */
#ifndef FROST_B200_H
#define FROST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status --------------------------------------------------------- */

/* Status codes. The C++ wrapper maps INVALID_ARGUMENT to
 * std::invalid_argument and the rest to std::runtime_error, as frost's
 * FROST_CUDA_CHECK does (lib/cuda/gpu_utils.cuh:13-20). */
enum frost_status {
    FROST_OK                   = 0,
    FROST_ERR_INVALID_ARGUMENT = -1,
    FROST_ERR_OUT_OF_MEMORY    = -2,
    FROST_ERR_DEVICE           = -3,
    FROST_ERR_TIMEOUT          = -4,
    FROST_ERR_STATE            = -5,
    FROST_ERR_OVERFLOW         = -6,
    FROST_ERR_IO               = -7,
    FROST_ERR_INTERNAL         = -8
};

/* Message of the calling thread's last failing call ("" if none). */
const char* frost_last_error(void);

/* Library version string. */
const char* frost_version(void);

/* ---- common types (include/frost/common/policies.hpp:52-60) ---------- */

enum frost_dtype {
    FROST_UINT1   = 0,
    FROST_UINT2   = 1,
    FROST_UINT4   = 2,
    FROST_UINT8   = 3,
    FROST_UINT16  = 4,
    FROST_UINT32  = 5,
    FROST_FLOAT32 = 6
};

/* Inclusive channel range (include/frost/prepare/rfi.hpp:14-18). */
typedef struct {
    uint64_t start;
    uint64_t end;
} frost_channel_range;

/* Inclusive frequency range in MHz (include/frost/prepare/rfi.hpp:21-25). */
typedef struct {
    double lo;
    double hi;
} frost_frequency_range;

/* ---- RFI excision (include/frost/prepare/rfi.hpp) -------------------- */

enum frost_fill_mode { FROST_FILL_NEIGHBOUR = 0, FROST_FILL_MEAN = 1, FROST_FILL_NOISE = 2 };
enum frost_zero_dm { FROST_ZERO_DM_OFF = 0, FROST_ZERO_DM_SUBTRACT = 1, FROST_ZERO_DM_ZDOT = 2 };

/* Flat form of RfiConfig (include/frost/prepare/rfi.hpp:167-191) with
 * every strategy's switch and thresholds. frost_rfi_config_default() gives
 * the reference defaults (narrow + broad, neighbour fill). Arrays are
 * borrowed for the duration of the create call only. */
typedef struct {
    const frost_channel_range* zap_chans;
    uint64_t n_zap_chans;
    const frost_frequency_range* zap_freqs;
    uint64_t n_zap_freqs;
    int32_t narrow_enabled;
    float narrow_threshold;
    int32_t broad_enabled;
    float broad_threshold;
    uint64_t broad_boxcar_max;
    int32_t dropout_enabled;
    float dropout_min_std_fraction;
    int32_t moments_enabled;
    float moments_threshold;
    int32_t moments_mean;
    int32_t moments_std;
    int32_t moments_skewness;
    int32_t moments_kurtosis;
    int32_t moments_autocorr;
    float moments_kurtosis_max;
    int32_t iqrm_enabled;
    float iqrm_threshold;
    uint64_t iqrm_radius;
    uint64_t mask_grow;
    int32_t kadane_channel_enabled;
    float kadane_channel_threshold;
    float kadane_channel_min_duration;
    int32_t kadane_spectrum_enabled;
    float kadane_spectrum_threshold;
    float kadane_spectrum_min_bandwidth;
    float kadane_spectrum_whole_band_fraction;
    int32_t zero_dm;  /* enum frost_zero_dm */
    int32_t equalize;
    int32_t fill;     /* enum frost_fill_mode */
    uint64_t seed;
} frost_rfi_config;

/* BlockLayout (include/frost/prepare/rfi.hpp:194-201). */
typedef struct {
    uint64_t nchans;
    uint64_t max_nsamps;
    int32_t dtype; /* enum frost_dtype */
    double tsamp;  /* seconds */
    double f0;     /* centre frequency of channel 0, MHz */
    double df;     /* channel spacing, MHz, may be negative */
} frost_block_layout;

/* RfiReport (include/frost/prepare/rfi.hpp:204-227). Stage times are
 * device (CUDA event) seconds. */
typedef struct {
    int32_t calibration_reused;
    uint64_t nsamps;
    uint64_t chans_zapped;
    uint64_t chans_dead;
    uint64_t chans_moments;
    uint64_t chans_iqrm;
    uint64_t chans_grown;
    uint64_t chans_masked;
    uint64_t samps_broad;
    uint64_t samps_dropout;
    uint64_t samps_kadane;
    uint64_t samps_flagged;
    uint64_t cells_narrow;
    uint64_t cells_kadane_spectrum;
    uint64_t cells_kadane_channel;
    uint64_t fill_fallbacks;
    double t_bandpass;
    double t_moments;
    double t_scan;
    double t_flags;
    double t_apply;
} frost_rfi_report;

/* Opaque RFICleaner handle (include/frost/prepare/rfi.hpp:243-297). */
typedef struct frost_rfi frost_rfi;

/* Fills `cfg` with RfiConfig's defaults (include/frost/prepare/rfi.hpp:167-191). */
void frost_rfi_config_default(frost_rfi_config* cfg);

/* RfiConfig::validate (lib/prepare/rfi_config.cpp:14-77). */
int frost_rfi_config_validate(const frost_rfi_config* cfg);

/* RFICleaner(RfiConfig, BlockLayout, baseline_length)
 * (include/frost/prepare/rfi.hpp:250-254, lib/cpu/rfi_cpu.cpp:24-60).
 * Validates configuration and geometry (lib/prepare/rfi_config.cpp:79-110)
 * before allocating device workspace on `device`. */
int frost_rfi_create(const frost_rfi_config* cfg,
                     const frost_block_layout* layout,
                     float baseline_length,
                     int device,
                     frost_rfi** out);

int frost_rfi_destroy(frost_rfi* rfi);

/* RFICleaner::execute_normalized (include/frost/prepare/rfi.hpp:266-282,
 * lib/cpu/rfi_cpu.cpp:161-260): cleans the packed time-major block in float
 * precision on the GPU and writes calibrated float32 in [channel][time]
 * order, low frequency first, `capacity = block_bytes / row_bytes` samples
 * per channel, masked channels and padding zero. `block` is host memory
 * (copied to the device inside the call) when `block_on_device` is 0, else a
 * device pointer, read after the work already queued on `stream` (which
 * must then not be NULL: FROST_ERR_INVALID_ARGUMENT). `nsamps` = 0 uses
 * every row. The device result is returned in `*out_device` (valid until the
 * next call) and is complete when the call returns. */
int frost_rfi_execute_normalized(frost_rfi* rfi,
                                 const uint8_t* block,
                                 size_t block_bytes,
                                 size_t nsamps,
                                 int block_on_device,
                                 void* stream,
                                 const float** out_device);

/* Copies the last normalized waterfall ([nchans][capacity] floats) to host
 * memory; synchronises the stream. */
int frost_rfi_download_normalized(frost_rfi* rfi, float* host, size_t count);

/* RFICleaner::channel_mask (include/frost/prepare/rfi.hpp:284-287). */
int frost_rfi_channel_mask(const frost_rfi* rfi, uint8_t* out, size_t nchans);

/* RFICleaner::report (include/frost/prepare/rfi.hpp:289). */
int frost_rfi_get_report(const frost_rfi* rfi, frost_rfi_report* out);

/* Per-sample time flags of the last full block (1 = flagged), as built by
 * RFICleaner::Impl::build_flags (lib/cpu/rfi_cpu.cpp:347-468). */
int frost_rfi_time_flags(const frost_rfi* rfi, uint8_t* out, size_t nsamps);

/* RFICleaner::memory_usage (include/frost/prepare/rfi.hpp:291): device bytes. */
int frost_rfi_memory_usage(const frost_rfi* rfi, size_t* bytes);

/* Kernels this cleaner has launched since it was created. */
int frost_rfi_launch_count(const frost_rfi* rfi, uint64_t* launches);

/* No counterpart in the reference. The cleaner's own stream (a
 * cudaStream_t): a caller that writes a device block on it, or that hands
 * the normalised waterfall to frost_search_execute, passes it as `stream`. */
int frost_rfi_get_stream(const frost_rfi* rfi, void** stream);

/* No counterpart in the reference. An allocation-free form of
 * frost_rfi_execute_normalized for callers that cannot call cudaMalloc once
 * they are processing (a real-time consumer that sizes all device memory at
 * start-up and must never block in or fail inside the device allocator, or a
 * host program whose device memory belongs to another framework's pool).
 * It cleans and normalises one block with the quiet configuration (no
 * automatic excision or zaps: per-window bandpass, dead channels zeroed,
 * (x - loc) / scale in [channel][time] order, low frequency first, padding
 * zero) — the same result as frost_rfi_execute_normalized with every
 * strategy off. `block` and `out` are device pointers; out holds
 * nchans * (block_bytes / row_bytes) floats; nsamps = 0 uses every row and
 * must otherwise be >= 64. Scratch is a fixed 32 MiB + 256 KiB static device
 * array in the library (held by every GPU that loads it until exit), limiting
 * windows x channels to 2684; larger blocks are rejected with
 * FROST_ERR_INVALID_ARGUMENT. The first call on a device looks up the
 * array's address, which also makes the driver load this library's device
 * code onto that device and set the array up (under CUDA's default lazy
 * module loading that is driver-side memory too), so make one call at
 * start-up, before processing begins, and before any stream capture; later
 * calls allocate nothing. All calls share the array: calls that overlap on
 * the GPU race. The block is read after the work queued on `stream`, which
 * must not be NULL; the call synchronises `stream` before returning. */
int frost_rfi_normalize_static(const frost_block_layout* layout,
                               float baseline_length,
                               const uint8_t* block,
                               size_t block_bytes,
                               size_t nsamps,
                               float* out,
                               size_t out_count,
                               void* stream);

/* IQRM channel mask (include/frost/prepare/rfi.hpp:56-59,
 * lib/cpu/rfi_masks_cpu.cpp:29-122) on an n-channel host statistic.
 * `ignore` may be NULL. Writes n flags (1 = flagged) to host `out`. */
int frost_iqrm_mask(const float* x,
                    size_t n,
                    uint64_t radius,
                    float threshold,
                    const uint8_t* ignore,
                    uint8_t* out);

/* apply_manual_killmask (include/frost/prepare/rfi.hpp:48-49,
 * lib/cpu/rfi_masks_cpu.cpp:16-27). */
int frost_apply_manual_killmask(uint8_t* killmask,
                                size_t nchans,
                                const frost_channel_range* zaps,
                                size_t nzaps);

/* read_kill_file (include/frost/prepare/rfi.hpp:40-41,
 * lib/prepare/kill_file.cpp:15-65). Writes merged inclusive ranges. */
int frost_read_kill_file(const char* path,
                         size_t nchans,
                         frost_channel_range* out,
                         size_t capacity,
                         size_t* count);

/* ---- dedispersion plan (include/frost/dedisp/dedisp.hpp) ------------- */

/* DedispPlanConfig (include/frost/dedisp/dedisp.hpp:12-27). */
typedef struct {
    uint64_t nchans;
    float dt;             /* seconds */
    float f0;             /* MHz, channel 0 */
    float df;             /* MHz, may be negative */
    float dm_min;
    float dm_max;
    float dm_pulse_width; /* microseconds */
    float dm_tol;
    int32_t dm_dtype;     /* enum frost_dtype of the DM-time output */
    uint64_t block_nsamps;
    uint64_t subband_depth;
} frost_dedisp_plan_config;

/* generate_dm_list (include/frost/dedisp/dedisp.hpp:29-30,
 * lib/dedisp/dedisp.cpp:16-69). With out == NULL only *count is set. */
int frost_generate_dm_list(const frost_dedisp_plan_config* cfg,
                           float* out,
                           size_t capacity,
                           size_t* count);

/* Ascending band edges of make_dmt_fdmt_plan (lib/dedisp/dedisp.cpp:71-89). */
int frost_fdmt_band_edges(const frost_dedisp_plan_config* cfg,
                          float* f_min,
                          float* f_max);

/* ---- search engine: streaming FDMT + boxcar (replaces dmt::FDMTBoxcar) -- */

/* dmt::PeakFindingMode as frost exposes it (docs/user_guide/search.md:43-49). */
enum frost_peak_mode {
    FROST_PEAK_PER_WIDTH     = 0, /* one peak per above-threshold run, per width */
    FROST_PEAK_ACROSS_WIDTHS = 1, /* one peak per run over all widths together */
    FROST_PEAK_ALL           = 2  /* every sample above threshold */
};

/* Storage of the FDMT intermediate planes (arithmetic is always float). */
enum frost_storage { FROST_STORAGE_FP32 = 0, FROST_STORAGE_FP16 = 1 };

/* dmt::BoxcarConfig as frost fills it (lib/pipeline/pipeline.cpp:316-330),
 * plus this engine's storage precision and time-tile length (0 = the whole
 * gulp, else a multiple of 4096 samples that bounds device memory). */
typedef struct {
    uint64_t max_boxcar;
    float wtsp;
    int32_t use_trapezoid;
    float detect_thresh;
    float noise_sigma;
    int32_t peak_mode;         /* enum frost_peak_mode */
    uint64_t max_candidates;   /* per execute call, over all planes */
    uint64_t max_cands_per_dm; /* per plane and DM trial; 0 = unlimited */
    int32_t skip_cold_prefix;
    int32_t input_nbits;       /* 32: float input */
    float input_mean;
    int32_t storage;           /* enum frost_storage */
    uint64_t tile_nsamps;
} frost_boxcar_config;

/* One detection (the RawCandidate fields frost reads,
 * lib/search/postprocess.cpp:79-116). Samples are absolute stream indices,
 * referenced to the bottom (lowest frequency) of the plane's band;
 * [begin, end] is the above-threshold run; channels are in FDMT (ascending
 * frequency) order, end exclusive. */
typedef struct {
    uint64_t peak_sample;
    uint64_t begin_sample;
    uint64_t end_sample;
    float snr;
    float dm;
    float f_low_mhz;
    float f_high_mhz;
    uint32_t filter_idx;
    uint32_t width;
    uint32_t dm_idx;
    uint32_t chan_begin;
    uint32_t chan_end;
    uint32_t beam_idx;
    uint32_t subband_level;
    uint32_t subband_idx;
} frost_candidate;

/* Plan-level facts (FDMTPlan queries used at lib/pipeline/pipeline.cpp:405,
 * 433-436). */
typedef struct {
    uint64_t nchans;
    uint64_t block_nsamps;
    uint64_t tile_nsamps;
    uint64_t dt_max;
    uint64_t ndm;          /* full-band DM trials */
    uint64_t nplanes;
    uint64_t nwidths;
    uint64_t levels;
    uint64_t device_bytes; /* device memory held by the engine */
    double f_min;
    double f_max;
} frost_search_info;

/* One search plane (get_search_plans()[p], tests/cpp/api/calibration_test.cpp:
 * 53-134). */
typedef struct {
    uint32_t subband_level;
    uint32_t subband_idx;
    uint32_t level;        /* FDMT height of the plane's node */
    uint32_t chan_begin;
    uint32_t chan_end;
    uint32_t staggered;
    uint64_t ndm;
    double f_low;
    double f_high;
} frost_search_plane;

typedef struct frost_search frost_search;

/* FDMTBoxcar(plan, BoxcarConfig, ..., memory budget, kill mask)
 * (lib/pipeline/pipeline.cpp:346-367). `kill_mask` has nchans entries in
 * FDMT order, 1 = keep, 0 = killed; NULL keeps every channel. Fails with
 * FROST_ERR_OUT_OF_MEMORY when the plan cannot fit in `memory_budget` bytes
 * (0 = no limit) at any tile length. */
int frost_search_create(const frost_dedisp_plan_config* plan,
                        const frost_boxcar_config* cfg,
                        const uint8_t* kill_mask,
                        size_t memory_budget,
                        int device,
                        frost_search** out);

int frost_search_destroy(frost_search* s);

/* FDMTBoxcar::execute (host span: lib/pipeline/pipeline.cpp:608; device
 * span + copy_result: :603-605). `waterfall` is [nchans][nsamps] float32,
 * low frequency first, nsamps <= block_nsamps, on the device when
 * `on_device` (read after the work queued on `stream`, which must then not
 * be NULL) else host memory. `mask` (nchans bytes, FDMT order) replaces the
 * constructor mask for this and later calls; NULL keeps the current one.
 * Results are complete when the call returns. */
int frost_search_execute(frost_search* s,
                         const float* waterfall,
                         size_t nsamps,
                         int on_device,
                         const uint8_t* mask,
                         void* stream);

/* FDMTBoxcar::drain (lib/pipeline/pipeline.cpp:517): closes every open
 * above-threshold run; its peaks become the current results. */
int frost_search_drain(frost_search* s);

/* CandidateResultView of the last execute/drain: count and drop counters. */
int frost_search_result_count(const frost_search* s,
                              size_t* count,
                              uint64_t* dropped_global,
                              uint64_t* dropped_per_dm);

/* Copies the last results, sorted by (plane, dm_idx, peak_sample, width). */
int frost_search_results(const frost_search* s,
                         frost_candidate* out,
                         size_t capacity,
                         size_t* count);

/* get_candidate_frontier (lib/pipeline/pipeline.cpp:493): the earliest
 * absolute sample a later call can still report a peak at. */
int frost_search_frontier(const frost_search* s, uint64_t* sample);

int frost_search_get_info(const frost_search* s, frost_search_info* out);

/* Plane p's facts; `dm_grid` and `warmup` (ndm entries each) may be NULL. */
int frost_search_plane_info(const frost_search* s,
                            size_t plane,
                            frost_search_plane* out,
                            float* dm_grid,
                            uint32_t* warmup);

/* Boxcar widths (shared by all planes). */
int frost_search_widths(const frost_search* s,
                        uint32_t* out,
                        size_t capacity,
                        size_t* count);

/* get_subband_variance_grid (tests/cpp/api/calibration_test.cpp:105-106):
 * exact FP64 noise variance of every DM row of `plane` at `width` for
 * `mask` (FDMT order; NULL = current mask). */
int frost_search_variance_grid(const frost_search* s,
                               size_t plane,
                               uint32_t width,
                               const uint8_t* mask,
                               double* out,
                               size_t capacity);

/* Keeps a float copy of every plane's DM-time rows of the next execute
 * calls (for checks against the FP64 oracle; costs memory and time). */
int frost_search_capture_planes(frost_search* s, int enable);

/* Copies plane p's captured rows of the last execute: [ndm][nsamps]. */
int frost_search_plane_data(const frost_search* s,
                            size_t plane,
                            float* out,
                            size_t capacity);

/* Per-phase device time of the execute calls since timing was enabled
 * (CUDA events on the engine's stream), the stage profile frost keeps in
 * RunProfile (include/frost/pipeline/profile.hpp:27-61) at kernel level.
 * `algorithmic_level_bytes` counts one read of every input row and one write
 * of every output row of the FDMT levels >= 2 (the HBM roofline's traffic).
 * `unfused_model_bytes` is the schedule-independent figure of the FDMT and
 * search per gulp of T samples: every level l = 1..L read and written once
 * with its history, sum_l (R_{l-1} + R_l) (T + H_l) s, plus one read of every
 * searched plane row, sum_p R_p T s (R_0 = channels, s = the plane element
 * size); fusing levels moves fewer bytes than it counts. */
typedef struct {
    double level1_ms;
    double level_ms;
    double search_ms;
    double history_ms;
    double variance_ms;
    uint64_t level_launches;
    uint64_t search_launches;
    uint64_t total_launches;
    uint64_t algorithmic_level_bytes;
    uint64_t algorithmic_level1_bytes;
    uint64_t algorithmic_search_bytes;
    uint64_t executes;
    uint64_t unfused_model_bytes;
} frost_search_timing;

/* No counterpart in the reference (dmt launches per call). With `enable`
 * (the default) the engine captures its per-gulp launch sequence (FDMT
 * steps, history copies, searches) as a CUDA graph on the first gulp and
 * replays it while the waterfall's address and length stay the same; the
 * gulp start and mask-change flag are read from device memory. Timing and
 * plane capture launch directly. Results are the same either way. */
int frost_search_use_graphs(frost_search* s, int enable);

/* No counterpart in the reference. The engine's own stream (a
 * cudaStream_t), on which it runs every launch of a gulp. */
int frost_search_get_stream(const frost_search* s, void** stream);

/* No counterpart in the reference; a diagnostic of the error path. The
 * pipelined level and search kernels wait for each bulk copy a bounded
 * number of tries (mbarrier.try_wait); a wait that runs out makes the call
 * fail with FROST_ERR_TIMEOUT instead of hanging. `tries` sets that bound
 * for the first wait on each copy (a negative value restores the default,
 * 2^22; 0 gives up at once, which forces the timeout path); a kernel that
 * gave up still waits for every copy it has in flight, with the default
 * bound, before it exits. */
int frost_search_set_wait_limit(frost_search* s, int64_t tries);

/* No counterpart in the reference. Starts the stream afresh (histories and
 * open runs cleared, sample count zero, the constructor's mask current), as
 * after a gulp that failed with FROST_ERR_TIMEOUT. */
int frost_search_restart(frost_search* s);

/* No counterpart in the reference. Measures this geometry's FDMT launch
 * shapes (fused two-level steps with 2, 3 or 4 bulk-copy stages, or single
 * levels; 4, 8, 16, 32, 64 or 128 tiles of 2048 samples per level-kernel CTA) with
 * one tile pass each on a zero waterfall, applies the fastest and restarts
 * the stream; results are cached per process by geometry. The search chunk
 * keeps its default (4096). Call before the first gulp. Any output pointer
 * may be NULL. */
int frost_search_autotune(frost_search* s, int* fused, int* tiles_per_cta, double* ms, int* cached);

/* No counterpart in the reference. The launch shape in use (autotune's
 * choice or the default): fused two-level steps, tiles of 2048 samples per
 * level-kernel CTA, the fused kernel's bulk-copy stages (0 = its default:
 * 4 with fp16 storage, 3 with float) and the search kernel's chunk (2048 or
 * 4096 samples). */
int frost_search_get_launch_shape(const frost_search* s,
                                  int* fused,
                                  int* tiles_per_cta,
                                  int* stages,
                                  int* search_chunk);

/* No counterpart in the reference. Pins a launch shape (for example one
 * autotune chose in an earlier process) and restarts the stream; call
 * before the first gulp. The level shape never changes results; the search
 * chunk changes where window sums are rounded from (relative 1e-7).
 * FROST_ERR_OUT_OF_MEMORY if the schedule does not fit the engine's memory
 * budget. */
int frost_search_set_launch_shape(frost_search* s, int fused, int tiles_per_cta, int stages, int search_chunk);

/* No counterpart in the reference. Caps the engine's FDMT level and search
 * kernels at `ctas_per_sm` resident CTAs per SM (0, the default: one CTA
 * per work item, each launch filling the GPU). A capped launch loops over
 * its work items and leaves the rest of every SM to kernels on other
 * streams, which is what lets several beams' HBM-bound level passes and
 * instruction-bound searches run side by side. Results do not depend on
 * it. Waits for the engine's stream. */
int frost_search_set_residency(frost_search* s, int ctas_per_sm);
int frost_search_get_residency(const frost_search* s, int* ctas_per_sm);

/* No counterpart in the reference. With `on` = 1 or 2 every single FDMT
 * level step into a searched level is fused with that level's search: the
 * search kernel computes each searched row from the level below (the same
 * sums and fp16 rounding as the level kernel), writes it and searches it in
 * one pass, staging `on` chunks of the row's two children at once, and the
 * level kernel computes only the rows no plane searches; 0 turns it off.
 * Results are identical either way. The default is 1. Two staged chunks
 * hold fewer CTAs an SM and measured slower. FROST_ERR_INVALID_ARGUMENT
 * outside 0..2. Waits for the engine's stream. */
int frost_search_set_fused_search(frost_search* s, int on);
int frost_search_get_fused_search(const frost_search* s, int* on);

/* Enables (and zeroes) or disables per-phase timing. */
int frost_search_enable_timing(frost_search* s, int enable);
int frost_search_get_timing(const frost_search* s, frost_search_timing* out);

/* ---- serving: many beams on one GPU -------------------------------------
 *
 * frost runs one beam per process and reads its next gulp on a side thread
 * while the current one is searched (GulpPrefetch,
 * lib/pipeline/pipeline.cpp:109-262). The server runs many beams on one
 * GPU: each beam keeps its RFI calibration and FDMT tails resident; beams
 * are admitted by device memory; gulps are taken by `slots` worker threads
 * as they arrive, oldest first, one gulp per beam at a time (a beam's gulps
 * stay in order), so one beam's host-side phases overlap other beams'
 * kernels. Latency is measured from submit to candidates ready. */

typedef struct {
    uint64_t completed;
    uint64_t beams;
    uint64_t device_bytes; /* charged to admitted beams */
    double beam_seconds;   /* data searched (valid samples x tsamp) */
    double wall_seconds;   /* first arrival to last completion */
    double p50_latency_s;
    double p99_latency_s;
    double max_latency_s;
    uint64_t launches;     /* kernels launched for the completed gulps */
} frost_server_stats;

typedef struct frost_server frost_server;

/* memory_budget 0 = 90% of the device's free memory. */
int frost_server_create(int device, size_t memory_budget, uint32_t slots, frost_server** out);
int frost_server_destroy(frost_server* s);

/* Admits a beam (RFICleaner + search engine, plan.block_nsamps ==
 * layout.max_nsamps): tunes the engine's FDMT launch shape
 * (frost_search_autotune, cached per geometry), allocates all of its
 * steady-state device buffers and charges their size, or fails with
 * FROST_ERR_OUT_OF_MEMORY when that would exceed the budget. */
int frost_server_add_beam(frost_server* s,
                          const frost_rfi_config* rfi,
                          const frost_block_layout* layout,
                          float baseline_length,
                          const frost_dedisp_plan_config* plan,
                          const frost_boxcar_config* search,
                          uint32_t* beam);

/* Waits for the beam's queued gulps, then releases it. */
int frost_server_remove_beam(frost_server* s, uint32_t beam);

/* Queues one gulp (a block of max_nsamps rows, `nread` valid) that is in
 * host memory, or in the server device's memory when on_device is non-zero;
 * the block must stay valid until frost_server_wait returns for the ticket.
 * The server reads it on its own streams, so a device block must be
 * complete when it is submitted (its writes synchronised). */
int frost_server_submit(frost_server* s,
                        uint32_t beam,
                        const uint8_t* block,
                        size_t block_bytes,
                        size_t nread,
                        int on_device,
                        uint64_t* ticket);

/* Blocks until the gulp is searched; copies up to `capacity` candidates
 * (sorted as frost_search_results), sets *count to the total and returns
 * FROST_ERR_OVERFLOW if some did not fit. */
int frost_server_wait(frost_server* s,
                      uint64_t ticket,
                      frost_candidate* out,
                      size_t capacity,
                      size_t* count,
                      double* latency_s);

/* drain() of one beam's engine (end of its stream). */
int frost_server_drain(frost_server* s,
                       uint32_t beam,
                       frost_candidate* out,
                       size_t capacity,
                       size_t* count);

/* Statistics since the server was created or since the last reset; a
 * reset while gulps are in flight counts them when they complete. */
int frost_server_get_stats(frost_server* s, frost_server_stats* out);
int frost_server_reset_stats(frost_server* s);

/* ---- batched multi-beam search -------------------------------------------
 *
 * No counterpart in the reference: frost runs one engine per pipeline and
 * one beam per process (lib/pipeline/pipeline.cpp:346-367). A batch runs one
 * gulp of each of its beams per call: the beams' RFI stages concurrently,
 * then their searches as rounds in which the level steps of all beams are
 * one launch and their searches one launch (segment tables over the beams'
 * buffers), captured once as a CUDA graph and replayed while the beams'
 * waterfalls stay in place. Beams may differ in channel count, sample type,
 * gulp length, DM range and plane count; each beam's candidates equal those
 * of the same beam run alone. */

typedef struct {
    uint64_t executes;
    uint64_t beams;
    uint64_t rounds;                  /* (tile, level step) rounds run */
    uint64_t merged_level_launches;   /* level launches covering many beams */
    uint64_t merged_search_launches;  /* search launches covering many beams */
    uint64_t beam_launches;           /* per-beam launches of the rounds */
    uint64_t graph_replays;
    uint64_t device_bytes;            /* charged to admitted beams */
} frost_batch_stats;

typedef struct frost_batch frost_batch;

/* memory_budget 0 = 90 % of the device's free memory. */
int frost_batch_create(int device, size_t memory_budget, frost_batch** out);
int frost_batch_destroy(frost_batch* b);

/* Admits a beam (as frost_server_add_beam: launch shape tuned, buffers
 * allocated, FROST_ERR_OUT_OF_MEMORY beyond the budget); beams are numbered
 * 0, 1, ... in the order they are added. */
int frost_batch_add_beam(frost_batch* b,
                         const frost_rfi_config* rfi,
                         const frost_block_layout* layout,
                         float baseline_length,
                         const frost_dedisp_plan_config* plan,
                         const frost_boxcar_config* search,
                         uint32_t* beam);

/* One gulp of every beam: blocks[i] is beam i's block of max_nsamps rows,
 * nread[i] of them valid, in host memory or (on_device) complete in device
 * memory. The candidates are read with frost_batch_results. */
int frost_batch_execute(frost_batch* b, const uint8_t* const* blocks, const size_t* nread, int on_device);

/* Copies up to `capacity` of beam's last candidates (sorted as
 * frost_search_results); *count is their number; FROST_ERR_OVERFLOW if some
 * did not fit. */
int frost_batch_results(const frost_batch* b, uint32_t beam, frost_candidate* out, size_t capacity, size_t* count);

/* drain() of one beam's engine (end of its stream). */
int frost_batch_drain(frost_batch* b, uint32_t beam, frost_candidate* out, size_t capacity, size_t* count);

/* CUDA-graph replay of the batched rounds (default on). */
int frost_batch_use_graph(frost_batch* b, int enable);

int frost_batch_get_stats(const frost_batch* b, frost_batch_stats* out);

/* ---- input staging (GulpPrefetch, lib/pipeline/pipeline.cpp:105-262) -----
 *
 * frost's GulpPrefetch reads the next block on a thread while the caller
 * searches the current one. Here a reader thread fills pinned host slots
 * from a block source and copies each to a device slot on its own stream,
 * so reading and the host-to-device copy of gulp k+1 overlap the kernels of
 * gulp k; gulps come out in order, already on the device. */

/* A block source: writes up to `max_rows` packed rows into `buf` and
 * returns how many (fewer than max_rows at the end, 0 once exhausted) or a
 * negative value on error. Called on the prefetch thread. */
typedef long (*frost_read_fn)(void* ctx, uint8_t* buf, size_t max_rows);

typedef struct {
    uint64_t gulps;
    uint64_t bytes;
    double read_s; /* reader thread: source reads and copy issue */
    double wait_s; /* caller blocked in frost_prefetch_next */
} frost_prefetch_stats;

typedef struct frost_prefetch frost_prefetch;

/* `depth` slots (2-8) of block_rows x row_bytes, pinned on the host and
 * resident on `device`; the reader starts at once. */
int frost_prefetch_create(size_t block_rows,
                          size_t row_bytes,
                          int depth,
                          int device,
                          frost_read_fn read,
                          void* ctx,
                          frost_prefetch** out);

/* The same over a file of packed rows after `header_bytes` of header (a
 * SIGPROC filterbank's data section, for instance). */
int frost_prefetch_create_file(const char* path,
                               uint64_t header_bytes,
                               size_t block_rows,
                               size_t row_bytes,
                               int depth,
                               int device,
                               frost_prefetch** out);

/* The SIGPROC filterbank header (the sigproc file input of frost's
 * open_input, lib/pipeline/input.cpp:32-69, read there through psrio):
 * the fields the search needs, where the data start and how many whole
 * rows follow. */
typedef struct {
    uint64_t header_bytes;   /* data start */
    uint64_t nchans;
    uint64_t row_bytes;      /* nchans * nbits / 8 */
    uint64_t data_rows;      /* whole rows after the header */
    uint64_t nsamples;       /* the header's nsamples keyword, 0 if absent */
    int32_t nbits;
    int32_t nifs;
    int32_t data_type;
    int32_t telescope_id;
    int32_t machine_id;
    int32_t ibeam;
    int32_t nbeams;
    int32_t signed_samples;  /* the `signed` keyword */
    double fch1;             /* MHz, channel 0 */
    double foff;             /* MHz */
    double tsamp;            /* seconds */
    double tstart;           /* MJD */
    double src_raj;
    double src_dej;
    double refdm;
    char source_name[80];
} frost_sigproc_header;

/* Reads the header of the SIGPROC filterbank at `path`. FROST_ERR_IO if it
 * cannot be opened; FROST_ERR_INVALID_ARGUMENT if the header is malformed,
 * names an unknown keyword, lacks nchans, nbits, tsamp, fch1 or foff, or
 * has more than one IF. */
int frost_sigproc_read_header(const char* path, frost_sigproc_header* out);

/* The BlockLayout of a SIGPROC file's rows for gulps of `block_rows`
 * samples: nbits 1/2/4/8/16 unsigned or 32 float, channel 0 at fch1,
 * spacing foff. */
int frost_sigproc_layout(const frost_sigproc_header* header, uint64_t block_rows, frost_block_layout* out);

/* frost_prefetch_create_file over a SIGPROC filterbank: its header is
 * parsed (written to `header` when not NULL) and the rows after it are
 * staged in gulps of `block_rows`. */
int frost_prefetch_create_sigproc(const char* path,
                                  size_t block_rows,
                                  int depth,
                                  int device,
                                  frost_sigproc_header* header,
                                  frost_prefetch** out);

/* The same over `total_rows` packed rows in caller host memory (kept valid
 * until destroy): the reader thread copies them into the pinned slots, as a
 * socket or ring-buffer reader would. */
int frost_prefetch_create_memory(const uint8_t* rows,
                                 size_t total_rows,
                                 size_t block_rows,
                                 size_t row_bytes,
                                 int depth,
                                 int device,
                                 frost_prefetch** out);

/* GulpPrefetch::next (pipeline.cpp:131-152): the next gulp on the device
 * (*block_device valid until the next call) and its row count (0 = end of
 * source). With a `stream`, that stream waits for the gulp's copy and the
 * slot is refilled only after the work the caller enqueues on it before its
 * next call; with NULL the call waits for the copy on the host and the
 * caller must have finished with the previous gulp (as a pipeline that reads
 * its candidates back has). A source error is returned here
 * (FROST_ERR_IO). */
int frost_prefetch_next(frost_prefetch* p, void* stream, const uint8_t** block_device, size_t* nread);

int frost_prefetch_get_stats(const frost_prefetch* p, frost_prefetch_stats* out);
int frost_prefetch_destroy(frost_prefetch* p);

/* ---- candidate post-processing (include/frost/search/postprocess.hpp) ---
 *
 * Friends-of-friends clustering within each FDMT plane, DM-wing seeding,
 * sub-band deduplication across planes, the per-plane rate limiter and the
 * streaming carry of unfinished clusters, run on the device
 * (lib/search/postprocess.cpp:67-241, clustering.cpp:24-226,
 * merge.cpp:8-37, subband_dedup.cpp:163-315, rate_limiter.cpp:5-30). */

/* search::Giant (include/frost/search/candidate.hpp:28-66). Its optional
 * location_best is flattened into loc_* with has_location_best. Sample,
 * index and channel fields are SizeType (64-bit). */
typedef struct {
    uint64_t samp_idx;         /* peak sample */
    uint64_t filter_idx;
    uint64_t filter_width;     /* 0 derives 1 << filter_idx */
    uint64_t dm_idx;
    uint64_t begin;
    uint64_t end;
    uint64_t members;
    uint64_t chan_begin;       /* inclusive, original channel order */
    uint64_t chan_end;         /* inclusive */
    uint64_t plane;            /* subband_level * nchans + subband_idx */
    uint64_t best_chan_begin;
    uint64_t best_chan_end;
    uint64_t n_extents;
    uint64_t loc_samp_idx;     /* location_best.samp_idx */
    uint64_t loc_filter_width; /* location_best.filter_width */
    float snr;
    float dm;
    float f_low;               /* MHz */
    float f_high;              /* MHz */
    float snr_best;
    float loc_dm;
    float loc_f_low;
    float loc_f_high;
    int32_t has_location_best;
    int32_t reserved;
} frost_giant;

/* ClusterTolerances (include/frost/search/clustering.hpp:22-33). */
typedef struct {
    uint64_t time_tol;
    uint64_t filter_tol;
    uint64_t dm_tol;
    double dm_smear;  /* 0 = trial count only */
    double tsamp;     /* seconds */
    double snr_floor; /* 0 disables the S/N growth of the DM gate */
} frost_cluster_tolerances;

/* ClusterMode (clustering.hpp:44) and SubbandDedupMode
 * (subband_dedup.hpp:42). */
enum frost_cluster_mode { FROST_CLUSTER_CHAIN = 0, FROST_CLUSTER_SEEDED = 1 };
enum frost_dedup_mode { FROST_DEDUP_TRANSITIVE = 0, FROST_DEDUP_SEEDED = 1 };

/* The SearchConfig fields the post-processor reads
 * (include/frost/config/config.hpp:57-97). */
typedef struct {
    uint64_t boxcar_max;
    uint64_t max_candidates;
    uint64_t max_pending_candidates; /* 0 = max_candidates */
    uint64_t cand_sep_time;
    uint64_t cand_sep_filter;
    uint64_t cand_sep_dm;
    float detect_thresh;
    float cand_sep_dm_smear;
    float max_giant_rate;            /* <= 0 disables the rate limiter */
    int32_t cluster;
    int32_t subband_dedup;           /* enum frost_dedup_mode */
    int32_t reserved;
} frost_postprocess_config;

/* CandidatePostprocessLayout (postprocess.hpp:12-16). */
typedef struct {
    uint64_t nchans;
    double tsamp;
    double frequency_step; /* MHz; negative = channels stored high first */
} frost_postprocess_layout;

/* CandidatePostprocessResult (postprocess.hpp:20-25); the giants are read
 * with frost_postprocess_results. */
typedef struct {
    size_t count;
    uint64_t pending_candidates;
    double cluster_s;
    double dedup_s;
    uint64_t launches; /* kernels this call launched */
} frost_postprocess_result;

typedef struct frost_postprocess frost_postprocess;

/* CandidatePostprocessPlan(cfg, layout) (postprocess.cpp:50-66): reserves
 * device memory for max_candidates incoming and max_pending_candidates
 * carried rows. */
int frost_postprocess_create(const frost_postprocess_config* cfg,
                             const frost_postprocess_layout* layout,
                             int device,
                             frost_postprocess** out);
int frost_postprocess_destroy(frost_postprocess* p);

/* Attaches a CandidatePostprocessPlan to a served beam: after the search of
 * each of its gulps the detections are clustered and deduplicated on the
 * device, as frost's Pipeline::publish does (lib/pipeline/pipeline.cpp:
 * 478-493, samples_read = the beam's samples so far, duration = the gulp's
 * rows, frontier = the engine's). Waits for the beam to be idle; the plan's
 * device memory is charged to the server budget (FROST_ERR_OUT_OF_MEMORY if
 * it does not fit). */
int frost_server_set_postprocess(frost_server* s, uint32_t beam, const frost_postprocess_config* cfg);

/* No counterpart in the reference. frost_search_set_residency for one
 * served beam (between its gulps). */
int frost_server_set_residency(frost_server* s, uint32_t beam, int ctas_per_sm);

/* GulpPrefetch's overlap of a gulp's upload with the work on the gulp
 * before it (lib/pipeline/pipeline.cpp:105-262), for served beams: gives the
 * idle beam `slots` (0-4) device blocks. A host gulp in pinned memory that
 * is submitted while a slot is free is copied into it at once, on a copy
 * stream of the beam's own; the beam's gulps still run in submission order.
 * Other host gulps are copied when they are processed. The blocks are charged
 * to the server budget (FROST_ERR_OUT_OF_MEMORY if they do not fit); 0
 * releases them. */
int frost_server_set_staging(frost_server* s, uint32_t beam, uint32_t slots);

/* frost_server_wait for a beam with a post-processor: the gulp's giants
 * (its raw candidates are dropped). */
int frost_server_wait_giants(frost_server* s,
                             uint64_t ticket,
                             frost_giant* out,
                             size_t capacity,
                             size_t* count,
                             double* latency_s);

/* drain() of a beam with a post-processor: the final call's giants (every
 * carried cluster released). */
int frost_server_drain_giants(frost_server* s, uint32_t beam, frost_giant* out, size_t capacity, size_t* count);

/* CandidatePostprocessPlan::execute (postprocess.cpp:67-180) over `n` raw
 * detections, on the device when `on_device` else in host memory. Fails
 * with FROST_ERR_INVALID_ARGUMENT on an invalid row (nothing changes) and
 * FROST_ERR_OVERFLOW when the carried rows would exceed
 * max_pending_candidates (the carry keeps its previous rows). */
int frost_postprocess_execute(frost_postprocess* p,
                              const frost_candidate* cands,
                              size_t n,
                              int on_device,
                              uint64_t samples_read,
                              uint64_t duration_samples,
                              int final_call,
                              uint64_t candidate_frontier,
                              frost_postprocess_result* out);

/* The same over the search handle's last results, read in place on the
 * device (pipeline.cpp:481-487 hands dmt's view over the same way). Both
 * handles must be on the same device; `s` is synchronised first. */
int frost_postprocess_execute_search(frost_postprocess* p,
                                     frost_search* s,
                                     uint64_t samples_read,
                                     uint64_t duration_samples,
                                     int final_call,
                                     uint64_t candidate_frontier,
                                     frost_postprocess_result* out);

/* Copies the last execute's giants (valid until the next execute). */
int frost_postprocess_results(const frost_postprocess* p,
                              frost_giant* out,
                              size_t capacity,
                              size_t* count);

/* memory_usage() and estimate_memory(cfg) (postprocess.cpp:181-286), in
 * device bytes of this implementation. */
int frost_postprocess_memory_usage(const frost_postprocess* p, uint64_t* bytes);
int frost_postprocess_estimate_memory(const frost_postprocess_config* cfg, uint64_t* bytes);

/* ClusterLabelPlan::execute (clustering.cpp:107-226) on the device: one
 * label per giant (its cluster's representative index). */
int frost_cluster_labels(const frost_giant* giants,
                         size_t n,
                         const frost_cluster_tolerances* tol,
                         int mode,
                         uint64_t* labels,
                         int device);

/* MergeCandidatesPlan::execute (merge.cpp:8-37) on the device; `out` holds
 * up to n rows, *count is the number of clusters. */
int frost_merge_candidates(const frost_giant* giants,
                           const uint64_t* labels,
                           size_t n,
                           frost_giant* out,
                           size_t* count,
                           int device);

/* SubbandDedupPlan::execute (subband_dedup.cpp:194-315) on the device;
 * `out` holds up to n rows. */
int frost_subband_dedup(const frost_giant* giants,
                        size_t n,
                        const frost_cluster_tolerances* tol,
                        float tsamp,
                        int mode,
                        frost_giant* out,
                        size_t* count,
                        int device);

/* are_coincident (clustering.cpp:24-67): `physical` selects the overload
 * with the DM-smearing gate. Host arithmetic identical to the kernels'. */
int frost_are_coincident(const frost_giant* a,
                         const frost_giant* b,
                         const frost_cluster_tolerances* tol,
                         int physical);

/* subband_time_shift_samples / subband_dm_step (subband_dedup.cpp:163-192). */
double frost_subband_time_shift_samples(float dm, float f_wide, float f_narrow, float tsamp);
double frost_subband_dm_step(float f_low, float f_high, float tsamp);

/* ---- candidate file (include/frost/output/cand_writer.hpp) --------------
 *
 * frost's `.cand` layout: 23 tab-separated columns per giant (snr,
 * samp_idx, time, filter_idx, dm_idx, dm, members, begin, end, f_low,
 * f_high, chan_begin, chan_end, snr_best, chan_begin_best, chan_end_best,
 * n_extents, samp_idx_best, time_best, dm_best, width_best, f_low_best,
 * f_high_best), printed as frost prints them. Host code: the giants come
 * from frost_postprocess_results or frost_server_wait_giants. */

typedef struct frost_cand_writer frost_cand_writer;

/* CandWriter(path, dt, mode) (cand_writer.hpp:38-45,
 * lib/output/cand_writer.cpp:26-38): creates missing parent directories;
 * `append` 0 truncates. FROST_ERR_IO if the file cannot be opened. */
int frost_cand_writer_open(const char* path, double dt, int append, frost_cand_writer** out);

/* CandWriter::write (cand_writer.cpp:40-71): one row per giant, sample
 * columns offset by `first_samp_idx`; flushes; FROST_ERR_IO on a failed
 * write. */
int frost_cand_writer_write(frost_cand_writer* w, const frost_giant* giants, size_t n, uint64_t first_samp_idx);

int frost_cand_writer_close(frost_cand_writer* w);

/* cand_filename (cand_writer.cpp:73-87): "YYYY-MM-DD-HH:MM:SS_BB.cand" of
 * `utc` (seconds since the epoch) and 1-based `beam`, into out[capacity]. */
int frost_cand_filename(int64_t utc, uint64_t beam, char* out, size_t capacity);

/* ---- memory planning (include/frost/pipeline/memory.hpp) ------------------
 *
 * The device counterpart of frost's planner (lib/pipeline/memory.cpp:294-508):
 * the device bytes of one beam's RFI cleaner, FDMT/search engine and
 * (optionally) post-processor, computed on the host from the plans without
 * allocating anything, and the gulp check frost runs before building them. */

typedef struct {
    uint64_t rfi_bytes;         /* RFI cleaner: raw block, float work and output, window / chunk tables */
    uint64_t fdmt_bytes;        /* FDMT level buffers and histories */
    uint64_t search_bytes;      /* plan and search tables, run state, candidate buffer */
    uint64_t postprocess_bytes; /* device post-processing (0 without a config) */
    uint64_t transient_bytes;   /* autotune's zero waterfall, freed before the first gulp */
    uint64_t total_bytes;       /* the sum of the above */
    uint64_t max_delay;         /* the plan's dispersion delay in samples */
} frost_memory_estimate;

/* The footprint of a beam of `layout` (max_nsamps is the gulp), `plan`
 * (block_nsamps must equal it), `search` and, if not NULL, `post`, as this
 * implementation allocates it (level buffers under either schedule the
 * autotuner may try; buffers sized by data at their largest). The same
 * errors as building them for an invalid configuration. */
int frost_estimate_memory(const frost_rfi_config* rfi, const frost_block_layout* layout, float baseline_length,
                          const frost_dedisp_plan_config* plan, const frost_boxcar_config* search,
                          const frost_postprocess_config* post, frost_memory_estimate* out);

/* MemoryCheck (include/frost/pipeline/memory.hpp). */
typedef struct {
    frost_memory_estimate estimate; /* at gulp_used */
    uint64_t requested_bytes;       /* total_bytes at gulp_requested */
    uint64_t available_bytes;       /* 0: unknown, nothing was enforced */
    uint64_t gulp_requested;
    uint64_t gulp_used;
    int32_t lowered;
    int32_t device_memory;          /* always 1: the budget is device memory */
} frost_memory_check;

/* check_memory (lib/pipeline/memory.cpp:294-508) for the device: compares
 * the estimate at the configured gulp with 90 % of `available_bytes` (0:
 * the free memory of `device`, further capped by `memory_limit_bytes` when
 * that is not 0; if neither is known, nothing is enforced). When it does not
 * fit and `gulp_is_default` is set, the gulp (layout->max_nsamps and
 * plan->block_nsamps) is lowered to the largest multiple of 1024 samples
 * that fits and `lowered` is set; otherwise, or when even the smallest
 * valid gulp (max_delay + boxcar_max + 1, rounded up to 1024) does not fit,
 * FROST_ERR_OUT_OF_MEMORY with a message naming the estimate, the budget
 * and the largest gulp that fits. */
int frost_check_memory(const frost_rfi_config* rfi, frost_block_layout* layout, float baseline_length,
                       frost_dedisp_plan_config* plan, const frost_boxcar_config* search,
                       const frost_postprocess_config* post, int gulp_is_default, uint64_t available_bytes,
                       uint64_t memory_limit_bytes, int device, frost_memory_check* out);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* FROST_B200_H */
