"""ctypes mirrors of the plain-C types declared in include/frost_b200.h.

Field order and widths follow the header exactly; the header is the
contract, this module only restates it for Python callers.
"""

import ctypes as C

# status codes (enum frost_status)
OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_OUT_OF_MEMORY = -2
ERR_DEVICE = -3
ERR_TIMEOUT = -4
ERR_STATE = -5
ERR_OVERFLOW = -6
ERR_IO = -7
ERR_INTERNAL = -8

# enum frost_dtype (include/frost/common/policies.hpp:52-60)
UINT1, UINT2, UINT4, UINT8, UINT16, UINT32, FLOAT32 = range(7)
DTYPE_BITS = {UINT1: 1, UINT2: 2, UINT4: 4, UINT8: 8, UINT16: 16, UINT32: 32, FLOAT32: 32}

FILL_NEIGHBOUR, FILL_MEAN, FILL_NOISE = range(3)
ZERO_DM_OFF, ZERO_DM_SUBTRACT, ZERO_DM_ZDOT = range(3)

# enum frost_peak_mode (dmt::PeakFindingMode as frost names it,
# docs/user_guide/search.md:43-49)
PEAK_PER_WIDTH, PEAK_ACROSS_WIDTHS, PEAK_ALL = range(3)

# enum frost_storage: FDMT intermediate plane storage
STORAGE_FP32, STORAGE_FP16 = range(2)


class ChannelRange(C.Structure):
    _fields_ = [("start", C.c_uint64), ("end", C.c_uint64)]


class FrequencyRange(C.Structure):
    _fields_ = [("lo", C.c_double), ("hi", C.c_double)]


class RfiConfigC(C.Structure):
    _fields_ = [
        ("zap_chans", C.POINTER(ChannelRange)),
        ("n_zap_chans", C.c_uint64),
        ("zap_freqs", C.POINTER(FrequencyRange)),
        ("n_zap_freqs", C.c_uint64),
        ("narrow_enabled", C.c_int32),
        ("narrow_threshold", C.c_float),
        ("broad_enabled", C.c_int32),
        ("broad_threshold", C.c_float),
        ("broad_boxcar_max", C.c_uint64),
        ("dropout_enabled", C.c_int32),
        ("dropout_min_std_fraction", C.c_float),
        ("moments_enabled", C.c_int32),
        ("moments_threshold", C.c_float),
        ("moments_mean", C.c_int32),
        ("moments_std", C.c_int32),
        ("moments_skewness", C.c_int32),
        ("moments_kurtosis", C.c_int32),
        ("moments_autocorr", C.c_int32),
        ("moments_kurtosis_max", C.c_float),
        ("iqrm_enabled", C.c_int32),
        ("iqrm_threshold", C.c_float),
        ("iqrm_radius", C.c_uint64),
        ("mask_grow", C.c_uint64),
        ("kadane_channel_enabled", C.c_int32),
        ("kadane_channel_threshold", C.c_float),
        ("kadane_channel_min_duration", C.c_float),
        ("kadane_spectrum_enabled", C.c_int32),
        ("kadane_spectrum_threshold", C.c_float),
        ("kadane_spectrum_min_bandwidth", C.c_float),
        ("kadane_spectrum_whole_band_fraction", C.c_float),
        ("zero_dm", C.c_int32),
        ("equalize", C.c_int32),
        ("fill", C.c_int32),
        ("seed", C.c_uint64),
    ]


class SigprocHeaderC(C.Structure):
    _fields_ = [
        ("header_bytes", C.c_uint64),
        ("nchans", C.c_uint64),
        ("row_bytes", C.c_uint64),
        ("data_rows", C.c_uint64),
        ("nsamples", C.c_uint64),
        ("nbits", C.c_int32),
        ("nifs", C.c_int32),
        ("data_type", C.c_int32),
        ("telescope_id", C.c_int32),
        ("machine_id", C.c_int32),
        ("ibeam", C.c_int32),
        ("nbeams", C.c_int32),
        ("signed_samples", C.c_int32),
        ("fch1", C.c_double),
        ("foff", C.c_double),
        ("tsamp", C.c_double),
        ("tstart", C.c_double),
        ("src_raj", C.c_double),
        ("src_dej", C.c_double),
        ("refdm", C.c_double),
        ("source_name", C.c_char * 80),
    ]

    def as_dict(self) -> dict:
        out = {k: getattr(self, k) for k, _ in self._fields_}
        out["source_name"] = self.source_name.decode(errors="replace")
        return out


class BlockLayoutC(C.Structure):
    _fields_ = [
        ("nchans", C.c_uint64),
        ("max_nsamps", C.c_uint64),
        ("dtype", C.c_int32),
        ("tsamp", C.c_double),
        ("f0", C.c_double),
        ("df", C.c_double),
    ]


class RfiReportC(C.Structure):
    _fields_ = [
        ("calibration_reused", C.c_int32),
        ("nsamps", C.c_uint64),
        ("chans_zapped", C.c_uint64),
        ("chans_dead", C.c_uint64),
        ("chans_moments", C.c_uint64),
        ("chans_iqrm", C.c_uint64),
        ("chans_grown", C.c_uint64),
        ("chans_masked", C.c_uint64),
        ("samps_broad", C.c_uint64),
        ("samps_dropout", C.c_uint64),
        ("samps_kadane", C.c_uint64),
        ("samps_flagged", C.c_uint64),
        ("cells_narrow", C.c_uint64),
        ("cells_kadane_spectrum", C.c_uint64),
        ("cells_kadane_channel", C.c_uint64),
        ("fill_fallbacks", C.c_uint64),
        ("t_bandpass", C.c_double),
        ("t_moments", C.c_double),
        ("t_scan", C.c_double),
        ("t_flags", C.c_double),
        ("t_apply", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class BoxcarConfigC(C.Structure):
    _fields_ = [
        ("max_boxcar", C.c_uint64),
        ("wtsp", C.c_float),
        ("use_trapezoid", C.c_int32),
        ("detect_thresh", C.c_float),
        ("noise_sigma", C.c_float),
        ("peak_mode", C.c_int32),
        ("max_candidates", C.c_uint64),
        ("max_cands_per_dm", C.c_uint64),
        ("skip_cold_prefix", C.c_int32),
        ("input_nbits", C.c_int32),
        ("input_mean", C.c_float),
        ("storage", C.c_int32),
        ("tile_nsamps", C.c_uint64),
    ]


class CandidateC(C.Structure):
    _fields_ = [
        ("peak_sample", C.c_uint64),
        ("begin_sample", C.c_uint64),
        ("end_sample", C.c_uint64),
        ("snr", C.c_float),
        ("dm", C.c_float),
        ("f_low_mhz", C.c_float),
        ("f_high_mhz", C.c_float),
        ("filter_idx", C.c_uint32),
        ("width", C.c_uint32),
        ("dm_idx", C.c_uint32),
        ("chan_begin", C.c_uint32),
        ("chan_end", C.c_uint32),
        ("beam_idx", C.c_uint32),
        ("subband_level", C.c_uint32),
        ("subband_idx", C.c_uint32),
    ]


class SearchInfoC(C.Structure):
    _fields_ = [
        ("nchans", C.c_uint64),
        ("block_nsamps", C.c_uint64),
        ("tile_nsamps", C.c_uint64),
        ("dt_max", C.c_uint64),
        ("ndm", C.c_uint64),
        ("nplanes", C.c_uint64),
        ("nwidths", C.c_uint64),
        ("levels", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("f_min", C.c_double),
        ("f_max", C.c_double),
    ]


class SearchPlaneC(C.Structure):
    _fields_ = [
        ("subband_level", C.c_uint32),
        ("subband_idx", C.c_uint32),
        ("level", C.c_uint32),
        ("chan_begin", C.c_uint32),
        ("chan_end", C.c_uint32),
        ("staggered", C.c_uint32),
        ("ndm", C.c_uint64),
        ("f_low", C.c_double),
        ("f_high", C.c_double),
    ]


class SearchTimingC(C.Structure):
    _fields_ = [
        ("level1_ms", C.c_double),
        ("level_ms", C.c_double),
        ("search_ms", C.c_double),
        ("history_ms", C.c_double),
        ("variance_ms", C.c_double),
        ("level_launches", C.c_uint64),
        ("search_launches", C.c_uint64),
        ("total_launches", C.c_uint64),
        ("algorithmic_level_bytes", C.c_uint64),
        ("algorithmic_level1_bytes", C.c_uint64),
        ("algorithmic_search_bytes", C.c_uint64),
        ("executes", C.c_uint64),
        ("unfused_model_bytes", C.c_uint64),
    ]


class DedispPlanConfigC(C.Structure):
    _fields_ = [
        ("nchans", C.c_uint64),
        ("dt", C.c_float),
        ("f0", C.c_float),
        ("df", C.c_float),
        ("dm_min", C.c_float),
        ("dm_max", C.c_float),
        ("dm_pulse_width", C.c_float),
        ("dm_tol", C.c_float),
        ("dm_dtype", C.c_int32),
        ("block_nsamps", C.c_uint64),
        ("subband_depth", C.c_uint64),
    ]


class ServerStatsC(C.Structure):
    _fields_ = [
        ("completed", C.c_uint64),
        ("beams", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("beam_seconds", C.c_double),
        ("wall_seconds", C.c_double),
        ("p50_latency_s", C.c_double),
        ("p99_latency_s", C.c_double),
        ("max_latency_s", C.c_double),
        ("launches", C.c_uint64),
    ]


class BatchStatsC(C.Structure):
    _fields_ = [
        ("executes", C.c_uint64),
        ("beams", C.c_uint64),
        ("rounds", C.c_uint64),
        ("merged_level_launches", C.c_uint64),
        ("merged_search_launches", C.c_uint64),
        ("beam_launches", C.c_uint64),
        ("graph_replays", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class GiantC(C.Structure):
    """frost_giant: search::Giant (include/frost/search/candidate.hpp:28-66)."""

    _fields_ = [
        ("samp_idx", C.c_uint64),
        ("filter_idx", C.c_uint64),
        ("filter_width", C.c_uint64),
        ("dm_idx", C.c_uint64),
        ("begin", C.c_uint64),
        ("end", C.c_uint64),
        ("members", C.c_uint64),
        ("chan_begin", C.c_uint64),
        ("chan_end", C.c_uint64),
        ("plane", C.c_uint64),
        ("best_chan_begin", C.c_uint64),
        ("best_chan_end", C.c_uint64),
        ("n_extents", C.c_uint64),
        ("loc_samp_idx", C.c_uint64),
        ("loc_filter_width", C.c_uint64),
        ("snr", C.c_float),
        ("dm", C.c_float),
        ("f_low", C.c_float),
        ("f_high", C.c_float),
        ("snr_best", C.c_float),
        ("loc_dm", C.c_float),
        ("loc_f_low", C.c_float),
        ("loc_f_high", C.c_float),
        ("has_location_best", C.c_int32),
        ("reserved", C.c_int32),
    ]


class ClusterTolerancesC(C.Structure):
    _fields_ = [
        ("time_tol", C.c_uint64),
        ("filter_tol", C.c_uint64),
        ("dm_tol", C.c_uint64),
        ("dm_smear", C.c_double),
        ("tsamp", C.c_double),
        ("snr_floor", C.c_double),
    ]


class PostprocessConfigC(C.Structure):
    _fields_ = [
        ("boxcar_max", C.c_uint64),
        ("max_candidates", C.c_uint64),
        ("max_pending_candidates", C.c_uint64),
        ("cand_sep_time", C.c_uint64),
        ("cand_sep_filter", C.c_uint64),
        ("cand_sep_dm", C.c_uint64),
        ("detect_thresh", C.c_float),
        ("cand_sep_dm_smear", C.c_float),
        ("max_giant_rate", C.c_float),
        ("cluster", C.c_int32),
        ("subband_dedup", C.c_int32),
        ("reserved", C.c_int32),
    ]


class PostprocessLayoutC(C.Structure):
    _fields_ = [("nchans", C.c_uint64), ("tsamp", C.c_double), ("frequency_step", C.c_double)]


class PostprocessResultC(C.Structure):
    _fields_ = [
        ("count", C.c_size_t),
        ("pending_candidates", C.c_uint64),
        ("cluster_s", C.c_double),
        ("dedup_s", C.c_double),
        ("launches", C.c_uint64),
    ]


class PrefetchStatsC(C.Structure):
    _fields_ = [("gulps", C.c_uint64), ("bytes", C.c_uint64), ("read_s", C.c_double), ("wait_s", C.c_double)]


READ_FN = C.CFUNCTYPE(C.c_long, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)


class MemoryEstimateC(C.Structure):
    _fields_ = [("rfi_bytes", C.c_uint64), ("fdmt_bytes", C.c_uint64), ("search_bytes", C.c_uint64),
                ("postprocess_bytes", C.c_uint64), ("transient_bytes", C.c_uint64), ("total_bytes", C.c_uint64),
                ("max_delay", C.c_uint64)]


class MemoryCheckC(C.Structure):
    _fields_ = [("estimate", MemoryEstimateC), ("requested_bytes", C.c_uint64), ("available_bytes", C.c_uint64),
                ("gulp_requested", C.c_uint64), ("gulp_used", C.c_uint64), ("lowered", C.c_int32),
                ("device_memory", C.c_int32)]
