"""Candidate post-processing on the GPU with frost's plan shapes:
CandidatePostprocessPlan (include/frost/search/postprocess.hpp:28-62),
ClusterLabelPlan / ClusterTolerances / are_coincident (clustering.hpp,
candidate.hpp:84-111), MergeCandidatesPlan (merge.hpp), SubbandDedupPlan with
subband_time_shift_samples / subband_dm_step (subband_dedup.hpp) and
RateLimiter (rate_limiter.hpp). Every plan runs through the C ABI of
frost_b200/lib/libfrost_b200.so; the per-plane limiter arithmetic is the only
host-side step, as in the reference.

Giants are numpy structured arrays of GIANT_DTYPE (frost_giant); raw
detections are CANDIDATE_DTYPE rows (frost_candidate) or an FDMTBoxcar whose
last results are read in place on the device.
"""

from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Optional, Union

import numpy as np

from . import _abi
from ._lib import check, lib
from .search import CANDIDATE_DTYPE, CandidateResult, FDMTBoxcar

GIANT_DTYPE = np.dtype([
    ("samp_idx", np.uint64), ("filter_idx", np.uint64), ("filter_width", np.uint64),
    ("dm_idx", np.uint64), ("begin", np.uint64), ("end", np.uint64), ("members", np.uint64),
    ("chan_begin", np.uint64), ("chan_end", np.uint64), ("plane", np.uint64),
    ("best_chan_begin", np.uint64), ("best_chan_end", np.uint64), ("n_extents", np.uint64),
    ("loc_samp_idx", np.uint64), ("loc_filter_width", np.uint64),
    ("snr", np.float32), ("dm", np.float32), ("f_low", np.float32), ("f_high", np.float32),
    ("snr_best", np.float32), ("loc_dm", np.float32), ("loc_f_low", np.float32),
    ("loc_f_high", np.float32), ("has_location_best", np.int32), ("reserved", np.int32)])
assert GIANT_DTYPE.itemsize == C.sizeof(_abi.GiantC)


def make_giants(n: int) -> np.ndarray:
    """n default Giants (members = n_extents = 1, everything else zero)."""
    g = np.zeros(n, GIANT_DTYPE)
    g["members"] = 1
    g["n_extents"] = 1
    return g


def giant_boxcar_width(g) -> int:
    """filter_width, or 1 << filter_idx (saturating at the top bit)."""
    fw = int(g["filter_width"])
    if fw > 0:
        return fw
    return 1 << min(int(g["filter_idx"]), 63)


class ClusterMode(enum.IntEnum):
    CHAIN = 0
    SEEDED = 1


class SubbandDedupMode(enum.IntEnum):
    TRANSITIVE = 0
    SEEDED = 1


@dataclass
class ClusterTolerances:
    """ClusterTolerances (include/frost/search/clustering.hpp:22-33)."""
    time_tol: int
    filter_tol: int
    dm_tol: int
    dm_smear: float = 0.0
    tsamp: float = 0.0
    snr_floor: float = 0.0

    def _c(self) -> _abi.ClusterTolerancesC:
        return _abi.ClusterTolerancesC(int(self.time_tol), int(self.filter_tol), int(self.dm_tol),
                                       float(self.dm_smear), float(self.tsamp), float(self.snr_floor))


@dataclass
class SearchConfig:
    """The config::SearchConfig fields the post-processor reads, with frost's
    defaults (include/frost/config/config.hpp:57-97)."""
    boxcar_max: int = 4096
    max_candidates: int = 131072
    max_pending_candidates: int = 0
    detect_thresh: float = 6.0
    cand_sep_time: int = 3
    cand_sep_filter: int = 3
    cand_sep_dm: int = 200
    cand_sep_dm_smear: float = 8.0
    max_giant_rate: float = 0.0
    cluster: bool = True
    subband_dedup: SubbandDedupMode = SubbandDedupMode.TRANSITIVE

    def _c(self) -> _abi.PostprocessConfigC:
        return _abi.PostprocessConfigC(
            int(self.boxcar_max), int(self.max_candidates), int(self.max_pending_candidates),
            int(self.cand_sep_time), int(self.cand_sep_filter), int(self.cand_sep_dm),
            float(self.detect_thresh), float(self.cand_sep_dm_smear), float(self.max_giant_rate),
            1 if self.cluster else 0, int(self.subband_dedup), 0)


@dataclass
class CandidatePostprocessLayout:
    """CandidatePostprocessLayout (postprocess.hpp:12-16)."""
    nchans: int
    tsamp: float
    frequency_step: float

    def _c(self) -> _abi.PostprocessLayoutC:
        return _abi.PostprocessLayoutC(int(self.nchans), float(self.tsamp), float(self.frequency_step))


@dataclass
class CandidatePostprocessResult:
    """CandidatePostprocessResult (postprocess.hpp:20-25)."""
    candidates: np.ndarray
    cluster_s: float
    dedup_s: float
    pending_candidates: int
    launches: int = 0


def _giants(g) -> np.ndarray:
    a = np.ascontiguousarray(g, dtype=GIANT_DTYPE)
    return a.reshape(-1)


class CandidatePostprocessPlan:
    """Consumes a search result view, converts coordinates, rate-limits,
    clusters across gulps and deduplicates sub-band extents, on the GPU."""

    def __init__(self, cfg: SearchConfig, layout: CandidatePostprocessLayout, device: int = 0):
        self._cfg = cfg
        h = C.c_void_p()
        check(lib().frost_postprocess_create(C.byref(cfg._c()), C.byref(layout._c()), int(device),
                                             C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_postprocess_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def execute(self, result: Union[CandidateResult, np.ndarray, FDMTBoxcar, None], samples_read: int,
                duration_samples: int, final: bool, candidate_frontier: int) -> CandidatePostprocessResult:
        out = _abi.PostprocessResultC()
        if isinstance(result, FDMTBoxcar):
            check(lib().frost_postprocess_execute_search(self._h, result._h, int(samples_read),
                                                         int(duration_samples), 1 if final else 0,
                                                         int(candidate_frontier), C.byref(out)))
        else:
            rows = result.candidates if isinstance(result, CandidateResult) else result
            if rows is None:
                rows = np.zeros(0, CANDIDATE_DTYPE)
            rows = np.ascontiguousarray(rows, dtype=CANDIDATE_DTYPE).reshape(-1)
            check(lib().frost_postprocess_execute(self._h, rows.ctypes.data if rows.size else None,
                                                  rows.size, 0, int(samples_read), int(duration_samples),
                                                  1 if final else 0, int(candidate_frontier), C.byref(out)))
        return CandidatePostprocessResult(self._results(out.count), out.cluster_s, out.dedup_s,
                                          int(out.pending_candidates), int(out.launches))

    def execute_device(self, ptr: int, n: int, samples_read: int, duration_samples: int, final: bool,
                       candidate_frontier: int) -> CandidatePostprocessResult:
        """execute over n frost_candidate rows already on the device."""
        out = _abi.PostprocessResultC()
        check(lib().frost_postprocess_execute(self._h, ptr, int(n), 1, int(samples_read),
                                              int(duration_samples), 1 if final else 0,
                                              int(candidate_frontier), C.byref(out)))
        return CandidatePostprocessResult(self._results(out.count), out.cluster_s, out.dedup_s,
                                          int(out.pending_candidates), int(out.launches))

    def _results(self, n: int) -> np.ndarray:
        g = np.zeros(n, GIANT_DTYPE)
        cnt = C.c_size_t()
        check(lib().frost_postprocess_results(self._h, g.ctypes.data if n else None, n, C.byref(cnt)))
        return g

    def memory_usage(self) -> int:
        v = C.c_uint64()
        check(lib().frost_postprocess_memory_usage(self._h, C.byref(v)))
        return int(v.value)

    @staticmethod
    def estimate_memory(cfg: SearchConfig) -> int:
        v = C.c_uint64()
        check(lib().frost_postprocess_estimate_memory(C.byref(cfg._c()), C.byref(v)))
        return int(v.value)


class ClusterLabelPlan:
    """ClusterLabelPlan (clustering.hpp:51-66), on the GPU."""

    def __init__(self, mode: ClusterMode = ClusterMode.CHAIN, device: int = 0):
        self.mode = ClusterMode(mode)
        self.device = device

    def execute(self, candidates, tol: ClusterTolerances) -> np.ndarray:
        g = _giants(candidates)
        labels = np.zeros(g.size, np.uint64)
        check(lib().frost_cluster_labels(g.ctypes.data if g.size else None, g.size, C.byref(tol._c()),
                                         int(self.mode), labels.ctypes.data if g.size else None,
                                         int(self.device)))
        return labels


class MergeCandidatesPlan:
    """MergeCandidatesPlan (merge.hpp:16-24), on the GPU."""

    def __init__(self, device: int = 0):
        self.device = device

    def execute(self, candidates, labels) -> np.ndarray:
        g = _giants(candidates)
        lab = np.ascontiguousarray(labels, dtype=np.uint64).reshape(-1)
        if lab.size != g.size:
            raise ValueError("candidates/labels size mismatch")
        out = np.zeros(g.size, GIANT_DTYPE)
        cnt = C.c_size_t()
        check(lib().frost_merge_candidates(g.ctypes.data if g.size else None,
                                           lab.ctypes.data if g.size else None, g.size,
                                           out.ctypes.data if g.size else None, C.byref(cnt),
                                           int(self.device)))
        return out[:cnt.value].copy()


class SubbandDedupPlan:
    """SubbandDedupPlan (subband_dedup.hpp:62-77), on the GPU."""

    def __init__(self, mode: SubbandDedupMode = SubbandDedupMode.TRANSITIVE, device: int = 0):
        self.mode = SubbandDedupMode(mode)
        self.device = device

    def execute(self, candidates, tol: ClusterTolerances, tsamp: float) -> np.ndarray:
        g = _giants(candidates)
        out = np.zeros(g.size, GIANT_DTYPE)
        cnt = C.c_size_t()
        check(lib().frost_subband_dedup(g.ctypes.data if g.size else None, g.size, C.byref(tol._c()),
                                        float(tsamp), int(self.mode), out.ctypes.data if g.size else None,
                                        C.byref(cnt), int(self.device)))
        return out[:cnt.value].copy()


def _giant_c(g) -> _abi.GiantC:
    a = _giants(np.asarray(g).reshape(1))
    return _abi.GiantC.from_buffer_copy(a.tobytes())


def are_coincident(a, b, tol_or_time_tol, filter_tol: Optional[int] = None, dm_tol: Optional[int] = None) -> bool:
    """are_coincident(a, b, time_tol, filter_tol, dm_tol) or
    are_coincident(a, b, ClusterTolerances) (candidate.hpp:95-110)."""
    if isinstance(tol_or_time_tol, ClusterTolerances):
        tol, physical = tol_or_time_tol, 1
    else:
        tol, physical = ClusterTolerances(int(tol_or_time_tol), int(filter_tol), int(dm_tol)), 0
    return bool(lib().frost_are_coincident(C.byref(_giant_c(a)), C.byref(_giant_c(b)), C.byref(tol._c()),
                                           physical))


def subband_time_shift_samples(dm: float, f_wide: float, f_narrow: float, tsamp: float) -> float:
    return float(lib().frost_subband_time_shift_samples(dm, f_wide, f_narrow, tsamp))


def subband_dm_step(f_low: float, f_high: float, tsamp: float) -> float:
    return float(lib().frost_subband_dm_step(f_low, f_high, tsamp))


class RateLimiter:
    """Giants-per-minute circuit breaker (rate_limiter.cpp:5-30)."""

    def __init__(self, max_giant_rate: float):
        self.max_giant_rate = float(np.float32(max_giant_rate))
        self.reset()

    def record(self, count: int, duration_seconds: float):
        self.total_giants += int(count)
        self.total_seconds += float(duration_seconds)

    def exceeded(self) -> bool:
        if self.max_giant_rate <= 0.0 or self.total_seconds <= 0.0:
            return False
        return float(self.total_giants) / (self.total_seconds / 60.0) > self.max_giant_rate

    def reset(self):
        self.total_giants = 0
        self.total_seconds = 0.0
