"""The streaming FDMT + boxcar search engine with dmt::FDMTBoxcar's call
shape as frost uses it (lib/pipeline/pipeline.cpp:346-367, 493, 517,
598-608), running on the GPU through the C ABI."""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import _abi
from ._lib import check, lib
from .config import BoxcarConfig, DedispPlanConfig

CANDIDATE_DTYPE = np.dtype([
    ("peak_sample", np.uint64), ("begin_sample", np.uint64), ("end_sample", np.uint64),
    ("snr", np.float32), ("dm", np.float32), ("f_low_mhz", np.float32), ("f_high_mhz", np.float32),
    ("filter_idx", np.uint32), ("width", np.uint32), ("dm_idx", np.uint32),
    ("chan_begin", np.uint32), ("chan_end", np.uint32), ("beam_idx", np.uint32),
    ("subband_level", np.uint32), ("subband_idx", np.uint32)])


@dataclass
class SearchPlane:
    """get_search_plans()[p] (tests/cpp/api/calibration_test.cpp:53-134)."""
    subband_level: int
    subband_idx: int
    level: int
    chan_begin: int
    chan_end: int
    staggered: bool
    f_low: float
    f_high: float
    dm_grid: np.ndarray
    warmup_samples: np.ndarray
    widths: List[int]


@dataclass
class CandidateResult:
    """CandidateResultView: candidates plus drop counters."""
    candidates: np.ndarray
    dropped_global: int
    dropped_per_dm: int

    def overflowed(self) -> bool:
        return self.dropped_global > 0 or self.dropped_per_dm > 0


def _boxcar_c(bc: BoxcarConfig, tile_nsamps: int = 0) -> _abi.BoxcarConfigC:
    c = _abi.BoxcarConfigC()
    c.max_boxcar = int(bc.max_boxcar)
    c.wtsp = float(bc.wtsp)
    c.use_trapezoid = int(bc.use_trapezoid)
    c.detect_thresh = float(bc.detect_thresh)
    c.noise_sigma = float(bc.noise_sigma)
    c.peak_mode = int(bc.peak_mode)
    c.max_candidates = int(bc.max_candidates)
    c.max_cands_per_dm = int(bc.max_cands_per_dm)
    c.skip_cold_prefix = int(bc.skip_cold_prefix)
    c.input_nbits = 32
    c.input_mean = 0.0
    c.storage = int(bc.storage)
    c.tile_nsamps = int(tile_nsamps or bc.tile_nsamps)
    return c


class FDMTBoxcar:
    """Streaming search of one beam. execute() takes the calibrated
    [nchans][nsamps] float32 waterfall (low frequency first) as a host numpy
    array or a device pointer, plus an optional per-gulp channel mask in FDMT
    order (1 = keep)."""

    def __init__(self, plan: DedispPlanConfig, cfg: BoxcarConfig, kill_mask=None,
                 memory_budget: int = 0, device: int = 0, tile_nsamps: int = 0):
        L = lib()
        pc = plan.to_c()
        bc = _boxcar_c(cfg, tile_nsamps)
        km = None
        if kill_mask is not None:
            km = np.ascontiguousarray(kill_mask, np.uint8)
            if km.size != plan.nchans:
                raise ValueError("kill_mask must have nchans entries")
        h = C.c_void_p()
        check(L.frost_search_create(C.byref(pc), C.byref(bc),
                                    km.ctypes.data_as(C.POINTER(C.c_uint8)) if km is not None else None,
                                    memory_budget, device, C.byref(h)))
        self._h = h
        self.plan_config = plan
        self.config = cfg
        self.nchans = plan.nchans

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_search_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _mask_ptr(self, mask):
        if mask is None or (hasattr(mask, "__len__") and len(mask) == 0):
            return None, None
        m = np.ascontiguousarray(mask, np.uint8)
        if m.size != self.nchans:
            raise ValueError("mask must have nchans entries")
        return m, m.ctypes.data_as(C.POINTER(C.c_uint8))

    def execute(self, waterfall: np.ndarray, mask=None) -> CandidateResult:
        wf = np.ascontiguousarray(waterfall, np.float32)
        if wf.ndim != 2 or wf.shape[0] != self.nchans:
            raise ValueError("waterfall must be [nchans][nsamps]")
        keep, mp = self._mask_ptr(mask)
        check(lib().frost_search_execute(self._h, wf.ctypes.data_as(C.POINTER(C.c_float)),
                                         wf.shape[1], 0, mp, None))
        return self.result()

    def stream(self) -> int:
        """The engine's own CUDA stream handle."""
        s = C.c_void_p()
        check(lib().frost_search_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def execute_device(self, ptr: int, nsamps: int, mask=None, stream: Optional[int] = None):
        """A device waterfall, read after the work queued on `stream`;
        without one it is read on the engine's own stream, so its writes
        must already be complete."""
        if not stream:
            stream = self.stream()
        keep, mp = self._mask_ptr(mask)
        check(lib().frost_search_execute(self._h, C.cast(C.c_void_p(ptr), C.POINTER(C.c_float)),
                                         nsamps, 1, mp, C.c_void_p(stream) if stream else None))
        return self.result()

    def drain(self) -> CandidateResult:
        check(lib().frost_search_drain(self._h))
        return self.result()

    def result(self) -> CandidateResult:
        n, dg, dd = C.c_size_t(), C.c_uint64(), C.c_uint64()
        check(lib().frost_search_result_count(self._h, C.byref(n), C.byref(dg), C.byref(dd)))
        out = np.zeros(n.value, CANDIDATE_DTYPE)
        if n.value:
            check(lib().frost_search_results(self._h, out.ctypes.data_as(C.POINTER(_abi.CandidateC)),
                                             n.value, C.byref(n)))
        return CandidateResult(out, dg.value, dd.value)

    def get_candidate_frontier(self) -> int:
        v = C.c_uint64()
        check(lib().frost_search_frontier(self._h, C.byref(v)))
        return v.value

    def info(self) -> dict:
        i = _abi.SearchInfoC()
        check(lib().frost_search_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_}

    def widths(self) -> List[int]:
        n = C.c_size_t()
        check(lib().frost_search_widths(self._h, None, 0, C.byref(n)))
        out = (C.c_uint32 * max(n.value, 1))()
        check(lib().frost_search_widths(self._h, out, n.value, C.byref(n)))
        return [int(out[i]) for i in range(n.value)]

    def get_search_plans(self) -> List[SearchPlane]:
        info = self.info()
        ws = self.widths()
        planes = []
        for p in range(info["nplanes"]):
            pi = _abi.SearchPlaneC()
            check(lib().frost_search_plane_info(self._h, p, C.byref(pi), None, None))
            dm = np.zeros(pi.ndm, np.float32)
            warm = np.zeros(pi.ndm, np.uint32)
            check(lib().frost_search_plane_info(self._h, p, C.byref(pi),
                                                dm.ctypes.data_as(C.POINTER(C.c_float)),
                                                warm.ctypes.data_as(C.POINTER(C.c_uint32))))
            planes.append(SearchPlane(pi.subband_level, pi.subband_idx, pi.level, pi.chan_begin,
                                      pi.chan_end, bool(pi.staggered), pi.f_low, pi.f_high, dm,
                                      warm, ws))
        return planes

    def get_subband_variance_grid(self, plane: int, width: int, mask=None) -> np.ndarray:
        ndm = self.get_search_plans()[plane].dm_grid.size
        out = np.zeros(ndm, np.float64)
        keep, mp = self._mask_ptr(mask)
        check(lib().frost_search_variance_grid(self._h, plane, width, mp,
                                               out.ctypes.data_as(C.POINTER(C.c_double)), ndm))
        return out

    def autotune(self) -> dict:
        """Measures and applies the fastest FDMT launch shape for this
        geometry (call before the first gulp)."""
        f, t, c = C.c_int(), C.c_int(), C.c_int()
        ms = C.c_double()
        check(lib().frost_search_autotune(self._h, C.byref(f), C.byref(t), C.byref(ms), C.byref(c)))
        out = self.launch_shape()
        out.update({"ms": ms.value, "cached": bool(c.value)})
        return out

    def launch_shape(self) -> dict:
        """The FDMT/search launch shape in use (autotune's choice or the default)."""
        f, t, st, ch = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().frost_search_get_launch_shape(self._h, C.byref(f), C.byref(t), C.byref(st), C.byref(ch)))
        return {"fused": bool(f.value), "tiles_per_cta": t.value, "stages": st.value, "search_chunk": ch.value}

    def set_launch_shape(self, fused: bool = True, tiles_per_cta: int = 16, stages: int = 0,
                         search_chunk: int = 4096):
        """Pins a launch shape and restarts the stream (call before the first gulp)."""
        check(lib().frost_search_set_launch_shape(self._h, 1 if fused else 0, int(tiles_per_cta), int(stages),
                                                  int(search_chunk)))

    def set_residency(self, ctas_per_sm: int):
        """Caps the level and search kernels at `ctas_per_sm` resident CTAs per
        SM (0: one CTA per work item); leaves room on every SM for other
        streams' kernels. Results do not depend on it."""
        check(lib().frost_search_set_residency(self._h, int(ctas_per_sm)))

    def residency(self) -> int:
        v = C.c_int()
        check(lib().frost_search_get_residency(self._h, C.byref(v)))
        return v.value

    def set_fused_search(self, mode: int = 1):
        """Fuses each single FDMT level step into a searched level with that
        level's search (mode 1 or 2: chunks staged at once; 0: off; default
        1). Results are identical either way."""
        check(lib().frost_search_set_fused_search(self._h, int(mode)))

    def fused_search(self) -> int:
        v = C.c_int()
        check(lib().frost_search_get_fused_search(self._h, C.byref(v)))
        return v.value

    def set_wait_limit(self, tries: int = -1):
        """Bound (mbarrier tries) of the kernels' first wait on each bulk
        copy; negative restores the default, 0 gives up at once. A
        diagnostic of the timeout path."""
        check(lib().frost_search_set_wait_limit(self._h, int(tries)))

    def restart(self):
        """Starts the stream afresh (after a gulp that failed)."""
        check(lib().frost_search_restart(self._h))

    def use_graphs(self, enable: bool = True):
        """CUDA-graph replay of the per-gulp launch sequence (default on)."""
        check(lib().frost_search_use_graphs(self._h, 1 if enable else 0))

    def enable_timing(self, enable: bool = True):
        check(lib().frost_search_enable_timing(self._h, int(enable)))

    def timing(self) -> dict:
        t = _abi.SearchTimingC()
        check(lib().frost_search_get_timing(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def capture_planes(self, enable: bool = True):
        check(lib().frost_search_capture_planes(self._h, int(enable)))

    def plane_data(self, plane: int, nsamps: int) -> np.ndarray:
        ndm = self.get_search_plans()[plane].dm_grid.size
        out = np.zeros((ndm, nsamps), np.float32)
        check(lib().frost_search_plane_data(self._h, plane, out.ctypes.data_as(C.POINTER(C.c_float)),
                                            out.size))
        return out


def candidate_list_diff(ref: np.ndarray, other: np.ndarray, snr_min: float = 7.0,
                        tie_rtol: float = 1e-2) -> dict:
    """Compares two candidate lists of the same stream (for example FP16
    plane storage against FP32) above `snr_min`.

    A detection is keyed by (subband_level, subband_idx, dm_idx, filter_idx).
    A detection of either list at S/N >= snr_min is `matched` when the other
    list (at any S/N it reports, down to its detection threshold) has the
    same key and the same peak sample; `moved` when the other list's
    detection of that key covers the same run with a different peak whose
    S/N is within tie_rtol (a near tie inside the run); otherwise it counts
    in `only_ref` / `only_other` (no detection of that key covers it, or the
    covering run peaks elsewhere with a different S/N: runs split or merged
    at the detection threshold). `max_snr_rel_err` is the largest relative
    S/N difference over matched pairs, `moved_max_snr_rel_err` over moved
    ones; `edge` counts matched pairs with one side below snr_min (a
    threshold crossing, not a missing detection)."""
    def index(cs):
        out = {}
        for c in cs:
            k = (int(c["subband_level"]), int(c["subband_idx"]), int(c["dm_idx"]), int(c["filter_idx"]))
            out.setdefault(k, []).append((int(c["begin_sample"]), int(c["end_sample"]),
                                          int(c["peak_sample"]), float(c["snr"])))
        return out
    a, b = index(ref), index(other)
    res = {"snr_min": snr_min, "n_ref": 0, "n_other": 0, "matched": 0, "moved": 0, "only_ref": 0,
           "only_other": 0, "edge": 0, "max_snr_rel_err": 0.0, "moved_max_snr_rel_err": 0.0}

    def walk(x, y, count_key, only_key, pairs):
        for k, lst in x.items():
            for beg, end, pk, snr in lst:
                if snr < snr_min:
                    continue
                res[count_key] += 1
                cand = y.get(k, [])
                same = [d for d in cand if d[2] == pk]
                if same:
                    # the second walk counts only pairs the first one skipped
                    # (the reference side below snr_min)
                    if pairs or same[0][3] < snr_min:
                        res["matched"] += 1
                        res["max_snr_rel_err"] = max(res["max_snr_rel_err"], abs(same[0][3] - snr) / abs(snr))
                        res["edge"] += int(same[0][3] < snr_min)
                    continue
                near = [d for d in cand if (d[0] <= pk <= d[1] or beg <= d[2] <= end)
                        and abs(d[3] - snr) <= tie_rtol * abs(snr)]
                if near:
                    if pairs or near[0][3] < snr_min:
                        res["moved"] += 1
                        res["moved_max_snr_rel_err"] = max(res["moved_max_snr_rel_err"],
                                                           abs(near[0][3] - snr) / abs(snr))
                    continue
                res[only_key] += 1
    walk(a, b, "n_ref", "only_ref", True)
    walk(b, a, "n_other", "only_other", False)
    res["identical"] = res["only_ref"] == 0 and res["only_other"] == 0 and res["moved"] == 0
    return res
