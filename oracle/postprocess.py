"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU checkers of the
candidate post-processing: this directory's C restatement
(postprocess_oracle.c in _build/libfrost_oracle.so) and, where it was built,
the reference's own lib/search sources (_ref/libfrost_ref_search.so, see
Makefile). Used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline as the checker; the product path never imports it.

Both back ends take and return the product's record types (frost_candidate
rows of CANDIDATE_DTYPE, frost_giant rows of GIANT_DTYPE).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from frost_b200 import _abi
from frost_b200.postprocess import (GIANT_DTYPE, CandidatePostprocessLayout, ClusterTolerances,
                                    SearchConfig)
from frost_b200.search import CANDIDATE_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(HERE, "_build", "libfrost_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libfrost_ref_search.so")

_vp, _sz, _u64 = C.c_void_p, C.c_size_t, C.c_uint64
_tolp = C.POINTER(_abi.ClusterTolerancesC)
_gp = C.POINTER(_abi.GiantC)


class PlanError(Exception):
    """An execute that the reference ends with an exception."""

    def __init__(self, kind: str, msg: str):
        super().__init__(msg)
        self.kind = kind  # "invalid_argument" or "runtime_error"


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


class Backend:
    """One CPU implementation: 'oracle' (restatement) or 'reference'."""

    def __init__(self, which: str):
        self.which = which
        if which == "oracle":
            L = C.CDLL(ORACLE_PATH)
            p = "oracle_"
            L.oracle_pp_last_error.restype = C.c_char_p
            self._err = L.oracle_pp_last_error
            L.oracle_coincident.argtypes = [_gp, _gp, _tolp]
            L.oracle_coincident_basic.argtypes = [_gp, _gp, _u64, _u64, _u64]
            L.oracle_time_shift.restype = C.c_double
            L.oracle_time_shift.argtypes = [C.c_float] * 4
            L.oracle_dm_step.restype = C.c_double
            L.oracle_dm_step.argtypes = [C.c_float] * 3
            L.oracle_cluster_labels.argtypes = [_vp, _sz, _tolp, C.c_int, _vp]
            L.oracle_merge.restype = _sz
            L.oracle_merge.argtypes = [_vp, _vp, _sz, _vp]
            L.oracle_subband_dedup.restype = C.c_long
            L.oracle_subband_dedup.argtypes = [_vp, _sz, _tolp, C.c_float, C.c_int, _vp]
            L.oracle_pp_create.restype = _vp
            L.oracle_pp_create.argtypes = [C.POINTER(_abi.PostprocessConfigC), C.POINTER(_abi.PostprocessLayoutC)]
            L.oracle_pp_destroy.argtypes = [_vp]
            L.oracle_pp_execute.restype = C.c_int
            L.oracle_pp_execute.argtypes = [_vp, _vp, _sz, _u64, _u64, C.c_int, _u64, C.POINTER(_u64)]
            L.oracle_pp_results.restype = _sz
            L.oracle_pp_results.argtypes = [_vp, _vp, _sz]
            self._merge, self._dedup, self._labels = L.oracle_merge, L.oracle_subband_dedup, L.oracle_cluster_labels
            self._create, self._destroy = L.oracle_pp_create, L.oracle_pp_destroy
            self._execute, self._results = L.oracle_pp_execute, L.oracle_pp_results
            self._shift, self._step = L.oracle_time_shift, L.oracle_dm_step
        else:
            if not ref_available():
                raise RuntimeError(f"{REF_PATH} is not built (make -C oracle ref)")
            L = C.CDLL(REF_PATH)
            L.refs_last_error.restype = C.c_char_p
            self._err = L.refs_last_error
            L.refs_are_coincident.argtypes = [_gp, _gp, _tolp, C.c_int]
            L.refs_time_shift.restype = C.c_double
            L.refs_time_shift.argtypes = [C.c_float] * 4
            L.refs_dm_step.restype = C.c_double
            L.refs_dm_step.argtypes = [C.c_float] * 3
            L.refs_cluster_labels.argtypes = [_vp, _sz, _tolp, C.c_int, _vp]
            L.refs_merge.restype = _sz
            L.refs_merge.argtypes = [_vp, _vp, _sz, _vp]
            L.refs_subband_dedup.restype = C.c_long
            L.refs_subband_dedup.argtypes = [_vp, _sz, _tolp, C.c_float, C.c_int, _vp]
            L.refs_pp_create.restype = _vp
            L.refs_pp_create.argtypes = [C.POINTER(_abi.PostprocessConfigC), C.POINTER(_abi.PostprocessLayoutC)]
            L.refs_pp_destroy.argtypes = [_vp]
            L.refs_pp_execute.restype = C.c_int
            L.refs_pp_execute.argtypes = [_vp, _vp, _sz, _u64, _u64, C.c_int, _u64, C.POINTER(_u64)]
            L.refs_pp_results.restype = _sz
            L.refs_pp_results.argtypes = [_vp, _vp, _sz]
            L.refs_cand_write.restype = C.c_int
            L.refs_cand_write.argtypes = [C.c_char_p, C.c_double, C.c_int, _vp, _sz, _u64]
            L.refs_cand_filename.restype = C.c_int
            L.refs_cand_filename.argtypes = [C.c_int64, _u64, C.c_char_p, _sz]
            L.refs_pp_memory_usage.restype = _u64
            L.refs_pp_memory_usage.argtypes = [_vp]
            self._merge, self._dedup, self._labels = L.refs_merge, L.refs_subband_dedup, L.refs_cluster_labels
            self._create, self._destroy = L.refs_pp_create, L.refs_pp_destroy
            self._execute, self._results = L.refs_pp_execute, L.refs_pp_results
            self._shift, self._step = L.refs_time_shift, L.refs_dm_step
        self.L = L

    def error(self) -> str:
        return self._err().decode(errors="replace")

    # ---- free functions ------------------------------------------------------
    def are_coincident(self, a, b, tol, physical: bool) -> bool:
        ga = _abi.GiantC.from_buffer_copy(np.asarray(a, GIANT_DTYPE).reshape(1).tobytes())
        gb = _abi.GiantC.from_buffer_copy(np.asarray(b, GIANT_DTYPE).reshape(1).tobytes())
        t = tol._c()
        if self.which == "oracle":
            if physical:
                return bool(self.L.oracle_coincident(C.byref(ga), C.byref(gb), C.byref(t)))
            return bool(self.L.oracle_coincident_basic(C.byref(ga), C.byref(gb), t.time_tol, t.filter_tol,
                                                       t.dm_tol))
        return bool(self.L.refs_are_coincident(C.byref(ga), C.byref(gb), C.byref(t), 1 if physical else 0))

    def time_shift(self, dm, f_wide, f_narrow, tsamp) -> float:
        return float(self._shift(dm, f_wide, f_narrow, tsamp))

    def dm_step(self, f_low, f_high, tsamp) -> float:
        return float(self._step(f_low, f_high, tsamp))

    def cluster_labels(self, giants, tol: ClusterTolerances, mode: int) -> np.ndarray:
        g = np.ascontiguousarray(giants, GIANT_DTYPE).reshape(-1)
        out = np.zeros(g.size, np.uint64)
        self._labels(g.ctypes.data, g.size, C.byref(tol._c()), int(mode), out.ctypes.data)
        return out

    def merge(self, giants, labels) -> np.ndarray:
        g = np.ascontiguousarray(giants, GIANT_DTYPE).reshape(-1)
        lab = np.ascontiguousarray(labels, np.uint64).reshape(-1)
        out = np.zeros(max(g.size, 1), GIANT_DTYPE)
        m = self._merge(g.ctypes.data, lab.ctypes.data, g.size, out.ctypes.data)
        return out[:m].copy()

    def subband_dedup(self, giants, tol: ClusterTolerances, tsamp: float, mode: int) -> np.ndarray:
        g = np.ascontiguousarray(giants, GIANT_DTYPE).reshape(-1)
        out = np.zeros(max(g.size, 1), GIANT_DTYPE)
        m = self._dedup(g.ctypes.data, g.size, C.byref(tol._c()), tsamp, int(mode), out.ctypes.data)
        if m < 0:
            raise PlanError("invalid_argument", self.error())
        return out[:m].copy()

    def cand_write(self, path: str, dt: float, append: bool, giants, first_samp_idx: int = 0):
        """The reference's own CandWriter (reference back end only)."""
        g = np.ascontiguousarray(giants, GIANT_DTYPE).reshape(-1)
        rc = self.L.refs_cand_write(path.encode(), dt, 1 if append else 0, g.ctypes.data if g.size else None,
                                    g.size, int(first_samp_idx))
        if rc != 0:
            raise PlanError("runtime_error", self.error())

    def cand_filename(self, utc: int, beam: int) -> str:
        buf = C.create_string_buffer(64)
        if self.L.refs_cand_filename(int(utc), int(beam), buf, len(buf)) != 0:
            raise PlanError("invalid_argument", self.error())
        return buf.value.decode()

    def plan(self, cfg: SearchConfig, layout: CandidatePostprocessLayout) -> "Plan":
        return Plan(self, cfg, layout)


class Plan:
    """CandidatePostprocessPlan on a CPU back end."""

    def __init__(self, be: Backend, cfg: SearchConfig, layout: CandidatePostprocessLayout):
        self.be = be
        self._h = be._create(C.byref(cfg._c()), C.byref(layout._c()))
        if not self._h:
            raise PlanError("invalid_argument", be.error())

    def close(self):
        if self._h:
            self.be._destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def execute(self, raw, samples_read, duration_samples, final, frontier):
        """Returns (giants, pending_candidates); raises PlanError."""
        r = np.ascontiguousarray(raw if raw is not None else np.zeros(0, CANDIDATE_DTYPE),
                                 CANDIDATE_DTYPE).reshape(-1)
        pending = C.c_uint64()
        rc = self.be._execute(self._h, r.ctypes.data if r.size else None, r.size, int(samples_read),
                              int(duration_samples), 1 if final else 0, int(frontier), C.byref(pending))
        if rc != 0:
            raise PlanError("invalid_argument" if rc == -1 else "runtime_error", self.be.error())
        n = self.be._results(self._h, None, 0)
        out = np.zeros(max(n, 1), GIANT_DTYPE)
        self.be._results(self._h, out.ctypes.data, n)
        return out[:n].copy(), int(pending.value)

    def memory_usage(self) -> int:
        return int(self.be.L.refs_pp_memory_usage(self._h))


_BACKENDS = {}


def backend(which: str = "oracle") -> Backend:
    if which not in _BACKENDS:
        _BACKENDS[which] = Backend(which)
    return _BACKENDS[which]
