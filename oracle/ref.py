"""TEST INFRASTRUCTURE ONLY — ctypes access to the reference's own CPU code
(oracle/_ref/libfrost_ref*.so, built from the reference sources by
oracle/Makefile). Used by the tests, smoke() and the CPU-baseline leg of
bench.py as the checker; the product path never imports it.

Wrapped: RFICleaner (lib/cpu/rfi_cpu.cpp), iqrm_mask
(lib/cpu/rfi_masks_cpu.cpp:29-122), broadband_time_flags
(lib/cpu/device_rfi_flags_cpu.cpp:17-75), spectra::measure_bandpass
(lib/cpu/spectra_cpu.cpp:73-130), KadaneState (lib/cpu/rfi_kernels.hpp:65-133),
generate_dm_list / make_dmt_fdmt_plan edges (lib/dedisp/dedisp.cpp:16-89),
read_kill_file (lib/prepare/kill_file.cpp:15-65).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from frost_b200 import _abi
from frost_b200.config import BlockLayout, DedispPlanConfig, RfiConfig

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


class ReferenceUnavailable(RuntimeError):
    pass


def lib_path(fast: bool = False) -> str:
    return os.path.join(HERE, "_ref", "libfrost_ref_fast.so" if fast else "libfrost_ref.so")


def available(fast: bool = False) -> bool:
    return os.path.exists(lib_path(fast))


def load(fast: bool = False):
    key = bool(fast)
    if key in _LIBS:
        return _LIBS[key]
    path = lib_path(fast)
    if not os.path.exists(path):
        raise ReferenceUnavailable(f"{path} is not built (run make -C oracle ref)")
    lib = C.CDLL(path)
    vp, sz, u8p, f32p = C.c_void_p, C.c_size_t, C.POINTER(C.c_uint8), C.POINTER(C.c_float)
    lib.ref_last_error.restype = C.c_char_p
    lib.ref_rfi_create.restype = vp
    lib.ref_rfi_create.argtypes = [C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC), C.c_float]
    lib.ref_rfi_destroy.argtypes = [vp]
    lib.ref_rfi_execute_normalized.argtypes = [vp, u8p, sz, sz, f32p, sz]
    lib.ref_rfi_execute.argtypes = [vp, u8p, sz]
    lib.ref_rfi_channel_mask.argtypes = [vp, u8p, sz]
    lib.ref_rfi_report.argtypes = [vp, C.POINTER(_abi.RfiReportC)]
    lib.ref_rfi_config_validate.argtypes = [C.POINTER(_abi.RfiConfigC)]
    lib.ref_iqrm_mask.argtypes = [f32p, sz, sz, C.c_float, u8p, u8p]
    lib.ref_broadband_time_flags.restype = C.c_long
    lib.ref_broadband_time_flags.argtypes = [f32p, sz, sz, C.c_float, sz, u8p]
    lib.ref_measure_bandpass.argtypes = [f32p, sz, sz, f32p, f32p]
    lib.ref_kadane.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_double), sz, sz,
                               C.POINTER(C.c_double), C.POINTER(C.c_int64),
                               C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    lib.ref_generate_dm_list.argtypes = [C.POINTER(_abi.DedispPlanConfigC), f32p, sz, C.POINTER(sz)]
    lib.ref_fdmt_band_edges.argtypes = [C.POINTER(_abi.DedispPlanConfigC), f32p, f32p]
    lib.ref_read_kill_file.argtypes = [C.c_char_p, sz, C.POINTER(_abi.ChannelRange), sz, C.POINTER(sz)]
    _LIBS[key] = lib
    return lib


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _check(lib, rc):
    if rc < 0:
        msg = lib.ref_last_error().decode()
        if rc == _abi.ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise RuntimeError(msg)
    return rc


class RefRFICleaner:
    """The reference RFICleaner (include/frost/prepare/rfi.hpp:243-297)."""

    def __init__(self, cfg: RfiConfig, layout: BlockLayout, baseline_length: float,
                 fast: bool = False):
        self.lib = load(fast)
        self.layout = layout
        c, self._keep = cfg.to_c()
        lay = layout.to_c()
        self.h = self.lib.ref_rfi_create(C.byref(c), C.byref(lay), C.c_float(baseline_length))
        if not self.h:
            raise ValueError(self.lib.ref_last_error().decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_rfi_destroy(self.h)
            self.h = None

    __del__ = close

    def execute_normalized(self, block: np.ndarray, nsamps: int = 0) -> np.ndarray:
        """Returns float32 [nchans][capacity]; `block` (uint8 bytes) is not modified."""
        buf = np.ascontiguousarray(block, dtype=np.uint8).copy()
        capacity = buf.size // self.layout.row_bytes
        out = np.empty((self.layout.nchans, capacity), dtype=np.float32)
        _check(self.lib, self.lib.ref_rfi_execute_normalized(
            self.h, _ptr(buf, C.c_uint8), buf.size, nsamps, _ptr(out, C.c_float), out.size))
        return out

    def execute(self, block: np.ndarray) -> np.ndarray:
        buf = np.ascontiguousarray(block, dtype=np.uint8).copy()
        _check(self.lib, self.lib.ref_rfi_execute(self.h, _ptr(buf, C.c_uint8), buf.size))
        return buf

    def channel_mask(self) -> np.ndarray:
        out = np.empty(self.layout.nchans, dtype=np.uint8)
        _check(self.lib, self.lib.ref_rfi_channel_mask(self.h, _ptr(out, C.c_uint8), out.size))
        return out

    def report(self) -> dict:
        r = _abi.RfiReportC()
        self.lib.ref_rfi_report(self.h, C.byref(r))
        return r.as_dict()


def iqrm_mask(x, radius, threshold, ignore=None, fast=False) -> np.ndarray:
    lib = load(fast)
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(x.size, dtype=np.uint8)
    ig = None
    if ignore is not None:
        ig = np.ascontiguousarray(ignore, dtype=np.uint8)
    _check(lib, lib.ref_iqrm_mask(_ptr(x, C.c_float), x.size, int(radius), C.c_float(threshold),
                                  _ptr(ig, C.c_uint8) if ig is not None else None,
                                  _ptr(out, C.c_uint8)))
    return out


def broadband_time_flags(series, smooth_radius, threshold, boxcar_max, flags=None):
    lib = load()
    s = np.ascontiguousarray(series, dtype=np.float32)
    f = np.zeros(s.size, dtype=np.uint8) if flags is None else np.ascontiguousarray(flags, np.uint8).copy()
    n = _check(lib, lib.ref_broadband_time_flags(_ptr(s, C.c_float), s.size, int(smooth_radius),
                                                 C.c_float(threshold), int(boxcar_max),
                                                 _ptr(f, C.c_uint8)))
    return n, f


def measure_bandpass(rows: np.ndarray):
    lib = load()
    rows = np.ascontiguousarray(rows, dtype=np.float32)
    nsamps, nchans = rows.shape
    bp = np.empty(nchans, np.float32)
    rms = np.empty(nchans, np.float32)
    _check(lib, lib.ref_measure_bandpass(_ptr(rows, C.c_float), nsamps, nchans,
                                         _ptr(bp, C.c_float), _ptr(rms, C.c_float)))
    return bp, rms


def kadane(u, idx=None, chunk_len=0):
    lib = load()
    u = np.ascontiguousarray(u, dtype=np.float64)
    idx = np.arange(u.size, dtype=np.int64) if idx is None else np.ascontiguousarray(idx, np.int64)
    s, a, b, t = C.c_double(), C.c_int64(), C.c_int64(), C.c_double()
    lib.ref_kadane(_ptr(idx, C.c_int64), _ptr(u, C.c_double), u.size, chunk_len,
                   C.byref(s), C.byref(a), C.byref(b), C.byref(t))
    return s.value, a.value, b.value, t.value


def generate_dm_list(cfg: DedispPlanConfig) -> np.ndarray:
    lib = load()
    c = cfg.to_c()
    n = C.c_size_t()
    _check(lib, lib.ref_generate_dm_list(C.byref(c), None, 0, C.byref(n)))
    out = np.empty(n.value, np.float32)
    _check(lib, lib.ref_generate_dm_list(C.byref(c), _ptr(out, C.c_float), out.size, C.byref(n)))
    return out


def fdmt_band_edges(cfg: DedispPlanConfig):
    lib = load()
    c = cfg.to_c()
    a, b = C.c_float(), C.c_float()
    _check(lib, lib.ref_fdmt_band_edges(C.byref(c), C.byref(a), C.byref(b)))
    return a.value, b.value


def read_kill_file(path: str, nchans: int):
    lib = load()
    out = (_abi.ChannelRange * max(nchans, 1))()
    n = C.c_size_t()
    _check(lib, lib.ref_read_kill_file(path.encode(), nchans, out, nchans, C.byref(n)))
    return [(out[i].start, out[i].end) for i in range(n.value)]


def rfi_config_validate(cfg: RfiConfig):
    lib = load()
    c, keep = cfg.to_c()
    _check(lib, lib.ref_rfi_config_validate(C.byref(c)))
