"""RFI excision with frost's RFICleaner interface
(include/frost/prepare/rfi.hpp:243-297), running on the GPU through the
C ABI."""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._lib import check, lib
from .config import BlockLayout, RfiConfig


def _u8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


class RFICleaner:
    """Cleans and normalises packed time-major gulps on `device`.

    execute_normalized() returns float32 [nchans][capacity], low frequency
    first, masked channels and padding zero — as the reference cleaner's
    execute_normalized (lib/cpu/rfi_cpu.cpp:161-260).
    """

    def __init__(self, cfg: RfiConfig, layout: BlockLayout, baseline_length: float,
                 device: int = 0):
        L = lib()
        c, keep = cfg.to_c()
        lay = layout.to_c()
        h = C.c_void_p()
        check(L.frost_rfi_create(C.byref(c), C.byref(lay), C.c_float(baseline_length), device,
                                 C.byref(h)))
        self._h = h
        self.cfg = cfg
        self.layout = layout
        self.device = device
        self._capacity = 0

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_rfi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self) -> int:
        """The cleaner's own CUDA stream handle."""
        s = C.c_void_p()
        check(lib().frost_rfi_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def execute_normalized_device(self, block_ptr: int, block_bytes: int, nsamps: int = 0,
                                  on_device: bool = True, stream: Optional[int] = None) -> int:
        """Runs on a block at `block_ptr` (device pointer when on_device, else a
        host address); returns the device pointer of the normalized waterfall
        (complete on return). A device block is read after the work queued
        on `stream`; without one it is read on the cleaner's own stream, so
        its writes must already be complete."""
        if on_device and not stream:
            stream = self.stream()
        out = C.c_void_p()
        check(lib().frost_rfi_execute_normalized(self._h, C.c_void_p(block_ptr), block_bytes, nsamps,
                                                 1 if on_device else 0,
                                                 C.c_void_p(stream) if stream else None,
                                                 C.byref(out)))
        self._capacity = block_bytes // self.layout.row_bytes
        return out.value

    def execute_normalized(self, block: np.ndarray, nsamps: int = 0) -> np.ndarray:
        """Host block in, host [nchans][capacity] float32 out (input unchanged)."""
        buf = np.ascontiguousarray(block).view(np.uint8).reshape(-1)
        self.execute_normalized_device(buf.ctypes.data, buf.size, nsamps, on_device=False)
        return self.download()

    def download(self) -> np.ndarray:
        out = np.empty((self.layout.nchans, self._capacity), dtype=np.float32)
        check(lib().frost_rfi_download_normalized(self._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                  out.size))
        return out

    def channel_mask(self) -> np.ndarray:
        out = np.empty(self.layout.nchans, np.uint8)
        check(lib().frost_rfi_channel_mask(self._h, _u8(out), out.size))
        return out

    def time_flags(self, nsamps: int) -> np.ndarray:
        out = np.zeros(nsamps, np.uint8)
        check(lib().frost_rfi_time_flags(self._h, _u8(out), out.size))
        return out

    def report(self) -> dict:
        r = _abi.RfiReportC()
        check(lib().frost_rfi_get_report(self._h, C.byref(r)))
        return r.as_dict()

    def launches(self) -> int:
        n = C.c_uint64()
        check(lib().frost_rfi_launch_count(self._h, C.byref(n)))
        return n.value

    def memory_usage(self) -> int:
        n = C.c_size_t()
        check(lib().frost_rfi_memory_usage(self._h, C.byref(n)))
        return n.value


def iqrm_mask(x, radius: int, threshold: float, ignore=None) -> np.ndarray:
    """IQRM (lib/cpu/rfi_masks_cpu.cpp:29-122); 1 = flagged."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros(x.size, np.uint8)
    ig = None if ignore is None else np.ascontiguousarray(ignore, dtype=np.uint8)
    check(lib().frost_iqrm_mask(x.ctypes.data_as(C.POINTER(C.c_float)), x.size, int(radius),
                                C.c_float(threshold), _u8(ig) if ig is not None else None, _u8(out)))
    return out


def apply_manual_killmask(killmask: np.ndarray, zaps) -> np.ndarray:
    m = np.ascontiguousarray(killmask, dtype=np.uint8).copy()
    arr = (_abi.ChannelRange * max(len(zaps), 1))(*[_abi.ChannelRange(a, b) for a, b in zaps])
    check(lib().frost_apply_manual_killmask(_u8(m), m.size, arr, len(zaps)))
    return m


def read_kill_file(path: str, nchans: int):
    out = (_abi.ChannelRange * max(nchans, 1))()
    n = C.c_size_t()
    check(lib().frost_read_kill_file(str(path).encode(), nchans, out, nchans, C.byref(n)))
    return [(out[i].start, out[i].end) for i in range(n.value)]
