"""The `.cand` candidate file with frost's layout
(include/frost/output/cand_writer.hpp): CandWriter and cand_filename, over
the C ABI. Rows are GIANT_DTYPE giants (frost_b200.postprocess)."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import check, lib
from .postprocess import GIANT_DTYPE


class CandWriter:
    """CandWriter(path, dt, append) (cand_writer.hpp:38-55)."""

    def __init__(self, path: str, dt: float, append: bool = False):
        h = C.c_void_p()
        check(lib().frost_cand_writer_open(os.fsencode(path), float(dt), 1 if append else 0, C.byref(h)))
        self._h = h

    def write(self, giants, first_samp_idx: int = 0):
        g = np.ascontiguousarray(giants, GIANT_DTYPE).reshape(-1)
        check(lib().frost_cand_writer_write(self._h, g.ctypes.data if g.size else None, g.size,
                                            int(first_samp_idx)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_cand_writer_close(self._h)
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


def cand_filename(utc: int, beam: int) -> str:
    """`YYYY-MM-DD-HH:MM:SS_BB.cand` (cand_writer.cpp:73-87)."""
    buf = C.create_string_buffer(64)
    check(lib().frost_cand_filename(int(utc), int(beam), buf, len(buf)))
    return buf.value.decode()
