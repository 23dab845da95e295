"""DM trial grid and FDMT band edges (include/frost/dedisp/dedisp.hpp)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .config import DedispPlanConfig


def generate_dm_list(cfg: DedispPlanConfig) -> np.ndarray:
    """generate_dm_list (lib/dedisp/dedisp.cpp:16-69)."""
    c = cfg.to_c()
    n = C.c_size_t()
    check(lib().frost_generate_dm_list(C.byref(c), None, 0, C.byref(n)))
    out = np.empty(n.value, np.float32)
    check(lib().frost_generate_dm_list(C.byref(c), out.ctypes.data_as(C.POINTER(C.c_float)),
                                       out.size, C.byref(n)))
    return out


def band_edges(cfg: DedispPlanConfig):
    """Ascending (f_min, f_max) of make_dmt_fdmt_plan (lib/dedisp/dedisp.cpp:71-89)."""
    c = cfg.to_c()
    a, b = C.c_float(), C.c_float()
    check(lib().frost_fdmt_band_edges(C.byref(c), C.byref(a), C.byref(b)))
    return a.value, b.value
