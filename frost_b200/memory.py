"""Memory planning for one beam on the device: frost's MemoryEstimate and
check_memory (include/frost/pipeline/memory.hpp, lib/pipeline/memory.cpp:
294-508) for this implementation's own buffers, computed on the host from
the plans without allocating anything (frost_estimate_memory,
frost_check_memory)."""

from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

from . import _abi
from ._lib import check, lib
from .config import BlockLayout, BoxcarConfig, DedispPlanConfig, RfiConfig
from .search import _boxcar_c


@dataclasses.dataclass
class MemoryEstimate:
    rfi_bytes: int
    fdmt_bytes: int
    search_bytes: int
    postprocess_bytes: int
    transient_bytes: int
    total_bytes: int
    max_delay: int

    @staticmethod
    def _of(c: _abi.MemoryEstimateC) -> "MemoryEstimate":
        return MemoryEstimate(*(int(getattr(c, f)) for f, _ in _abi.MemoryEstimateC._fields_))


@dataclasses.dataclass
class MemoryCheck:
    estimate: MemoryEstimate
    requested_bytes: int
    available_bytes: int
    gulp_requested: int
    gulp_used: int
    lowered: bool
    device_memory: bool


def _args(rfi_cfg: RfiConfig, layout: BlockLayout, plan: DedispPlanConfig, search_cfg: BoxcarConfig, post):
    rc, keep = rfi_cfg.to_c()
    return rc, keep, layout.to_c(), plan.to_c(), _boxcar_c(search_cfg), (post._c() if post is not None else None)


def estimate_memory(rfi_cfg: RfiConfig, layout: BlockLayout, baseline_length: float, plan: DedispPlanConfig,
                    search_cfg: BoxcarConfig, post=None) -> MemoryEstimate:
    """Device bytes of a beam of `layout` (max_nsamps is the gulp; the
    plan's block_nsamps must equal it), `plan`, `search_cfg` and, if given,
    the post-processor (frost_b200.postprocess.SearchConfig)."""
    rc, keep, lay, pc, bc, pp = _args(rfi_cfg, layout, plan, search_cfg, post)
    out = _abi.MemoryEstimateC()
    check(lib().frost_estimate_memory(C.byref(rc), C.byref(lay), C.c_float(baseline_length), C.byref(pc),
                                      C.byref(bc), C.byref(pp) if pp is not None else None, C.byref(out)))
    return MemoryEstimate._of(out)


def check_memory(rfi_cfg: RfiConfig, layout: BlockLayout, baseline_length: float, plan: DedispPlanConfig,
                 search_cfg: BoxcarConfig, post=None, gulp_is_default: bool = True, available_bytes: int = 0,
                 memory_limit_bytes: int = 0, device: int = 0) -> MemoryCheck:
    """check_memory for the device: compares the estimate with 90 % of the
    available device memory (`available_bytes`, else the device's free
    memory, capped by `memory_limit_bytes`); lowers a default gulp to the
    largest multiple of 1024 samples that fits (`layout.max_nsamps` and
    `plan.block_nsamps` are updated), or raises FrostError with code
    FROST_ERR_OUT_OF_MEMORY naming the largest gulp that fits."""
    rc, keep, lay, pc, bc, pp = _args(rfi_cfg, layout, plan, search_cfg, post)
    out = _abi.MemoryCheckC()
    check(lib().frost_check_memory(C.byref(rc), C.byref(lay), C.c_float(baseline_length), C.byref(pc),
                                   C.byref(bc), C.byref(pp) if pp is not None else None,
                                   1 if gulp_is_default else 0, int(available_bytes), int(memory_limit_bytes),
                                   int(device), C.byref(out)))
    if out.lowered:
        layout.max_nsamps = int(out.gulp_used)
        plan.block_nsamps = int(out.gulp_used)
    return MemoryCheck(MemoryEstimate._of(out.estimate), int(out.requested_bytes), int(out.available_bytes),
                       int(out.gulp_requested), int(out.gulp_used), bool(out.lowered), bool(out.device_memory))
