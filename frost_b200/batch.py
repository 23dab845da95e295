"""Batched multi-beam search through the C ABI (frost_batch_*): one gulp of
every beam per call, the beams' RFI stages run concurrently, then their
searches in rounds whose level steps and searches are single launches over
all beams (segment tables), captured once as a CUDA graph. Beams may differ
in channel count, sample type, gulp length, DM range and plane count; a
beam's candidates equal those of the same beam run alone. frost itself runs
one engine per pipeline and one beam per process
(lib/pipeline/pipeline.cpp:346-367)."""

from __future__ import annotations

import ctypes as C
from typing import List, Sequence

import numpy as np

from . import _abi
from ._lib import check, lib
from .config import BlockLayout, BoxcarConfig, DedispPlanConfig, RfiConfig
from .search import CANDIDATE_DTYPE, _boxcar_c


class BeamBatch:
    def __init__(self, device: int = 0, memory_budget: int = 0):
        h = C.c_void_p()
        check(lib().frost_batch_create(device, memory_budget, C.byref(h)))
        self._h = h
        self._capacity: List[int] = []
        self._layouts: List[BlockLayout] = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_beam(self, rfi_cfg: RfiConfig, layout: BlockLayout, baseline_length: float,
                 plan: DedispPlanConfig, search_cfg: BoxcarConfig) -> int:
        """Admits a beam (numbered in the order added); raises
        FrostError(ERR_OUT_OF_MEMORY) beyond the batch's budget."""
        c, keep = rfi_cfg.to_c()
        lay, pc, bc = layout.to_c(), plan.to_c(), _boxcar_c(search_cfg)
        beam = C.c_uint32()
        check(lib().frost_batch_add_beam(self._h, C.byref(c), C.byref(lay), C.c_float(baseline_length),
                                         C.byref(pc), C.byref(bc), C.byref(beam)))
        self._capacity.append(max(1, int(search_cfg.max_candidates)))
        self._layouts.append(layout)
        return beam.value

    def execute_ptrs(self, ptrs: Sequence[int], nread: Sequence[int], on_device: bool) -> None:
        """One gulp of every beam from block addresses (device memory when
        on_device, complete; else host memory, preferably pinned)."""
        n = len(self._layouts)
        if len(ptrs) != n or len(nread) != n:
            raise ValueError("one block and one nread per beam")
        blocks = (C.c_void_p * n)(*[C.c_void_p(int(p)) for p in ptrs])
        counts = (C.c_size_t * n)(*[int(x) for x in nread])
        check(lib().frost_batch_execute(self._h, blocks, counts, 1 if on_device else 0))

    def execute(self, blocks: Sequence[np.ndarray], nread: Sequence[int] = ()) -> List[np.ndarray]:
        """One gulp of every beam from host blocks (whole blocks of each
        beam's max_nsamps rows); returns each beam's candidates."""
        bufs = [np.ascontiguousarray(b).view(np.uint8).reshape(-1) for b in blocks]
        counts = list(nread) or [lay.max_nsamps for lay in self._layouts]
        self.execute_ptrs([b.ctypes.data for b in bufs], counts, on_device=False)
        return [self.results(k) for k in range(len(bufs))]

    def results(self, beam: int) -> np.ndarray:
        cap = self._capacity[beam]
        out = np.zeros(cap, CANDIDATE_DTYPE)
        n = C.c_size_t()
        check(lib().frost_batch_results(self._h, beam, out.ctypes.data_as(C.POINTER(_abi.CandidateC)), cap,
                                        C.byref(n)))
        return out[:n.value]

    def drain(self, beam: int) -> np.ndarray:
        cap = self._capacity[beam]
        out = np.zeros(cap, CANDIDATE_DTYPE)
        n = C.c_size_t()
        check(lib().frost_batch_drain(self._h, beam, out.ctypes.data_as(C.POINTER(_abi.CandidateC)), cap,
                                      C.byref(n)))
        return out[:n.value]

    def use_graph(self, enable: bool = True) -> None:
        check(lib().frost_batch_use_graph(self._h, 1 if enable else 0))

    def stats(self) -> dict:
        s = _abi.BatchStatsC()
        check(lib().frost_batch_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}
