"""Per-gulp search pipeline of one beam: Pipeline::execute_block's hot path
(lib/pipeline/pipeline.cpp:529-619) — RFI excision and normalisation, the
channel mask in FDMT order (fdmt_kill_mask, :334-344), the streaming FDMT +
boxcar search, and frost's searched-samples accounting (:610-614) — with the
waterfall kept on the GPU between the stages."""

from __future__ import annotations

from typing import Optional

import numpy as np

from .config import BlockLayout, BoxcarConfig, DedispPlanConfig, RfiConfig
from .rfi import RFICleaner
from .search import CandidateResult, FDMTBoxcar


def plan_for(layout: BlockLayout, dm_min: float, dm_max: float, subband_depth: int,
             dm_tol: float = 1.25, dm_pulse_width: float = 40.0) -> DedispPlanConfig:
    """make_dedisp_plan_config (lib/pipeline/pipeline.cpp:290-304)."""
    return DedispPlanConfig(nchans=layout.nchans, dt=float(layout.tsamp), f0=float(layout.f0),
                            df=float(layout.df), dm_min=dm_min, dm_max=dm_max,
                            dm_pulse_width=dm_pulse_width, dm_tol=dm_tol,
                            block_nsamps=layout.max_nsamps, subband_depth=subband_depth)


class GulpPipeline:
    def __init__(self, rfi_cfg: RfiConfig, layout: BlockLayout, baseline_length: float,
                 plan: DedispPlanConfig, search_cfg: BoxcarConfig, device: int = 0,
                 tile_nsamps: int = 0, memory_budget: int = 0, postprocess=None):
        """`postprocess` (a frost_b200.postprocess.SearchConfig) adds
        CandidatePostprocessPlan after every gulp's search, as
        Pipeline::publish does (lib/pipeline/pipeline.cpp:478-493); its
        result of the last gulp is `self.postprocessed`."""
        self.layout = layout
        self.rfi = RFICleaner(rfi_cfg, layout, baseline_length, device)
        self.descending = layout.df < 0
        static = self.rfi.channel_mask()
        self.static_fdmt = static[::-1].copy() if self.descending else static.copy()
        self.search = FDMTBoxcar(plan, search_cfg, kill_mask=self.static_fdmt,
                                 memory_budget=memory_budget, device=device,
                                 tile_nsamps=tile_nsamps)
        self.max_delay = self.search.info()["dt_max"]
        self.samples_read = 0
        self.samples_searched = 0
        self.block = layout.max_nsamps
        self.post = None
        self.postprocessed = None
        self._last_nread = 0
        if postprocess is not None:
            from .postprocess import CandidatePostprocessLayout, CandidatePostprocessPlan
            self.post = CandidatePostprocessPlan(
                postprocess, CandidatePostprocessLayout(layout.nchans, layout.tsamp, layout.df), device)

    def _fdmt_mask(self):
        m = self.rfi.channel_mask()
        return m[::-1].copy() if self.descending else m

    def _account(self, nread: int):
        self.samples_read += nread
        previous = self.samples_read - nread
        if self.samples_read > self.max_delay:
            self.samples_searched += self.samples_read - max(previous, self.max_delay)

    def execute_device(self, raw_ptr: int, nread: int, on_device: bool = True,
                       stream: Optional[int] = None) -> CandidateResult:
        """One gulp whose packed block (block rows, `nread` valid) is at
        raw_ptr (device, or pinned host when on_device is False). A device
        block is read after the work queued on `stream` (default: the
        cleaner's own stream, so the block must be complete)."""
        nbytes = self.block * self.layout.row_bytes
        s = stream or self.rfi.stream()
        wf = self.rfi.execute_normalized_device(raw_ptr, nbytes, nread, on_device=on_device, stream=s)
        # the engine reads the waterfall after the cleaner's work on `s`
        res = self.search.execute_device(wf, self.block, self._fdmt_mask(), stream=s)
        self._account(nread)
        self._last_nread = nread
        if self.post is not None:
            self.postprocessed = self.post.execute(self.search, self.samples_read, nread, False,
                                                   self.search.get_candidate_frontier())
        return res

    def execute(self, block: np.ndarray, nread: int = 0) -> CandidateResult:
        buf = np.ascontiguousarray(block).view(np.uint8).reshape(-1)
        nread = nread or self.block
        return self.execute_device(buf.ctypes.data, nread, on_device=False)

    def flush(self) -> CandidateResult:
        res = self.search.drain()
        if self.post is not None:
            self.postprocessed = self.post.execute(self.search, self.samples_read, self._last_nread, True,
                                                   self.search.get_candidate_frontier())
        return res
