"""Many beams searched on one GPU through the C ABI's server
(frost_server_*): each beam keeps its RFI calibration and FDMT tails
resident, beams are admitted by device memory, and queued gulps are taken by
worker slots oldest first, one gulp per beam at a time. frost itself runs one
beam per process and overlaps only the read of the next gulp
(GulpPrefetch, lib/pipeline/pipeline.cpp:109-262)."""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, Tuple

import numpy as np

from . import _abi
from ._lib import check, lib
from .config import BlockLayout, BoxcarConfig, DedispPlanConfig, RfiConfig
from .search import CANDIDATE_DTYPE, _boxcar_c


@dataclass
class ServerStats:
    completed: int
    beams: int
    device_bytes: int
    beam_seconds: float
    wall_seconds: float
    p50_latency_s: float
    p99_latency_s: float
    max_latency_s: float
    launches: int

    @property
    def beam_seconds_per_second(self) -> float:
        return self.beam_seconds / self.wall_seconds if self.wall_seconds > 0 else 0.0


class BeamServer:
    def __init__(self, device: int = 0, memory_budget: int = 0, slots: int = 4):
        h = C.c_void_p()
        check(lib().frost_server_create(device, memory_budget, slots, C.byref(h)))
        self._h = h
        self._capacity: Dict[int, int] = {}
        self._beam_of: Dict[int, int] = {}
        self._blocks: Dict[int, np.ndarray] = {}
        self._giant_capacity: Dict[int, int] = {}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_beam(self, rfi_cfg: RfiConfig, layout: BlockLayout, baseline_length: float,
                 plan: DedispPlanConfig, search_cfg: BoxcarConfig) -> int:
        """Admits a beam; raises FrostError(ERR_OUT_OF_MEMORY) when its
        device memory would exceed the server's budget."""
        c, keep = rfi_cfg.to_c()
        lay, pc, bc = layout.to_c(), plan.to_c(), _boxcar_c(search_cfg)
        beam = C.c_uint32()
        check(lib().frost_server_add_beam(self._h, C.byref(c), C.byref(lay), C.c_float(baseline_length),
                                          C.byref(pc), C.byref(bc), C.byref(beam)))
        # results of one gulp never exceed the engine's max_candidates
        self._capacity[beam.value] = max(1, int(search_cfg.max_candidates))
        return beam.value

    def remove_beam(self, beam: int):
        check(lib().frost_server_remove_beam(self._h, beam))
        self._capacity.pop(beam, None)

    def submit(self, beam: int, block: np.ndarray, nread: int) -> int:
        """Queues one gulp (a whole host block of max_nsamps rows, `nread`
        valid); the block is kept alive until wait() returns its ticket."""
        buf = np.ascontiguousarray(block).view(np.uint8).reshape(-1)
        ticket = self.submit_ptr(beam, buf.ctypes.data, buf.size, nread, on_device=False)
        self._blocks[ticket] = buf
        return ticket

    def submit_ptr(self, beam: int, ptr: int, nbytes: int, nread: int, on_device: bool) -> int:
        """Queues one gulp at `ptr` (device memory of the server's device
        when on_device, else host memory, preferably pinned); the caller
        keeps it valid until wait() returns the ticket."""
        ticket = C.c_uint64()
        check(lib().frost_server_submit(self._h, beam, C.c_void_p(ptr), nbytes, nread,
                                        1 if on_device else 0, C.byref(ticket)))
        self._beam_of[ticket.value] = beam
        return ticket.value

    def wait(self, ticket: int) -> Tuple[np.ndarray, float]:
        """Candidates of the gulp (sorted as the engine's results) and its
        latency from submit to candidates ready, in seconds."""
        cap = self._capacity[self._beam_of[ticket]]
        out = np.zeros(cap, CANDIDATE_DTYPE)
        n, lat = C.c_size_t(), C.c_double()
        try:
            check(lib().frost_server_wait(self._h, ticket, out.ctypes.data_as(C.POINTER(_abi.CandidateC)),
                                          cap, C.byref(n), C.byref(lat)))
        finally:
            self._blocks.pop(ticket, None)
            self._beam_of.pop(ticket, None)
        return out[:n.value], lat.value

    def set_residency(self, beam: int, ctas_per_sm: int) -> None:
        """Caps the beam's level and search kernels at `ctas_per_sm` resident
        CTAs per SM (0: one CTA per work item), so that the served beams'
        kernels share the SMs instead of queueing behind each other."""
        check(lib().frost_server_set_residency(self._h, beam, int(ctas_per_sm)))

    def set_staging(self, beam: int, slots: int) -> None:
        """Gives `beam` `slots` (0-4) device blocks that pinned host gulps
        are copied into when they are submitted, so that with more than one
        gulp in flight a gulp's upload overlaps the work on the one before
        it (GulpPrefetch's overlap, lib/pipeline/pipeline.cpp:105-262).
        Charged to the server's memory budget."""
        check(lib().frost_server_set_staging(self._h, beam, int(slots)))

    def set_postprocess(self, beam: int, cfg) -> None:
        """Adds CandidatePostprocessPlan (frost_b200.postprocess.SearchConfig)
        after every gulp's search of `beam`; wait_giants / drain_giants then
        return its giants."""
        check(lib().frost_server_set_postprocess(self._h, beam, C.byref(cfg._c())))
        pend = cfg.max_pending_candidates or cfg.max_candidates
        self._giant_capacity[beam] = max(1, int(cfg.max_candidates + pend))

    def wait_giants(self, ticket: int):
        """The gulp's post-processed giants (GIANT_DTYPE) and its latency."""
        from .postprocess import GIANT_DTYPE
        cap = self._giant_capacity[self._beam_of[ticket]]
        out = np.zeros(cap, GIANT_DTYPE)
        n, lat = C.c_size_t(), C.c_double()
        try:
            check(lib().frost_server_wait_giants(self._h, ticket, out.ctypes.data, cap, C.byref(n),
                                                 C.byref(lat)))
        finally:
            self._blocks.pop(ticket, None)
            self._beam_of.pop(ticket, None)
        return out[:n.value].copy(), lat.value

    def drain_giants(self, beam: int) -> np.ndarray:
        from .postprocess import GIANT_DTYPE
        cap = self._giant_capacity[beam]
        out = np.zeros(cap, GIANT_DTYPE)
        n = C.c_size_t()
        check(lib().frost_server_drain_giants(self._h, beam, out.ctypes.data, cap, C.byref(n)))
        return out[:n.value].copy()

    def drain(self, beam: int) -> np.ndarray:
        cap = self._capacity[beam]
        out = np.zeros(cap, CANDIDATE_DTYPE)
        n = C.c_size_t()
        check(lib().frost_server_drain(self._h, beam, out.ctypes.data_as(C.POINTER(_abi.CandidateC)),
                                       cap, C.byref(n)))
        return out[:n.value]

    def stats(self) -> ServerStats:
        s = _abi.ServerStatsC()
        check(lib().frost_server_get_stats(self._h, C.byref(s)))
        return ServerStats(s.completed, s.beams, s.device_bytes, s.beam_seconds, s.wall_seconds,
                           s.p50_latency_s, s.p99_latency_s, s.max_latency_s, s.launches)

    def reset_stats(self):
        check(lib().frost_server_reset_stats(self._h))
