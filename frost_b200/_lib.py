"""Loads the in-tree C-ABI library (frost_b200/lib/libfrost_b200.so) and
declares the signatures of include/frost_b200.h. There is no fallback: a
missing library raises, so every call in this package runs the CUDA path.
"""

from __future__ import annotations

import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfrost_b200.so")

_lib = None


class FrostError(RuntimeError):
    """A frost_b200 call failed with a status other than INVALID_ARGUMENT."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


# Every symbol include/frost_b200.h declares, with (restype, argtypes).
_vp, _sz, _u8p, _f32p, _u64 = C.c_void_p, C.c_size_t, C.POINTER(C.c_uint8), C.POINTER(C.c_float), C.c_uint64
SIGNATURES = {
    "frost_last_error": (C.c_char_p, []),
    "frost_version": (C.c_char_p, []),
    "frost_rfi_config_default": (None, [C.POINTER(_abi.RfiConfigC)]),
    "frost_rfi_config_validate": (C.c_int, [C.POINTER(_abi.RfiConfigC)]),
    "frost_rfi_create": (C.c_int, [C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC),
                                   C.c_float, C.c_int, C.POINTER(_vp)]),
    "frost_rfi_destroy": (C.c_int, [_vp]),
    "frost_rfi_execute_normalized": (C.c_int, [_vp, _vp, _sz, _sz, C.c_int, _vp, C.POINTER(_vp)]),
    "frost_rfi_download_normalized": (C.c_int, [_vp, _f32p, _sz]),
    "frost_rfi_channel_mask": (C.c_int, [_vp, _u8p, _sz]),
    "frost_rfi_get_report": (C.c_int, [_vp, C.POINTER(_abi.RfiReportC)]),
    "frost_rfi_time_flags": (C.c_int, [_vp, _u8p, _sz]),
    "frost_rfi_memory_usage": (C.c_int, [_vp, C.POINTER(_sz)]),
    "frost_rfi_launch_count": (C.c_int, [_vp, C.POINTER(_u64)]),
    "frost_rfi_normalize_static": (C.c_int, [C.POINTER(_abi.BlockLayoutC), C.c_float, _vp, _sz, _sz,
                                             _vp, _sz, _vp]),
    "frost_iqrm_mask": (C.c_int, [_f32p, _sz, _u64, C.c_float, _u8p, _u8p]),
    "frost_apply_manual_killmask": (C.c_int, [_u8p, _sz, C.POINTER(_abi.ChannelRange), _sz]),
    "frost_read_kill_file": (C.c_int, [C.c_char_p, _sz, C.POINTER(_abi.ChannelRange), _sz,
                                       C.POINTER(_sz)]),
    "frost_generate_dm_list": (C.c_int, [C.POINTER(_abi.DedispPlanConfigC), _f32p, _sz, C.POINTER(_sz)]),
    "frost_fdmt_band_edges": (C.c_int, [C.POINTER(_abi.DedispPlanConfigC), _f32p, _f32p]),
    "frost_search_create": (C.c_int, [C.POINTER(_abi.DedispPlanConfigC), C.POINTER(_abi.BoxcarConfigC),
                                      _u8p, _sz, C.c_int, C.POINTER(_vp)]),
    "frost_search_destroy": (C.c_int, [_vp]),
    "frost_search_execute": (C.c_int, [_vp, _f32p, _sz, C.c_int, _u8p, _vp]),
    "frost_search_get_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "frost_search_set_wait_limit": (C.c_int, [_vp, C.c_int64]),
    "frost_search_restart": (C.c_int, [_vp]),
    "frost_batch_create": (C.c_int, [C.c_int, _sz, C.POINTER(_vp)]),
    "frost_batch_destroy": (C.c_int, [_vp]),
    "frost_batch_add_beam": (C.c_int, [_vp, C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC), C.c_float,
                                       C.POINTER(_abi.DedispPlanConfigC), C.POINTER(_abi.BoxcarConfigC),
                                       C.POINTER(C.c_uint32)]),
    "frost_batch_execute": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_sz), C.c_int]),
    "frost_batch_results": (C.c_int, [_vp, C.c_uint32, _vp, _sz, C.POINTER(_sz)]),
    "frost_batch_drain": (C.c_int, [_vp, C.c_uint32, _vp, _sz, C.POINTER(_sz)]),
    "frost_batch_use_graph": (C.c_int, [_vp, C.c_int]),
    "frost_batch_get_stats": (C.c_int, [_vp, C.POINTER(_abi.BatchStatsC)]),
    "frost_rfi_get_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "frost_search_drain": (C.c_int, [_vp]),
    "frost_search_result_count": (C.c_int, [_vp, C.POINTER(_sz), C.POINTER(_u64), C.POINTER(_u64)]),
    "frost_search_results": (C.c_int, [_vp, C.POINTER(_abi.CandidateC), _sz, C.POINTER(_sz)]),
    "frost_search_frontier": (C.c_int, [_vp, C.POINTER(_u64)]),
    "frost_search_get_info": (C.c_int, [_vp, C.POINTER(_abi.SearchInfoC)]),
    "frost_search_plane_info": (C.c_int, [_vp, _sz, C.POINTER(_abi.SearchPlaneC), _f32p,
                                          C.POINTER(C.c_uint32)]),
    "frost_search_widths": (C.c_int, [_vp, C.POINTER(C.c_uint32), _sz, C.POINTER(_sz)]),
    "frost_search_variance_grid": (C.c_int, [_vp, _sz, C.c_uint32, _u8p, C.POINTER(C.c_double), _sz]),
    "frost_search_capture_planes": (C.c_int, [_vp, C.c_int]),
    "frost_search_plane_data": (C.c_int, [_vp, _sz, _f32p, _sz]),
    "frost_search_use_graphs": (C.c_int, [_vp, C.c_int]),
    "frost_search_autotune": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                        C.POINTER(C.c_int)]),
    "frost_search_set_launch_shape": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "frost_search_set_residency": (C.c_int, [_vp, C.c_int]),
    "frost_search_get_residency": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "frost_search_set_fused_search": (C.c_int, [_vp, C.c_int]),
    "frost_search_get_fused_search": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "frost_search_get_launch_shape": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                C.POINTER(C.c_int)]),
    "frost_search_enable_timing": (C.c_int, [_vp, C.c_int]),
    "frost_search_get_timing": (C.c_int, [_vp, C.POINTER(_abi.SearchTimingC)]),
    "frost_server_create": (C.c_int, [C.c_int, _sz, C.c_uint32, C.POINTER(_vp)]),
    "frost_server_destroy": (C.c_int, [_vp]),
    "frost_server_add_beam": (C.c_int, [_vp, C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC),
                                        C.c_float, C.POINTER(_abi.DedispPlanConfigC),
                                        C.POINTER(_abi.BoxcarConfigC), C.POINTER(C.c_uint32)]),
    "frost_server_remove_beam": (C.c_int, [_vp, C.c_uint32]),
    "frost_server_submit": (C.c_int, [_vp, C.c_uint32, _vp, _sz, _sz, C.c_int, C.POINTER(_u64)]),
    "frost_server_wait": (C.c_int, [_vp, _u64, C.POINTER(_abi.CandidateC), _sz, C.POINTER(_sz),
                                    C.POINTER(C.c_double)]),
    "frost_server_drain": (C.c_int, [_vp, C.c_uint32, C.POINTER(_abi.CandidateC), _sz,
                                     C.POINTER(_sz)]),
    "frost_server_get_stats": (C.c_int, [_vp, C.POINTER(_abi.ServerStatsC)]),
    "frost_server_reset_stats": (C.c_int, [_vp]),
    "frost_server_set_postprocess": (C.c_int, [_vp, C.c_uint32, C.POINTER(_abi.PostprocessConfigC)]),
    "frost_server_set_residency": (C.c_int, [_vp, C.c_uint32, C.c_int]),
    "frost_server_set_staging": (C.c_int, [_vp, C.c_uint32, C.c_uint32]),
    "frost_server_wait_giants": (C.c_int, [_vp, _u64, _vp, _sz, C.POINTER(_sz), C.POINTER(C.c_double)]),
    "frost_server_drain_giants": (C.c_int, [_vp, C.c_uint32, _vp, _sz, C.POINTER(_sz)]),
    "frost_cand_writer_open": (C.c_int, [C.c_char_p, C.c_double, C.c_int, C.POINTER(_vp)]),
    "frost_cand_writer_write": (C.c_int, [_vp, _vp, _sz, _u64]),
    "frost_cand_writer_close": (C.c_int, [_vp]),
    "frost_cand_filename": (C.c_int, [C.c_int64, _u64, C.c_char_p, _sz]),
    "frost_prefetch_create": (C.c_int, [_sz, _sz, C.c_int, C.c_int, _abi.READ_FN, _vp, C.POINTER(_vp)]),
    "frost_prefetch_create_file": (C.c_int, [C.c_char_p, _u64, _sz, _sz, C.c_int, C.c_int, C.POINTER(_vp)]),
    "frost_prefetch_create_memory": (C.c_int, [_vp, _sz, _sz, _sz, C.c_int, C.c_int, C.POINTER(_vp)]),
    "frost_prefetch_next": (C.c_int, [_vp, _vp, C.POINTER(_vp), C.POINTER(_sz)]),
    "frost_sigproc_read_header": (C.c_int, [C.c_char_p, C.POINTER(_abi.SigprocHeaderC)]),
    "frost_sigproc_layout": (C.c_int, [C.POINTER(_abi.SigprocHeaderC), _u64, C.POINTER(_abi.BlockLayoutC)]),
    "frost_prefetch_create_sigproc": (C.c_int, [C.c_char_p, _sz, C.c_int, C.c_int,
                                                C.POINTER(_abi.SigprocHeaderC), C.POINTER(_vp)]),
    "frost_prefetch_get_stats": (C.c_int, [_vp, C.POINTER(_abi.PrefetchStatsC)]),
    "frost_estimate_memory": (C.c_int, [C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC), C.c_float,
                                        C.POINTER(_abi.DedispPlanConfigC), C.POINTER(_abi.BoxcarConfigC),
                                        C.POINTER(_abi.PostprocessConfigC), C.POINTER(_abi.MemoryEstimateC)]),
    "frost_check_memory": (C.c_int, [C.POINTER(_abi.RfiConfigC), C.POINTER(_abi.BlockLayoutC), C.c_float,
                                     C.POINTER(_abi.DedispPlanConfigC), C.POINTER(_abi.BoxcarConfigC),
                                     C.POINTER(_abi.PostprocessConfigC), C.c_int, C.c_uint64, C.c_uint64, C.c_int,
                                     C.POINTER(_abi.MemoryCheckC)]),
    "frost_prefetch_destroy": (C.c_int, [_vp]),
    "frost_postprocess_create": (C.c_int, [C.POINTER(_abi.PostprocessConfigC), C.POINTER(_abi.PostprocessLayoutC),
                                           C.c_int, C.POINTER(_vp)]),
    "frost_postprocess_destroy": (C.c_int, [_vp]),
    "frost_postprocess_execute": (C.c_int, [_vp, _vp, _sz, C.c_int, _u64, _u64, C.c_int, _u64,
                                            C.POINTER(_abi.PostprocessResultC)]),
    "frost_postprocess_execute_search": (C.c_int, [_vp, _vp, _u64, _u64, C.c_int, _u64,
                                                   C.POINTER(_abi.PostprocessResultC)]),
    "frost_postprocess_results": (C.c_int, [_vp, _vp, _sz, C.POINTER(_sz)]),
    "frost_postprocess_memory_usage": (C.c_int, [_vp, C.POINTER(_u64)]),
    "frost_postprocess_estimate_memory": (C.c_int, [C.POINTER(_abi.PostprocessConfigC), C.POINTER(_u64)]),
    "frost_cluster_labels": (C.c_int, [_vp, _sz, C.POINTER(_abi.ClusterTolerancesC), C.c_int, _vp, C.c_int]),
    "frost_merge_candidates": (C.c_int, [_vp, _vp, _sz, _vp, C.POINTER(_sz), C.c_int]),
    "frost_subband_dedup": (C.c_int, [_vp, _sz, C.POINTER(_abi.ClusterTolerancesC), C.c_float, C.c_int, _vp,
                                      C.POINTER(_sz), C.c_int]),
    "frost_are_coincident": (C.c_int, [C.POINTER(_abi.GiantC), C.POINTER(_abi.GiantC),
                                       C.POINTER(_abi.ClusterTolerancesC), C.c_int]),
    "frost_subband_time_shift_samples": (C.c_double, [C.c_float, C.c_float, C.c_float, C.c_float]),
    "frost_subband_dm_step": (C.c_double, [C.c_float, C.c_float, C.c_float]),
}


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"frost_b200: {LIB_PATH} is not built; run "
                          "`python -c 'import __graft_entry__ as g; g.build()'` or "
                          "`make -C frost_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> int:
    if rc == _abi.OK:
        return rc
    msg = lib().frost_last_error().decode(errors="replace")
    if rc == _abi.ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise FrostError(rc, msg)
