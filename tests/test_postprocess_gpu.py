"""GPU parity of the candidate post-processing: the reference tests' known
answers, and bit-identical giants against the CPU oracle
(oracle/postprocess_oracle.c, itself pinned to the reference's sources) on
seeded streams, standalone plans, a large clustered gulp, and the search
engine's own device results."""

import numpy as np
import pytest

from frost_b200._lib import FrostError
from frost_b200.config import BoxcarConfig
from frost_b200.postprocess import (CandidatePostprocessLayout, CandidatePostprocessPlan, ClusterLabelPlan,
                                    ClusterTolerances, MergeCandidatesPlan, SearchConfig, SubbandDedupPlan,
                                    are_coincident, subband_dm_step, subband_time_shift_samples)
from oracle import postprocess as op
from tests import postprocess_kats as K
from tests.postprocess_cases import make_stream, random_giants, same_giants

pytestmark = pytest.mark.gpu


class Failure(Exception):
    pass


class GpuPlan:
    def __init__(self, cfg, layout):
        try:
            self.p = CandidatePostprocessPlan(cfg, layout)
        except ValueError as e:
            raise Failure(str(e))

    def execute(self, raw, sr, dur, final, frontier):
        try:
            r = self.p.execute(raw, sr, dur, final, frontier)
        except (ValueError, FrostError) as e:
            raise Failure(str(e))
        return r.candidates, r.pending_candidates


class GpuApi:
    def are_coincident(self, a, b, tol, physical):
        if physical:
            return are_coincident(a, b, tol)
        return are_coincident(a, b, tol.time_tol, tol.filter_tol, tol.dm_tol)

    def cluster_labels(self, g, tol, mode):
        return ClusterLabelPlan(mode).execute(g, tol)

    def merge(self, g, labels):
        return MergeCandidatesPlan().execute(g, labels)

    def subband_dedup(self, g, tol, tsamp, mode):
        return SubbandDedupPlan(mode).execute(g, tol, tsamp)

    def time_shift(self, *a):
        return subband_time_shift_samples(*a)

    def dm_step(self, *a):
        return subband_dm_step(*a)

    def plan(self, cfg, layout):
        return GpuPlan(cfg, layout)


API = GpuApi()
ORACLE = op.backend("oracle")


@pytest.mark.parametrize("case", K.CLUSTER_KATS, ids=lambda f: f.__name__)
def test_cluster_kats(case):
    case(API)


def test_integer_boundaries():
    K.kat_integer_boundaries(API)


def test_sweep_equals_pairwise():
    K.kat_sweep_equals_pairwise(API, lambda g, tol: ORACLE.cluster_labels(g, tol, 0))


def _layout(n, ts, df):
    return CandidatePostprocessLayout(n, ts, df)


@pytest.mark.parametrize("case", [K.kat_pp_channel_order, K.kat_pp_retain_and_drain, K.kat_pp_bridge,
                                  K.kat_pp_wing_members, K.kat_pp_rate_limiter, K.kat_pp_frontier],
                         ids=lambda f: f.__name__)
def test_plan_kats(case):
    case(API, _layout)


def test_plan_failures_keep_state():
    K.kat_pp_bounded_pending(API, _layout, Failure)
    K.kat_pp_pending_counts_members(API, _layout, Failure)
    K.kat_pp_geometry(API, _layout, Failure)
    K.kat_pp_malformed(API, _layout, Failure)


def test_memory_bounded_and_reused():
    cfg = SearchConfig(boxcar_max=16, max_candidates=4, max_pending_candidates=1, cand_sep_dm=0,
                       cand_sep_dm_smear=0.0)
    p = CandidatePostprocessPlan(cfg, _layout(8, 0.001, 1.0))
    reserved = p.memory_usage()
    assert reserved <= CandidatePostprocessPlan.estimate_memory(cfg)
    p.execute(K.rows(K.peak()), 110, 110, False, 110)
    p.execute(None, 200, 90, True, 200)
    assert p.memory_usage() == reserved


TOLS = [ClusterTolerances(3, 3, 200), ClusterTolerances(3, 3, 10), ClusterTolerances(3, 3, 200, 8.0, 1e-3, 6.0),
        ClusterTolerances(1, 1, 50, 3.0, 1e-3, 0.0)]


@pytest.mark.parametrize("seed", range(3))
def test_standalone_plans_match_oracle(seed):
    g = random_giants(seed, 700)
    for tol in TOLS:
        for mode in (0, 1):
            assert np.array_equal(ClusterLabelPlan(mode).execute(g, tol), ORACLE.cluster_labels(g, tol, mode))
            assert same_giants(SubbandDedupPlan(mode).execute(g, tol, 1e-3),
                               ORACLE.subband_dedup(g, tol, 1e-3, mode))
        lab = ORACLE.cluster_labels(g, tol, 0)
        assert same_giants(MergeCandidatesPlan().execute(g, lab), ORACLE.merge(g, lab))
    arbitrary = np.random.default_rng(seed).integers(0, 1 << 40, g.size).astype(np.uint64) * 3
    arbitrary[::7] = arbitrary[0]
    assert same_giants(MergeCandidatesPlan().execute(g, arbitrary), ORACLE.merge(g, arbitrary))


CONFIGS = [dict(), dict(cand_sep_dm_smear=0.0), dict(cluster=False), dict(subband_dedup=1),
           dict(max_giant_rate=2000.0), dict(cand_sep_time=1), dict(cand_sep_dm=5, cand_sep_filter=1)]


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("cfgkw", CONFIGS, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()) or "default")
def test_streams_match_oracle(seed, cfgkw):
    cfg = SearchConfig(boxcar_max=64, max_candidates=100000, **cfgkw)
    lay = CandidatePostprocessLayout(64, 1e-3, -4.0 if seed % 2 else 4.0)
    gpu, orc = CandidatePostprocessPlan(cfg, lay), ORACLE.plan(cfg, lay)
    for raw, sr, dur, fin, fr in make_stream(seed):
        r = gpu.execute(raw, sr, dur, fin, fr)
        b, pb = orc.execute(raw, sr, dur, fin, fr)
        assert r.pending_candidates == pb
        assert same_giants(r.candidates, b)


def test_large_dense_gulps_match_oracle():
    """Tens of thousands of rows in dense pulse clusters over many DM
    trials, widths and planes, carried across gulps."""
    cfg = SearchConfig(boxcar_max=256, max_candidates=400000)
    lay = CandidatePostprocessLayout(64, 1e-3, 4.0)
    stream = make_stream(11, ngulps=3, gulp=16384, n_pulses=20, n_noise=3000, max_width_idx=8, n_dm=1200,
                         max_spread=80, width_span=3, snr_range=(20.0, 200.0))
    gpu, orc = CandidatePostprocessPlan(cfg, lay), ORACLE.plan(cfg, lay)
    total = 0
    for raw, sr, dur, fin, fr in stream:
        total += raw.size
        r = gpu.execute(raw, sr, dur, fin, fr)
        b, pb = orc.execute(raw, sr, dur, fin, fr)
        assert r.pending_candidates == pb
        assert same_giants(r.candidates, b)
    assert total > 20000


def test_engine_results_in_place_match_host_and_oracle():
    from frost_b200.search import FDMTBoxcar
    from tests.search_cases import make_stream as wf_stream
    from tests.search_cases import plan_config
    pc = plan_config(depth=2)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    pulses = ((1500, 20.0, 3.0, 1.2), (5000, 45.0, 8.0, 0.5), (9300, 5.0, 1.0, 2.5), (8190, 33.0, 4.0, 0.8))
    stream = wf_stream(pc, 3, seed=9, pulses=pulses)
    eng = FDMTBoxcar(pc, bc)
    cfg = SearchConfig(boxcar_max=16, detect_thresh=6.0, max_candidates=bc.max_candidates)
    lay = CandidatePostprocessLayout(pc.nchans, pc.dt, pc.df)
    dev, host, orc = CandidatePostprocessPlan(cfg, lay), CandidatePostprocessPlan(cfg, lay), ORACLE.plan(cfg, lay)
    gulp = pc.block_nsamps
    n_out = 0
    for g in range(3):
        res = eng.execute(np.ascontiguousarray(stream[:, g * gulp:(g + 1) * gulp]))
        sr, fr = (g + 1) * gulp, eng.get_candidate_frontier()
        a = dev.execute(eng, sr, gulp, False, fr)
        b = host.execute(res.candidates, sr, gulp, False, fr)
        c, pc_ = orc.execute(res.candidates, sr, gulp, False, fr)
        assert same_giants(a.candidates, b.candidates) and same_giants(a.candidates, c)
        assert a.pending_candidates == b.pending_candidates == pc_
        n_out += a.candidates.size
    res = eng.drain()
    a = dev.execute(eng, 3 * gulp, 0, True, 3 * gulp)
    c, _ = orc.execute(res.candidates, 3 * gulp, 0, True, 3 * gulp)
    assert same_giants(a.candidates, c)
    n_out += a.candidates.size
    assert n_out >= 4
