"""CPU checks of the candidate post-processing checkers: the C restatement
(oracle/postprocess_oracle.c) against the reference tests' known answers and
against the reference's own lib/search sources compiled into
oracle/_ref/libfrost_ref_search.so, on seeded streams and giants."""

import numpy as np
import pytest

from frost_b200.postprocess import CandidatePostprocessLayout, ClusterTolerances, SearchConfig
from oracle import postprocess as op
from tests import postprocess_kats as K
from tests.postprocess_cases import make_stream, random_giants, same_giants

BACKENDS = ["oracle"] + (["reference"] if op.ref_available() else [])


class CpuApi:
    def __init__(self, which):
        self.be = op.backend(which)

    def are_coincident(self, a, b, tol, physical):
        return self.be.are_coincident(a, b, tol, physical)

    def cluster_labels(self, g, tol, mode):
        return self.be.cluster_labels(g, tol, mode)

    def merge(self, g, labels):
        return self.be.merge(g, labels)

    def subband_dedup(self, g, tol, tsamp, mode):
        return self.be.subband_dedup(g, tol, tsamp, mode)

    def time_shift(self, *a):
        return self.be.time_shift(*a)

    def dm_step(self, *a):
        return self.be.dm_step(*a)

    def plan(self, cfg, layout):
        return self.be.plan(cfg, layout)


class Invalid(op.PlanError):
    pass


def _invalid_types():
    return (op.PlanError,)


@pytest.fixture(params=BACKENDS)
def api(request):
    return CpuApi(request.param)


@pytest.mark.parametrize("case", K.CLUSTER_KATS, ids=lambda f: f.__name__)
def test_cluster_kats(api, case):
    case(api)


def test_integer_boundaries(api):
    K.kat_integer_boundaries(api)


def test_sweep_equals_pairwise(api):
    K.kat_sweep_equals_pairwise(api, lambda g, tol: K.pairwise_labels(api, g, tol))


def _layout(n, ts, df):
    return CandidatePostprocessLayout(n, ts, df)


@pytest.mark.parametrize("case", [K.kat_pp_channel_order, K.kat_pp_retain_and_drain, K.kat_pp_bridge,
                                  K.kat_pp_wing_members, K.kat_pp_rate_limiter, K.kat_pp_frontier],
                         ids=lambda f: f.__name__)
def test_plan_kats(api, case):
    case(api, _layout)


def test_plan_failures(api):
    K.kat_pp_bounded_pending(api, _layout, op.PlanError)
    K.kat_pp_pending_counts_members(api, _layout, op.PlanError)
    K.kat_pp_geometry(api, _layout, op.PlanError)
    K.kat_pp_malformed(api, _layout, op.PlanError)


TOLS = [ClusterTolerances(3, 3, 200), ClusterTolerances(3, 3, 10), ClusterTolerances(3, 3, 200, 8.0, 1e-3, 6.0),
        ClusterTolerances(1, 1, 50, 3.0, 1e-3, 0.0)]


@pytest.mark.skipif(not op.ref_available(), reason="reference search sources not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", range(3))
def test_standalone_matches_reference(seed):
    O, R = op.backend("oracle"), op.backend("reference")
    g = random_giants(seed, 500)
    for tol in TOLS:
        for mode in (0, 1):
            assert np.array_equal(O.cluster_labels(g, tol, mode), R.cluster_labels(g, tol, mode))
            assert same_giants(O.subband_dedup(g, tol, 1e-3, mode), R.subband_dedup(g, tol, 1e-3, mode))
        lab = O.cluster_labels(g, tol, 0)
        assert same_giants(O.merge(g, lab), R.merge(g, lab))


CONFIGS = [dict(), dict(cand_sep_dm_smear=0.0), dict(cluster=False), dict(subband_dedup=1),
           dict(max_giant_rate=2000.0), dict(cand_sep_time=1), dict(cand_sep_dm=5, cand_sep_filter=1)]


@pytest.mark.skipif(not op.ref_available(), reason="reference search sources not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("cfgkw", CONFIGS, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()) or "default")
def test_streams_match_reference(seed, cfgkw):
    O, R = op.backend("oracle"), op.backend("reference")
    cfg = SearchConfig(boxcar_max=64, max_candidates=100000, **cfgkw)
    lay = CandidatePostprocessLayout(64, 1e-3, -4.0 if seed % 2 else 4.0)
    po, pr = O.plan(cfg, lay), R.plan(cfg, lay)
    for raw, sr, dur, fin, fr in make_stream(seed):
        a, pa = po.execute(raw, sr, dur, fin, fr)
        b, pb = pr.execute(raw, sr, dur, fin, fr)
        assert pa == pb
        assert same_giants(a, b)


@pytest.mark.skipif(not op.ref_available(), reason="reference search sources not built (make -C oracle ref)")
def test_reference_memory_bound():
    """memory_usage stays within estimate_memory and does not grow
    (postprocess_test.cpp:71-95), on the reference's own plan."""
    R = op.backend("reference")
    cfg = SearchConfig(boxcar_max=16, max_candidates=4, max_pending_candidates=1, cand_sep_dm=0,
                       cand_sep_dm_smear=0.0)
    p = R.plan(cfg, CandidatePostprocessLayout(8, 0.001, 1.0))
    before = p.memory_usage()
    p.execute(K.rows(K.peak()), 110, 110, False, 110)
    assert p.memory_usage() == before
