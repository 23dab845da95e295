"""Known-answer cases of the candidate post-processing, restated from the
reference's own tests (tests/cpp/api/clustering_test.cpp,
clustering_boundary_test.cpp, merge_test.cpp, candidate_test.cpp,
subband_dedup_test.cpp, postprocess_test.cpp). Each case takes an `api`
with the calls of ApiLike below, so the same assertions pin the CPU oracle,
the compiled reference and the GPU implementation.
"""

from __future__ import annotations

import math

import numpy as np

from frost_b200.postprocess import ClusterTolerances, SearchConfig, make_giants
from frost_b200.search import CANDIDATE_DTYPE

KMAX = (1 << 64) - 1


class ApiLike:
    """are_coincident(a, b, tol, physical) -> bool
    cluster_labels(giants, tol, mode) -> uint64 labels
    merge(giants, labels) -> giants
    subband_dedup(giants, tol, tsamp, mode) -> giants (raises on bad tsamp)
    time_shift(dm, f_wide, f_narrow, tsamp), dm_step(f_low, f_high, tsamp)
    plan(cfg, layout) -> object with execute(raw, samples_read, duration,
        final, frontier) -> (giants, pending); errors raise PlanFailure-like
        exceptions carrying .kind in {"invalid_argument", "runtime_error"}."""


def giant(snr, samp, filter_idx, dm_idx, **kw):
    g = make_giants(1)[0]
    g["snr"], g["samp_idx"], g["filter_idx"], g["dm_idx"] = snr, samp, filter_idx, dm_idx
    for k, v in kw.items():
        g[k] = v
    return g


def stack(*gs):
    out = make_giants(len(gs))
    for i, g in enumerate(gs):
        out[i] = g
    return out


# ---- clustering_test.cpp ------------------------------------------------------------

def kat_direct_coincidence(api):
    g = stack(giant(5, 1000, 0, 10), giant(8, 1002, 0, 11), giant(6, 5000, 0, 10))
    lab = api.cluster_labels(g, ClusterTolerances(5, 1, 2), 0)
    assert lab[0] == lab[1] and lab[0] != lab[2]


def kat_transitive_chain(api):
    g = stack(giant(5, 1000, 0, 10), giant(6, 1004, 0, 11), giant(7, 1008, 0, 12))
    lab = api.cluster_labels(g, ClusterTolerances(4, 1, 1), 0)
    assert lab[0] == lab[1] == lab[2]


def kat_all_separate(api):
    g = stack(giant(5, 0, 0, 0), giant(5, 10000, 0, 0), giant(5, 20000, 0, 0))
    lab = api.cluster_labels(g, ClusterTolerances(2, 1, 1), 0)
    assert len(set(lab.tolist())) == 3


def kat_extents_apart(api):
    g = stack(giant(8, 1000, 0, 10, chan_begin=0, chan_end=15), giant(7, 1001, 0, 10, chan_begin=0, chan_end=3))
    lab = api.cluster_labels(g, ClusterTolerances(5, 1, 2), 0)
    assert lab[0] != lab[1]


def kat_empty_labels(api):
    assert api.cluster_labels(make_giants(0), ClusterTolerances(1, 1, 1), 0).size == 0


def uwl_giant(snr, samp, dm_idx):
    """704-4032 MHz at 512 us on 338 trials over DM 0-250."""
    return giant(snr, samp, 5, dm_idx, filter_width=32, dm=np.float32(np.float32(dm_idx) * np.float32(250.0) /
                                                                       np.float32(337.0)),
                 f_low=704.0, f_high=4032.0, chan_begin=0, chan_end=6655)


def kat_long_chain_vs_strong(api):
    g = [uwl_giant(6.5, 5000 + (d % 5), d) for d in range(150)] + [uwl_giant(30.0, 5000, 300)]
    g = stack(*g)
    lab = api.cluster_labels(g, ClusterTolerances(3, 3, 200, 3.0, 512.0e-6), 0)
    assert np.all(lab[1:150] == lab[0]) and lab[150] != lab[0]
    by_trials = api.cluster_labels(g, ClusterTolerances(3, 3, 200), 0)
    assert by_trials[150] == by_trials[0]


def kat_physical_tolerance(api):
    tol = ClusterTolerances(3, 3, 200, 3.0, 512.0e-6)
    base = uwl_giant(10.0, 5000, 100)
    assert api.are_coincident(base, uwl_giant(9.0, 5000, 101), tol, True)
    assert api.are_coincident(base, uwl_giant(9.0, 5000, 106), tol, True)
    assert not api.are_coincident(base, uwl_giant(9.0, 5000, 130), tol, True)
    a, b = uwl_giant(10.0, 5000, 100), uwl_giant(9.0, 5000, 101)
    a["filter_width"] = b["filter_width"] = 1
    a["filter_idx"] = b["filter_idx"] = 0
    assert api.are_coincident(a, b, tol, True)


def lcg_giants():
    state = [12345]

    def nxt(mod):
        state[0] = (state[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return (state[0] >> 8) % mod

    out = []
    for _ in range(1500):
        g = uwl_giant(np.float32(6.0) + np.float32(nxt(400)) / np.float32(10.0), nxt(20000), nxt(338))
        g["filter_idx"] = nxt(6)
        g["filter_width"] = 1 << int(g["filter_idx"])
        g["chan_end"] = 3327 if nxt(3) == 0 else 6655
        out.append(g)
    return stack(*out)


def pairwise_labels(api, g, tol):
    n = g.size
    parent = list(range(n))

    def root(x):
        while parent[x] != x:
            x = parent[x]
        return x

    for i in range(n):
        for j in range(i + 1, n):
            if api.are_coincident(g[i], g[j], tol, True):
                a, b = root(i), root(j)
                if a != b:
                    parent[max(a, b)] = min(a, b)
    return np.array([root(i) for i in range(n)], np.uint64)


def kat_sweep_equals_pairwise(api, pairwise):
    """`pairwise(g, tol)` gives the O(N^2) labels (computed by the caller
    with a trusted are_coincident)."""
    g = lcg_giants()
    for tol in (ClusterTolerances(3, 3, 200), ClusterTolerances(3, 3, 10),
                ClusterTolerances(3, 3, 200, 8.0, 512.0e-6)):
        assert np.array_equal(api.cluster_labels(g, tol, 0), pairwise(g, tol))


def kat_seeded_bounded(api):
    g = stack(uwl_giant(8.0, 5000, 100), uwl_giant(20.0, 5000, 103), uwl_giant(7.0, 5000, 106),
              uwl_giant(6.5, 5000, 109))
    g["filter_idx"] = 0
    g["filter_width"] = 1
    tol = ClusterTolerances(3, 3, 200, 10.0, 512.0e-6)
    none = api.cluster_labels(g, tol, 0)
    assert none[0] != none[1]
    tol.dm_smear = 30.0
    still = api.cluster_labels(g, tol, 0)
    assert still[0] != still[1]
    tol.dm_smear = 40.0
    chain = api.cluster_labels(g, tol, 0)
    assert chain[0] == chain[3]
    seeded = api.cluster_labels(g, tol, 1)
    assert seeded.tolist() == [1, 1, 1, 3]


# ---- clustering_boundary_test.cpp ---------------------------------------------------

def boundary_giants():
    out = []
    for width in (1, 2, 3, KMAX // 2 + 1, KMAX):
        for sample in (0, 1, 63, KMAX // 2, KMAX - 1, KMAX):
            g = make_giants(1)[0]
            g["samp_idx"] = sample
            g["filter_width"] = width
            g["snr"] = float(len(out) % 7 + 1)
            out.append(g)
    return stack(*out)


def math_coincident(a, b, time_tol):
    """Without the product: ceil(dt / width) <= time_tol."""
    w = max(int(a["filter_width"]), int(b["filter_width"]))
    dt = abs(int(a["samp_idx"]) - int(b["samp_idx"]))
    return -(-dt // w) <= time_tol


def math_labels(g, time_tol, mode):
    n = g.size
    labels = list(range(n))
    if mode == 0:
        def root(x):
            while labels[x] != x:
                x = labels[x]
            return x
        for i in range(n):
            for j in range(i + 1, n):
                if math_coincident(g[i], g[j], time_tol):
                    a, b = root(i), root(j)
                    labels[max(a, b)] = min(a, b)
        return [root(i) for i in range(n)]
    order = sorted(range(n), key=lambda i: -float(g[i]["snr"]))
    assigned = [False] * n
    for seed in order:
        if assigned[seed]:
            continue
        assigned[seed] = True
        for j in range(n):
            if not assigned[j] and math_coincident(g[seed], g[j], time_tol):
                assigned[j] = True
                labels[j] = seed
    return labels


def kat_integer_boundaries(api):
    g = boundary_giants()
    for time_tol in (0, 1, 2, KMAX // 2, KMAX // 2 + 1, KMAX):
        tol = ClusterTolerances(time_tol, 0, 0)
        for i in range(g.size):
            for j in range(g.size):
                assert api.are_coincident(g[i], g[j], tol, True) == math_coincident(g[i], g[j], time_tol)
        for mode in (0, 1):
            assert api.cluster_labels(g, tol, mode).tolist() == math_labels(g, time_tol, mode)


# ---- merge_test.cpp -------------------------------------------------------------------

def kat_merge(api):
    g = make_giants(4)
    g["snr"] = [5, 9, 3, 7]
    m = api.merge(g, np.array([0, 0, 0, 1], np.uint64))
    assert m.size == 2
    assert m[0]["snr"] == 9 and m[0]["members"] == 3
    assert m[1]["snr"] == 7 and m[1]["members"] == 1
    one = make_giants(1)
    one["snr"], one["members"] = 4, 2
    m = api.merge(one, np.array([0], np.uint64))
    assert m.size == 1 and m[0]["snr"] == 4 and m[0]["members"] == 2
    g = make_giants(5)
    g["snr"] = [1, 2, 3, 4, 5]
    m = api.merge(g, np.array([40, 7, 19, 3, 7], np.uint64))
    assert m["snr"].tolist() == [4, 5, 3, 1] and m[1]["members"] == 2


# ---- candidate_test.cpp ------------------------------------------------------------------

def kat_candidate(api):
    a = giant(0, 1000, 3, 10)
    b = a.copy()
    b["samp_idx"] = 1040
    assert api.are_coincident(a, b, ClusterTolerances(5, 1, 2), False)
    c = a.copy()
    c["samp_idx"] = 1048
    assert not api.are_coincident(a, c, ClusterTolerances(5, 1, 2), False)
    a = giant(0, 500, 0, 10)
    far_dm = a.copy()
    far_dm["dm_idx"] = 20
    assert not api.are_coincident(a, far_dm, ClusterTolerances(5, 1, 2), False)
    far_f = a.copy()
    far_f["filter_idx"] = 5
    assert not api.are_coincident(a, far_f, ClusterTolerances(5, 1, 2), False)
    a, b = make_giants(1)[0], make_giants(1)[0]
    a["snr"] = b["snr"] = 10
    a["chan_end"] = b["chan_end"] = 7
    b["plane"] = 1
    assert not api.are_coincident(a, b, ClusterTolerances(3, 3, 200), False)
    b["plane"] = a["plane"]
    assert api.are_coincident(a, b, ClusterTolerances(3, 3, 200), False)


# ---- subband_dedup_test.cpp --------------------------------------------------------------

TS = np.float32(0.001)
KTOL = ClusterTolerances(3, 1, 10)
KDM_ = 100.0


def band_g(snr, samp, dm, flo, fhi, cb, ce):
    return giant(snr, samp, 2, 0, dm=dm, filter_width=4, f_low=flo, f_high=fhi, chan_begin=cb, chan_end=ce)


def full_band(snr, samp, dm=KDM_):
    return band_g(snr, samp, dm, 1000.0, 1256.0, 0, 63)


def nested_band(snr, samp, dm=KDM_):
    return band_g(snr, samp, dm, 1100.0, 1164.0, 16, 31)


def shifted(api, wide_samp, dm, fw, fn):
    return wide_samp - int(round(api.time_shift(dm, fw, fn, TS)))


def kat_dedup(api):
    tr = 0
    shift = api.time_shift(KDM_, 1000.0, 1100.0, TS)
    assert shift > 3 * 4 + 1.0
    wide = full_band(8.0, 5000)
    narrow = nested_band(9.0, shifted(api, 5000, KDM_, 1000.0, 1100.0))
    narrow["members"] = 2
    m = api.subband_dedup(stack(wide, narrow), KTOL, TS, tr)
    assert m.size == 1 and m[0]["chan_begin"] == 0 and m[0]["chan_end"] == 63 and m[0]["samp_idx"] == 5000
    assert m[0]["dm"] == np.float32(KDM_) and m[0]["snr"] == 8 and m[0]["members"] == 3
    # delay missing
    assert api.subband_dedup(stack(full_band(8.0, 5000), nested_band(9.0, 5000)), KTOL, TS, tr).size == 2
    # disjoint ranges
    bottom = band_g(10.0, 5000, KDM_, 1000.0, 1064.0, 0, 15)
    top = band_g(12.0, shifted(api, 5000, KDM_, 1000.0, 1192.0), KDM_, 1192.0, 1256.0, 48, 63)
    assert api.subband_dedup(stack(bottom, top), KTOL, TS, tr).size == 2
    # both quarters through the full band
    low = band_g(9.0, 5000, KDM_, 1000.0, 1064.0, 0, 15)
    high = band_g(10.0, shifted(api, 5000, KDM_, 1000.0, 1192.0), KDM_, 1192.0, 1256.0, 48, 63)
    m = api.subband_dedup(stack(low, full_band(8.0, 5000), high), KTOL, TS, tr)
    assert m.size == 1 and m[0]["chan_end"] == 63 and m[0]["samp_idx"] == 5000 and m[0]["snr"] == 8
    assert m[0]["members"] == 3
    # DM gate
    proto = nested_band(9.0, 5000)
    step = api.dm_step(proto["f_low"], proto["f_high"], TS)
    assert step > 0
    ns = shifted(api, 5000, KDM_, 1000.0, 1100.0)
    inside = nested_band(9.0, ns, np.float32(KDM_ + np.float32(step)))
    side = nested_band(9.0, ns, np.float32(KDM_ + np.float32(2.5 * step)))
    outside = nested_band(9.0, ns, np.float32(KDM_ + np.float32(6.0 * step)))
    assert api.subband_dedup(stack(full_band(8.0, 5000), inside), KTOL, TS, tr).size == 1
    assert api.subband_dedup(stack(full_band(8.0, 5000), side), KTOL, TS, tr).size == 1
    assert api.subband_dedup(stack(full_band(8.0, 5000), outside), KTOL, TS, tr).size == 2
    # filter tolerance
    nf = nested_band(9.0, ns)
    nf["filter_idx"] = 2 + 1 + 1
    assert api.subband_dedup(stack(full_band(8.0, 5000), nf), KTOL, TS, tr).size == 2
    # equal-span tie by S/N across planes
    quiet, loud = full_band(7.0, 5000), full_band(9.0, 5000)
    quiet["plane"] = 1
    loud["members"] = 4
    m = api.subband_dedup(stack(quiet, nested_band(9.0, ns), loud), KTOL, TS, tr)
    assert m.size == 1 and m[0]["snr"] == 9 and m[0]["members"] == 6 and m[0]["chan_end"] == 63
    # equal extents of one plane stay apart
    assert api.subband_dedup(stack(full_band(8.0, 5000), full_band(12.0, 5001)), KTOL, TS, tr).size == 2
    # seeded does not bridge two wide events
    early, late = full_band(8.0, 5000), full_band(9.0, 5020)
    mid = nested_band(9.0, shifted(api, 5010, KDM_, 1000.0, 1100.0))
    assert api.subband_dedup(stack(early, mid), KTOL, TS, tr).size == 1
    assert api.subband_dedup(stack(late, mid), KTOL, TS, tr).size == 1
    assert api.subband_dedup(stack(early, mid, late), KTOL, TS, tr).size == 1
    for order in ((early, mid, late), (mid, late, early)):
        m = api.subband_dedup(stack(*order), KTOL, TS, 1)
        assert m.size == 2 and set(m["chan_end"].tolist()) == {63} and int(m["members"].sum()) == 3
        assert set(m["samp_idx"].tolist()) == {5000, 5020}
        assert int(m[m["samp_idx"] == 5020][0]["members"]) == 2
    m = api.subband_dedup(stack(low, full_band(8.0, 5000), high), KTOL, TS, 1)
    assert m.size == 1 and m[0]["chan_end"] == 63 and m[0]["members"] == 3 and m[0]["n_extents"] == 3
    assert api.subband_dedup(make_giants(0), KTOL, TS, tr).size == 0


UWL_TS = np.float32(512.0e-6)
UWL_TOL = ClusterTolerances(3, 3, 200, 3.0, float(UWL_TS))


def uwl(snr, samp, dm, flo, fhi, cb, ce, width):
    g = band_g(snr, samp, dm, flo, fhi, cb, ce)
    g["filter_width"] = width
    g["filter_idx"] = int(math.log2(width)) if width > 1 else 0
    return g


def kat_dedup_uwl(api):
    wide = uwl(6.5, 7245, 104.5, 704.0, 4032.0, 0, 6655, 32)
    shift = api.time_shift(np.float32(104.5), 704.0, 3776.0, UWL_TS)
    assert shift > 1000.0
    narrow = uwl(18.9, 7245 - int(round(shift)), 200.0, 3776.0, 4032.0, 0, 511, 32)
    assert api.dm_step(3776.0, 4032.0, UWL_TS) > 10.0
    m = api.subband_dedup(stack(wide, narrow), UWL_TOL, UWL_TS, 0)
    assert m.size == 2 and any(r["snr"] == np.float32(18.9) and r["chan_end"] == 511 for r in m)
    strong = uwl(70.0, 7245, 104.5, 704.0, 4032.0, 0, 6655, 32)
    weak = uwl(18.9, narrow["samp_idx"], 200.0, 3776.0, 4032.0, 0, 511, 32)
    one = api.subband_dedup(stack(strong, weak), UWL_TOL, UWL_TS, 0)
    assert one.size == 1 and one[0]["chan_end"] == 6655 and one[0]["snr"] == 70 and one[0]["n_extents"] == 2
    # one pass-1 scatter apart
    wide = uwl(27.9, 5000, 120.06, 704.0, 4032.0, 0, 6655, 8)
    narrow = uwl(26.4, 5000, 119.29, 704.0, 2752.0, 2560, 6655, 8)
    m = api.subband_dedup(stack(narrow, wide), UWL_TOL, UWL_TS, 0)
    assert m.size == 1 and m[0]["chan_end"] == 6655
    unscaled = ClusterTolerances(3, 3, 200, 0.0, float(UWL_TS))
    assert api.subband_dedup(stack(narrow, wide), unscaled, UWL_TS, 0).size == 2
    # strongest member and extent count
    wide = uwl(54.5, 5000, 120.0, 704.0, 4032.0, 0, 6655, 8)
    low = uwl(82.9, 5000, 120.1, 704.0, 1728.0, 4608, 6655, 8)
    for order in ((wide, low), (low, wide)):
        m = api.subband_dedup(stack(*order), UWL_TOL, UWL_TS, 0)
        assert m.size == 1
        r = m[0]
        assert r["chan_end"] == 6655 and r["snr"] == np.float32(54.5)
        assert max(r["snr_best"], r["snr"]) == np.float32(82.9)
        assert r["best_chan_begin"] == 4608 and r["best_chan_end"] == 6655 and r["n_extents"] == 2
        assert r["has_location_best"] == 1 and r["loc_samp_idx"] == low["samp_idx"]
        assert r["loc_dm"] == low["dm"] and r["loc_filter_width"] == 8
        assert r["loc_f_low"] == low["f_low"] and r["loc_f_high"] == low["f_high"]
        twice = api.subband_dedup(m, UWL_TOL, UWL_TS, 0)
        assert twice.size == 1 and twice[0]["loc_dm"] == low["dm"]
    # one node searched as two planes
    a = uwl(12.0, 5000, 50.0, 704.0, 1728.0, 4608, 6655, 8)
    b = a.copy()
    b["plane"] = 1
    b["snr"] = 11.0
    m = api.subband_dedup(stack(a, b), UWL_TOL, UWL_TS, 0)
    assert m.size == 1 and m[0]["snr"] == 12 and m[0]["n_extents"] == 1
    b["plane"] = 0
    assert api.subband_dedup(stack(a, b), UWL_TOL, UWL_TS, 0).size == 2
    b["plane"] = 1
    b["dm"] = a["dm"] + np.float32(5.0)
    assert api.subband_dedup(stack(a, b), UWL_TOL, UWL_TS, 0).size == 2


# ---- postprocess_test.cpp ----------------------------------------------------------------

def peak():
    r = np.zeros(1, CANDIDATE_DTYPE)[0]
    r["peak_sample"], r["begin_sample"], r["end_sample"] = 100, 99, 101
    r["snr"], r["dm"], r["width"] = 10.0, 20.0, 4
    r["chan_begin"], r["chan_end"] = 1, 5
    r["f_low_mhz"], r["f_high_mhz"] = 1400.0, 1404.0
    return r


def rows(*rs):
    out = np.zeros(len(rs), CANDIDATE_DTYPE)
    for i, r in enumerate(rs):
        out[i] = r
    return out


def kat_pp_channel_order(api, layout):
    cfg = SearchConfig(cluster=False)
    for df in (-1.0, 1.0):
        plan = api.plan(cfg, layout(8, 0.001, df))
        r = peak()
        r["end_sample"] = 1000
        out, _ = plan.execute(rows(r), 200, 200, False, 200)
        assert out.size == 1 and out[0]["samp_idx"] == 100 and out[0]["end"] == 199
        assert out[0]["chan_begin"] == (3 if df < 0 else 1) and out[0]["chan_end"] == (6 if df < 0 else 4)
        assert out[0]["snr"] == 10
        assert plan.execute(None, 200, 0, True, 200)[0].size == 0


def kat_pp_retain_and_drain(api, layout):
    cfg = SearchConfig(boxcar_max=16, cand_sep_dm_smear=0.0)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    r = peak()
    first, pend = plan.execute(rows(r), 110, 110, False, 100)
    assert first.size == 0 and pend == 1
    r["snr"], r["width"], r["filter_idx"], r["end_sample"] = 20.0, 8, 1, 111
    last, pend = plan.execute(rows(r), 120, 10, True, 120)
    assert last.size == 1 and last[0]["snr"] == 20 and last[0]["members"] == 2 and pend == 0
    assert plan.execute(None, 120, 0, True, 120)[0].size == 0


def kat_pp_bounded_pending(api, layout, failure):
    cfg = SearchConfig(boxcar_max=16, max_candidates=4, max_pending_candidates=1, cand_sep_dm=0,
                       cand_sep_dm_smear=0.0)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    a, b = peak(), peak()
    b["dm_idx"] = 100
    try:
        plan.execute(rows(a, b), 110, 110, False, 100)
        raise AssertionError("pending capacity not enforced")
    except failure as e:
        assert "Pending candidate capacity exceeded" in str(e)
    bounded = api.plan(cfg, layout(8, 0.001, 1.0))
    bounded.execute(rows(peak()), 110, 110, False, 110)
    bounded.execute(None, 200, 90, True, 200)


def kat_pp_bridge(api, layout):
    cfg = SearchConfig(boxcar_max=16, cand_sep_time=1, cand_sep_dm_smear=0.0, max_pending_candidates=4)
    for read in (120, 140):
        plan = api.plan(cfg, layout(8, 0.001, 1.0))
        strong = peak()
        strong["width"], strong["snr"] = 16, 20
        bridge = strong.copy()
        bridge["snr"], bridge["peak_sample"], bridge["begin_sample"], bridge["end_sample"] = 10, 115, 114, 116
        out, pend = plan.execute(rows(strong, bridge), read, read, False, read)
        assert out.size == 0 and pend == 2
        later = bridge.copy()
        later["snr"], later["peak_sample"], later["begin_sample"], later["end_sample"] = 9, 130, 129, 131
        out, pend = plan.execute(rows(later), 200, 200 - read, True, 200)
        assert out.size == 1 and out[0]["samp_idx"] == 100 and out[0]["snr"] == 20 and out[0]["members"] == 3
        assert out[0]["begin"] == 99 and out[0]["end"] == 101 and pend == 0


def kat_pp_wing_members(api, layout):
    cfg = SearchConfig(boxcar_max=16, cand_sep_time=1, cand_sep_dm_smear=3.0, max_pending_candidates=4)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    strong = peak()
    strong["f_low_mhz"], strong["f_high_mhz"], strong["dm"], strong["dm_idx"], strong["snr"] = 1000, 1500, 30, 10, 50
    bridge = strong.copy()
    bridge["dm"], bridge["dm_idx"], bridge["snr"] = 20, 0, 10
    bridge["peak_sample"], bridge["begin_sample"], bridge["end_sample"] = 104, 103, 105
    old = strong.copy()
    old["peak_sample"] = old["begin_sample"] = old["end_sample"] = 0
    old["snr"], old["dm_idx"], old["dm"] = 8, 100, 100
    out, pend = plan.execute(rows(strong, bridge, old), 136, 136, False, 136)
    assert out.size == 1 and out[0]["samp_idx"] == 0 and pend == 2
    later = bridge.copy()
    later["snr"], later["peak_sample"], later["begin_sample"], later["end_sample"] = 9, 108, 107, 109
    out, pend = plan.execute(rows(later), 200, 64, True, 200)
    assert out.size == 1 and out[0]["samp_idx"] == 100 and out[0]["dm"] == 30 and out[0]["snr"] == 50
    assert out[0]["members"] == 3 and pend == 0


def kat_pp_pending_counts_members(api, layout, failure):
    cfg = SearchConfig(boxcar_max=16, cand_sep_dm_smear=0.0, max_pending_candidates=1)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    a = peak()
    b = a.copy()
    b["peak_sample"], b["end_sample"] = 101, 102
    try:
        plan.execute(rows(a, b), 110, 110, False, 100)
        raise AssertionError("pending members not counted")
    except failure as e:
        assert "Pending candidate capacity exceeded" in str(e)


def kat_pp_geometry(api, layout, invalid):
    cfg = SearchConfig()
    for bad in (0.0, -1.0, math.inf, math.nan):
        try:
            api.plan(cfg, layout(8, bad, 1.0))
            raise AssertionError("bad tsamp accepted")
        except invalid:
            pass
    for bad in (0.0, math.inf, math.nan):
        try:
            api.plan(cfg, layout(8, 0.001, bad))
            raise AssertionError("bad frequency step accepted")
        except invalid:
            pass


def kat_pp_malformed(api, layout, invalid):
    cfg = SearchConfig(boxcar_max=16, cluster=False)
    for field, value in (("beam_idx", 1), ("width", 0), ("width", 17), ("begin_sample", 101), ("end_sample", 99)):
        plan = api.plan(cfg, layout(8, 0.001, 1.0))
        bad = peak()
        bad[field] = value
        try:
            plan.execute(rows(bad), 200, 200, False, 200)
            raise AssertionError(f"{field}={value} accepted")
        except invalid:
            pass
        out, _ = plan.execute(rows(peak()), 200, 200, False, 200)
        assert out.size == 1 and out[0]["samp_idx"] == 100


def kat_pp_rate_limiter(api, layout):
    cfg = SearchConfig(cluster=False, max_giant_rate=60.0)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    r = [peak() for _ in range(4)]
    r[1]["peak_sample"] = r[1]["end_sample"] = 110
    r[2]["peak_sample"] = r[2]["end_sample"] = 120
    r[3]["subband_level"], r[3]["chan_end"] = 1, 3
    out, _ = plan.execute(rows(*r), 1000, 1000, True, 1000)
    assert out.size == 3 and out[0]["samp_idx"] == 100 and out[1]["samp_idx"] == 110
    assert out[2]["plane"] != out[0]["plane"]


def kat_pp_frontier(api, layout):
    cfg = SearchConfig(boxcar_max=16, cand_sep_time=1, cand_sep_dm_smear=0.0)
    plan = api.plan(cfg, layout(8, 0.001, 1.0))
    held, pend = plan.execute(rows(peak()), 100_000, 100_000, False, 90)
    assert held.size == 0 and pend == 1
    held, pend = plan.execute(None, 100_000, 0, False, 101 + 32)
    assert held.size == 0 and pend == 1
    rel, pend = plan.execute(None, 100_000, 0, False, 101 + 33)
    assert rel.size == 1 and rel[0]["samp_idx"] == 100 and pend == 0


CLUSTER_KATS = [kat_direct_coincidence, kat_transitive_chain, kat_all_separate, kat_extents_apart, kat_empty_labels,
                kat_long_chain_vs_strong, kat_physical_tolerance, kat_seeded_bounded, kat_merge, kat_candidate,
                kat_dedup, kat_dedup_uwl]
