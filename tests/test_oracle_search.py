"""Pins the FP64 search oracle (oracle/fdmt_oracle.c) to frost's engine
contracts — the only pins available while dmt itself is absent. CPU only."""

import numpy as np
import pytest

from oracle.fdmt import Oracle, bands, widths


def test_plane_geometry_counts_and_staggering():
    """dedisp_test.cpp:30-54: depth 0/1/2 gives 1/4/11 planes, 0/1/4 of
    them staggered, each staggered band strictly inside the band; balanced
    non-power-of-two extents (pipeline_test.cpp:647-): 24 -> 12/6."""
    for depth, total, stag in ((0, 1, 0), (1, 4, 1), (2, 11, 4)):
        bs = bands(16, depth)
        assert len(bs) == total
        assert sum(b.staggered for b in bs) == stag
        for b in bs:
            if b.staggered:
                assert b.a > 0 and b.b < 16
    bs = bands(24, 2)
    assert [(b.a, b.b) for b in bs if b.level == 1 and not b.staggered] == [(0, 12), (12, 24)]
    assert [(b.a, b.b) for b in bs if b.level == 2 and not b.staggered] == [(0, 6), (6, 12), (12, 18), (18, 24)]


def test_width_list():
    """robustness_test.cpp:229-241: ceil(wtsp * w), at least one sample of
    progress, never above max."""
    assert widths(256, 2.0) == [1, 2, 4, 8, 16, 32, 64, 128, 256]
    w = widths(64, 1.3)
    assert w[0] == 1 and all(b > a for a, b in zip(w, w[1:])) and w[-1] <= 64
    assert widths(5, 1.0) == [1, 2, 3, 4, 5]


def small_oracle(**kw):
    args = dict(nchans=32, f_min=796.0, f_max=1052.0, tsamp=1e-3,
                dm_list=np.linspace(0, 60, 25).astype(np.float32), depth=2, max_boxcar=16)
    args.update(kw)
    return Oracle(**args)


def test_unit_noise_in_every_plane_masked_or_not():
    """calibration_test.cpp:159-168: S/N of pure noise has sigma 1 +- 0.15
    for every plane, DM and width, unmasked, alternating and half-band masks,
    without any global rescaling."""
    rng = np.random.default_rng(0xCA11B)
    T = 8192
    o = small_oracle()
    for name, mask in (("unmasked", np.ones(32, np.uint8)),
                       ("alternating", (np.arange(32) % 2).astype(np.uint8)),
                       ("half", (np.arange(32) >= 16).astype(np.uint8))):
        x = rng.standard_normal((32, T)) * mask[:, None]
        for band in o.bands:
            if not mask[band.a:band.b].any():
                continue
            rows = o.dedisperse(x, band)
            for W in (1, 4, 16):
                var = o.variance(band, mask, W)
                for r in (0, rows.shape[0] // 2, rows.shape[0] - 1):
                    begin = band.delays[r] + W - 1
                    s = np.convolve(rows[r], np.ones(W))[: T][begin:] / np.sqrt(var[r])
                    assert abs(s.mean()) < 0.15, (name, band, W)
                    assert abs(s.std() - 1.0) < 0.15, (name, band.a, band.b, W, s.std())


def test_variance_closed_form_and_trapezoid():
    """For a single channel window of L samples and a width-W boxcar the
    squared multiplicities sum to L^2 (W - L + 1) + (L - 1) L (2L - 1) / 3
    (L <= W); the trapezoid costs variance, keeps unit noise."""
    o = small_oracle()
    band = o.bands[0]
    _, lens = o.geometry(band)
    mask = np.ones(32, np.uint8)
    v = o.variance(band, mask, 8)
    expect = sum(L * L * (8 - L + 1) + (L - 1) * L * (2 * L - 1) / 3 if L <= 8 else
                 8 * 8 * (L - 8 + 1) + (8 - 1) * 8 * (2 * 8 - 1) / 3 for L in lens[0])
    assert v[0] == pytest.approx(expect)
    ot = small_oracle(trapezoid=True)
    assert np.all(ot.variance(band, mask, 8) < v)


def test_pulse_peak_at_window_end_and_bottom_of_band_reference():
    """gpu_parity_test.cpp:148: a flat DM-0 pulse of width w starting at s
    peaks at s + w - 1 at width w; pipeline_end_to_end_test.cpp:116-119: a
    dispersed pulse is timed at the bottom of the band."""
    o = small_oracle(thresh=8.0, max_boxcar=8)
    T = 4096
    x = np.random.default_rng(1).standard_normal((32, T)) * 0.05
    x[:, 1000:1008] += 1.0
    cands = o.search(x, T, [np.ones(32, np.uint8)])
    full = [c for c in cands if c["plane"] == (0, 0) and c["dm_idx"] == 0 and c["width"] == 8]
    assert full and full[0]["peak"] == 1007
    # dispersed: arrival at the top edge at t0, expected at the bottom at
    # t0 + delay(f_min, f_max)
    o2 = small_oracle(thresh=8.0, max_boxcar=4, depth=0)
    dm_idx = 20
    dm = float(o2.dm_list[dm_idx])
    t0 = 1500
    y = np.random.default_rng(2).standard_normal((32, T)) * 0.05
    centres = []
    for c in range(32):
        f = o2.edge(c) + 4.0
        d = 4.148808e3 * dm * (1 / f ** 2 - 1 / o2.f_max ** 2) / 1e-3
        y[c, t0 + int(round(d))] += 3.0
        centres.append(d)
    cands = o2.search(y, T, [np.ones(32, np.uint8)])
    best = max(cands, key=lambda c: c["snr"])
    bottom = t0 + 4.148808e3 * dm * (1 / o2.f_min ** 2 - 1 / o2.f_max ** 2) / 1e-3
    assert abs(best["peak"] - bottom) <= 3
    assert abs(best["dm"] - dm) <= 5.0
