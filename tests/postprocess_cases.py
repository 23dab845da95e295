"""Seeded candidate streams for the post-processing parity tests.

A stream is a list of gulps (raw rows of CANDIDATE_DTYPE, samples_read,
duration_samples, final, frontier). Rows imitate what a sub-band FDMT search
reports: a few dispersed pulses, each seen on several planes (full band,
halves, quarters and a staggered half) over neighbouring DM trials and
widths, with peaks referenced to the bottom of each plane's band, plus
scattered single noise rows. Tolerances are chosen so that chains, wings,
nested-extent matches and carried clusters all occur.
"""

from __future__ import annotations

from typing import List, Tuple

import numpy as np

from frost_b200.postprocess import GIANT_DTYPE, make_giants
from frost_b200.search import CANDIDATE_DTYPE

KDM = 4.148808e3

# plane -> (subband_level, subband_idx, chan_begin, chan_end) over 64 channels
PLANES = [(0, 0, 0, 64), (1, 0, 0, 32), (1, 1, 32, 64), (1, 2, 16, 48), (2, 0, 0, 16), (2, 3, 48, 64)]


def band(nchans: int, f0: float, df: float, cb: int, ce: int) -> Tuple[float, float]:
    """(f_low, f_high) of channels [cb, ce) in ascending-frequency order."""
    lo, hi = f0 + cb * df, f0 + ce * df
    return (lo, hi)


def make_stream(seed: int, ngulps: int = 3, gulp: int = 4096, nchans: int = 64, f0: float = 1200.0,
                df: float = 4.0, tsamp: float = 1e-3, n_pulses: int = 6, n_noise: int = 80,
                max_width_idx: int = 5, dm_step: float = 0.5, n_dm: int = 400, max_spread: int = 12,
                width_span: int = 1, snr_range: Tuple[float, float] = (7.0, 60.0)) -> List[tuple]:
    rng = np.random.default_rng(seed)
    rows = []
    total = ngulps * gulp
    for _ in range(n_pulses):
        t_inf = float(rng.uniform(200, total - 800))
        dm0 = float(rng.uniform(20, (n_dm - 20) * dm_step))
        wi0 = int(rng.integers(0, max_width_idx + 1))
        snr0 = float(rng.uniform(*snr_range))
        for (lev, idx, cb, ce) in PLANES:
            if rng.random() < 0.2:
                continue
            flo, fhi = band(nchans, f0, df, cb, ce)
            frac = np.sqrt((ce - cb) / nchans)
            d0 = int(round(dm0 / dm_step))
            spread = int(rng.integers(1, max_spread))
            for d in range(max(0, d0 - spread), min(n_dm, d0 + spread + 1)):
                for wi in range(max(0, wi0 - width_span), min(max_width_idx, wi0 + width_span) + 1):
                    if rng.random() < 0.3:
                        continue
                    w = 1 << wi
                    dm = d * dm_step
                    arr = t_inf + KDM * dm0 / flo ** 2 / tsamp
                    jitter = (d - d0) * float(rng.normal(0, 0.6)) + float(rng.normal(0, 1))
                    peak = int(round(arr + jitter))
                    if peak < 0:
                        continue
                    snr = snr0 * frac * float(np.exp(-abs(d - d0) / max(spread, 1))) * float(rng.uniform(0.8, 1.1))
                    if snr < 6.0:
                        continue
                    rows.append((peak, w, wi, d, dm, flo, fhi, cb, ce, lev, idx, snr))
    for _ in range(n_noise):
        lev, idx, cb, ce = PLANES[int(rng.integers(0, len(PLANES)))]
        flo, fhi = band(nchans, f0, df, cb, ce)
        wi = int(rng.integers(0, max_width_idx + 1))
        d = int(rng.integers(0, n_dm))
        rows.append((int(rng.integers(0, total)), 1 << wi, wi, d, d * dm_step, flo, fhi, cb, ce, lev, idx,
                     float(rng.uniform(6.0, 8.0))))
    raw = np.zeros(len(rows), CANDIDATE_DTYPE)
    for k, (peak, w, wi, d, dm, flo, fhi, cb, ce, lev, idx, snr) in enumerate(rows):
        r = raw[k]
        r["peak_sample"] = peak
        r["begin_sample"] = max(0, peak - int(rng.integers(0, w + 1)))
        r["end_sample"] = peak + int(rng.integers(0, w + 1))
        r["snr"] = snr
        r["dm"] = dm
        r["f_low_mhz"] = flo
        r["f_high_mhz"] = fhi
        r["filter_idx"] = wi
        r["width"] = w
        r["dm_idx"] = d
        r["chan_begin"] = cb
        r["chan_end"] = ce
        r["subband_level"] = lev
        r["subband_idx"] = idx
    raw = raw[rng.permutation(raw.size)]
    gulps = []
    for gi in range(ngulps):
        end = (gi + 1) * gulp
        start = gi * gulp
        # A gulp reports the peaks of excursions that closed inside it.
        sel = (raw["end_sample"] >= start) & (raw["end_sample"] < end) if gi + 1 < ngulps else \
            (raw["end_sample"] >= start)
        last = gi + 1 == ngulps
        frontier = end - int(rng.integers(0, 64))
        gulps.append((raw[sel].copy(), end if not last else total + 4 * gulp, gulp, last, frontier))
    return gulps


def random_giants(seed: int, n: int, nchans: int = 64, f0: float = 1200.0, df: float = 4.0,
                  tsamp: float = 1e-3, spread: int = 3000, planes: int = 3) -> np.ndarray:
    """Giants for the standalone plans: clustered in time, DM and width, on a
    few planes and nested extents, with location_best set on some rows."""
    rng = np.random.default_rng(seed)
    g = make_giants(n)
    centres = rng.uniform(0, spread, size=max(1, n // 25))
    for i in range(n):
        lev, idx, cb, ce = PLANES[int(rng.integers(0, len(PLANES)))]
        flo, fhi = band(nchans, f0, df, cb, ce)
        c = centres[int(rng.integers(0, centres.size))]
        wi = int(rng.integers(0, 6))
        d = int(rng.integers(0, 60)) + int(c) % 200
        dm = d * 0.5
        arr = c + KDM * dm / flo ** 2 / tsamp * 0.001
        g[i]["samp_idx"] = int(max(0, round(arr + rng.normal(0, 6))))
        g[i]["filter_idx"] = wi
        g[i]["filter_width"] = (1 << wi) if rng.random() < 0.9 else 0
        g[i]["dm_idx"] = d
        g[i]["dm"] = dm
        g[i]["f_low"] = flo
        g[i]["f_high"] = fhi
        g[i]["chan_begin"] = cb
        g[i]["chan_end"] = ce - 1
        g[i]["plane"] = int(rng.integers(0, planes))
        g[i]["snr"] = float(rng.uniform(6, 40))
        g[i]["members"] = int(rng.integers(1, 4))
        g[i]["begin"] = g[i]["samp_idx"]
        g[i]["end"] = g[i]["samp_idx"] + (1 << wi)
        if rng.random() < 0.2:
            g[i]["snr_best"] = g[i]["snr"] + float(rng.uniform(0, 5))
            g[i]["best_chan_begin"] = cb
            g[i]["best_chan_end"] = ce - 1
        if rng.random() < 0.1:
            g[i]["has_location_best"] = 1
            g[i]["loc_samp_idx"] = g[i]["samp_idx"] + 1
            g[i]["loc_dm"] = dm + 0.25
            g[i]["loc_filter_width"] = 1 << wi
            g[i]["loc_f_low"] = flo
            g[i]["loc_f_high"] = fhi
    return g


def same_giants(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-identical rows (every field)."""
    a = np.ascontiguousarray(a, GIANT_DTYPE)
    b = np.ascontiguousarray(b, GIANT_DTYPE)
    return a.shape == b.shape and a.tobytes() == b.tobytes()
