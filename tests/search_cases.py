"""Seeded streams for the search parity tests: calibrated unit-noise
waterfalls ([nchans][T], low frequency first) with dispersed Gaussian pulses,
plus the helpers that run the GPU engine over a stream gulp by gulp and
compare its candidates with the FP64 oracle's."""

from __future__ import annotations

import numpy as np

from frost_b200.config import BoxcarConfig, DedispPlanConfig, PeakMode, Storage
from frost_b200.dedisp import band_edges, generate_dm_list

KDM = 4.148808e3


def plan_config(nchans=64, gulp=4096, depth=2, dm_max=60.0, tsamp=1e-3, f_top=1052.0, foff=-4.0):
    return DedispPlanConfig(nchans=nchans, dt=tsamp, f0=f_top + foff / 2, df=foff, dm_min=0.0,
                            dm_max=dm_max, dm_pulse_width=1000.0, dm_tol=1.25,
                            block_nsamps=gulp, subband_depth=depth)


def make_stream(pc: DedispPlanConfig, ngulps: int, seed: int, pulses=(), noise=1.0):
    """pulses: (t_bottom, dm, width_fwhm, amplitude per channel-sample)."""
    f_min, f_max = band_edges(pc)
    C, T = pc.nchans, pc.block_nsamps * ngulps
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal((C, T)) * noise).astype(np.float32)
    bw = (f_max - f_min) / C
    t = np.arange(T)
    for t_bot, dm, width, amp in pulses:
        sig = max(width / 2.355, 0.3)
        for c in range(C):
            f = f_min + (c + 0.5) * bw
            centre = t_bot - KDM * dm * (1 / f_min ** 2 - 1 / f ** 2) / pc.dt
            lo, hi = int(centre - 5 * sig) - 1, int(centre + 5 * sig) + 2
            lo, hi = max(lo, 0), min(hi, T)
            if lo >= hi:
                continue
            prof = np.exp(-0.5 * ((t[lo:hi] - centre) / sig) ** 2)
            x[c, lo:hi] += (amp * prof).astype(np.float32)
    return x


def run_engine(engine, stream, gulp, masks=None, drain=True):
    """Executes gulp by gulp (mask g applied by zeroing, as the RFI stage
    does), then drains; returns all candidates (numpy structured array)."""
    out = []
    ngulps = stream.shape[1] // gulp
    for g in range(ngulps):
        wf = np.ascontiguousarray(stream[:, g * gulp:(g + 1) * gulp])
        mask = None
        if masks is not None:
            mask = masks[g]
            wf = wf * mask[:, None].astype(np.float32)
        res = engine.execute(wf, mask)
        assert not res.overflowed()
        out.append(res.candidates.copy())
    if drain:
        out.append(engine.drain().candidates.copy())
    return np.concatenate(out) if out else np.zeros(0)


def key(plane, dm_idx, width_idx, peak):
    return (int(plane[0]), int(plane[1]), int(dm_idx), int(width_idx), int(peak))


def compare(gpu, oracle_cands, thresh, snr_rtol=1e-3, margin=0.02):
    """Every oracle peak clear of the threshold must be reported by the GPU
    with the same plane, DM index, width and peak sample, and S/N within
    snr_rtol; and vice versa. Returns (matched, details)."""
    g = {key((c["subband_level"], c["subband_idx"]), c["dm_idx"], c["filter_idx"], c["peak_sample"]): c
         for c in gpu}
    o = {key(c["plane"], c["dm_idx"], c["width_idx"], c["peak"]): c for c in oracle_cands}
    missing, extra, bad = [], [], []
    for k, c in o.items():
        if c["snr"] < thresh + margin:
            continue
        if k not in g:
            missing.append((k, c["snr"]))
            continue
        rel = abs(float(g[k]["snr"]) - c["snr"]) / c["snr"]
        if rel > snr_rtol:
            bad.append((k, float(g[k]["snr"]), c["snr"]))
    for k, c in g.items():
        if float(c["snr"]) >= thresh + margin and k not in o:
            extra.append((k, float(c["snr"])))
    return len(o), missing, extra, bad


def same_detections(a, b, thresh, snr_rtol=1e-5, margin=0.02):
    """Two engines' candidates agree: every peak clear of the threshold in
    either list is in the other with the same plane, DM index, width and
    peak sample, S/N within snr_rtol (search steps of different lengths
    round their window sums from different prefix origins)."""
    ka = {key((c["subband_level"], c["subband_idx"]), c["dm_idx"], c["filter_idx"], c["peak_sample"]): float(c["snr"])
          for c in a}
    kb = {key((c["subband_level"], c["subband_idx"]), c["dm_idx"], c["filter_idx"], c["peak_sample"]): float(c["snr"])
          for c in b}
    for x, y in ((ka, kb), (kb, ka)):
        for k, s in x.items():
            if s < thresh + margin:
                continue
            if k not in y or abs(y[k] - s) > snr_rtol * s:
                return False
    return True
