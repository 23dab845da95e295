"""Seeded synthetic filterbanks with the shapes, value distributions and
injections of the benchmark configurations (no public dataset exists for
this path; these inputs are the whole workload).

Noise: N(mean, sd) rounded and clipped to the sample range (uint8) or kept as
float32. Pulses: Gaussian profiles (sigma_t = width / 2.355) dispersed by
Delta t = 4.148808e3 DM (f^-2 - f_top^-2) / tsamp relative to the top
channel, with per-channel amplitude S/N * sd / sqrt(C_active * w_eff),
w_eff = max(1, 1.064 width) — the recipe of frost's fake filterbank
(tests/cpp/support/fake_filterbank.hpp:18-125) with Gaussian instead of
boxcar profiles. RFI: noisy narrow-band channels, zero-DM broadband bursts
and dropout runs.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

KDM = 4.148808e3  # s MHz^2 / (pc cm^-3)


@dataclass
class Pulse:
    t0: float      # arrival sample at the top channel
    dm: float
    width: float   # FWHM in samples
    snr: float


@dataclass
class Filterbank:
    data: np.ndarray          # [nsamps][nchans], uint8 or float32
    fch1: float
    foff: float
    tsamp: float
    pulses: List[Pulse] = field(default_factory=list)
    rfi_channels: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    bursts: List[Tuple[int, int]] = field(default_factory=list)
    dropouts: List[Tuple[int, int]] = field(default_factory=list)

    @property
    def nsamps(self):
        return self.data.shape[0]

    @property
    def nchans(self):
        return self.data.shape[1]

    def freqs(self):
        return self.fch1 + self.foff * np.arange(self.nchans)


def dispersion_delay(dm, f, f_ref, tsamp):
    """Delay in samples of frequency f relative to f_ref."""
    return KDM * dm * (1.0 / np.square(f) - 1.0 / (f_ref * f_ref)) / tsamp


_CHUNK_ROWS = 8192


def _chunks(nsamps):
    return [(a, min(a + _CHUNK_ROWS, nsamps)) for a in range(0, nsamps, _CHUNK_ROWS)]


def _parallel(fn, items):
    """Runs fn over items on host threads (numpy's random fills and ufuncs
    release the GIL); the result does not depend on the thread count."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    workers = max(1, min(len(items), os.cpu_count() or 1))
    if workers == 1:
        for it in items:
            fn(it)
        return
    with ThreadPoolExecutor(workers) as ex:
        list(ex.map(fn, items))


def make_filterbank(nchans: int, nsamps: int, fch1: float, foff: float, tsamp: float,
                    seed: int, dtype: str = "uint8", mean: float = 128.0, sd: float = 16.0,
                    pulses: Optional[List[Pulse]] = None, n_pulses: int = 0,
                    dm_range=(50.0, 450.0), width_range=(1.0, 16.0), snr_range=(8.0, 30.0),
                    rfi_channel_fraction: float = 0.0, rfi_var_factor: float = 10.0,
                    n_bursts: int = 0, burst_len=(1, 50), burst_sigma: float = 40.0,
                    n_dropouts: int = 0, dropout_len: int = 512,
                    first_sample: int = 0) -> Filterbank:
    """A seeded filterbank. `first_sample` offsets pulse times so successive
    gulps of one stream can be generated independently. The noise of each
    8192-row chunk comes from its own generator spawned from `seed`, so the
    output is the same however many threads fill it."""
    rng = np.random.default_rng(seed)
    chunks = _chunks(nsamps)
    streams = np.random.SeedSequence(seed).spawn(len(chunks))
    noise = np.empty((nsamps, nchans), np.float32)
    freqs = fch1 + foff * np.arange(nchans)
    f_top = freqs.max()
    rfi_channels = np.zeros(0, np.int64)
    if rfi_channel_fraction > 0:
        k = int(round(rfi_channel_fraction * nchans))
        rfi_channels = np.sort(rng.choice(nchans, size=k, replace=False))
    extra = np.sqrt(rfi_var_factor - 1.0) * sd if rfi_channels.size else 0.0

    def fill(i):
        a, b = chunks[i]
        g = np.random.default_rng(streams[i])
        part = noise[a:b]
        g.standard_normal(out=part, dtype=np.float32)
        part *= sd
        part += mean
        if rfi_channels.size:
            part[:, rfi_channels] += extra * g.standard_normal((b - a, rfi_channels.size), dtype=np.float32)
    _parallel(fill, range(len(chunks)))
    if pulses is None:
        pulses = []
        delay_max = dispersion_delay(dm_range[1], freqs.min(), f_top, tsamp)
        for _ in range(n_pulses):
            width = float(rng.uniform(*width_range))
            dm = float(rng.uniform(*dm_range))
            lo = 2 * width
            hi = max(lo + 1, nsamps - delay_max - 2 * width)
            pulses.append(Pulse(float(rng.uniform(lo, hi)) + first_sample, dm, width,
                                float(rng.uniform(*snr_range))))
    if pulses:
        n_active = nchans
        t = np.arange(nsamps, dtype=np.float64) + first_sample
        for p in pulses:
            sig_t = max(p.width / 2.355, 0.25)
            w_eff = max(1.0, 1.064 * p.width)
            amp = p.snr * sd / np.sqrt(n_active * w_eff)
            delays = dispersion_delay(p.dm, freqs, f_top, tsamp)
            half = int(np.ceil(4 * sig_t)) + 1
            for c in range(nchans):
                centre = p.t0 + delays[c]
                a = int(np.floor(centre)) - half - first_sample
                b = int(np.ceil(centre)) + half + 1 - first_sample
                a0, b0 = max(a, 0), min(b, nsamps)
                if a0 >= b0:
                    continue
                tt = t[a0:b0]
                prof = np.exp(-0.5 * np.square((tt - centre) / sig_t))
                prof *= 1.0 / (prof.sum() if prof.sum() > 0 else 1.0)
                # per-channel fluence amp * w_eff spread over the profile
                noise[a0:b0, c] += (amp * w_eff * prof).astype(np.float32)
    bursts = []
    for _ in range(n_bursts):
        length = int(rng.integers(burst_len[0], burst_len[1] + 1))
        start = int(rng.integers(0, max(nsamps - length, 1)))
        noise[start:start + length, :] += burst_sigma * sd
        bursts.append((start, length))
    dropouts = []
    for _ in range(n_dropouts):
        start = int(rng.integers(0, max(nsamps - dropout_len, 1)))
        noise[start:start + dropout_len, :] = 0.0
        dropouts.append((start, dropout_len))
    if dtype == "uint8":
        data = np.empty((nsamps, nchans), np.uint8)

        def quantise(i):
            a, b = chunks[i]
            part = noise[a:b]
            np.rint(part, out=part)
            np.clip(part, 0, 255, out=part)
            data[a:b] = part
        _parallel(quantise, range(len(chunks)))
    elif dtype == "float32":
        data = noise
    else:
        raise ValueError(dtype)
    return Filterbank(data, fch1, foff, tsamp, pulses, rfi_channels, bursts, dropouts)


def config1_gulp(seed: int = 0x46524F5354, nsamps: int = 65536, gulp_index: int = 0) -> Filterbank:
    """1024 channels from 1500 MHz, foff -0.29296875, 64 us, default RFI."""
    return make_filterbank(1024, nsamps, 1500.0, -0.29296875, 64e-6, seed + gulp_index,
                           n_pulses=5 if gulp_index == 0 else 0, dm_range=(50, 450),
                           width_range=(1, 16), snr_range=(8, 30),
                           first_sample=gulp_index * nsamps)


def config2_gulp(seed: int = 0x46524F5354, nsamps: int = 262144, nchans: int = 4096,
                 n_pulses: int = 20) -> Filterbank:
    """4096 channels over 1200-1536 MHz, 64 us, with narrow-band, burst and
    dropout RFI and 20 pulses at DM 100-1900."""
    foff = -0.08203125 * (4096 / nchans)
    fch1 = 1536.0 + foff / 2
    return make_filterbank(nchans, nsamps, fch1, foff, 64e-6, seed, n_pulses=n_pulses,
                           dm_range=(100, 1900), width_range=(1, 128), snr_range=(7, 50),
                           rfi_channel_fraction=0.05, n_bursts=20, n_dropouts=3)
