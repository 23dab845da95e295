"""Seeded RFI-cleaner scenarios shared by the golden-fixture generator and
the GPU parity tests. Each covers one strategy mix of frost's RFICleaner
(include/frost/prepare/rfi.hpp) on a small block the CPU reference finishes
in well under a second; together they reach every strategy, fill mode and
transform, every packed dtype, short tails with and without a retained
calibration, dead and fully masked channels."""

from __future__ import annotations

import numpy as np

from frost_b200.config import (BlockLayout, DataType, FillMode, RfiConfig, ZeroDMMode)


def pack(values: np.ndarray, dtype: DataType) -> np.ndarray:
    """Time-major [nsamps][nchans] values -> packed bytes (LSB-first below 8 bits)."""
    v = np.asarray(values)
    if dtype == DataType.FLOAT32:
        return np.ascontiguousarray(v, dtype=np.float32).view(np.uint8).reshape(-1)
    if dtype == DataType.UINT8:
        return np.ascontiguousarray(v, dtype=np.uint8).reshape(-1)
    if dtype == DataType.UINT16:
        return np.ascontiguousarray(v, dtype=np.uint16).view(np.uint8).reshape(-1)
    if dtype == DataType.UINT32:
        return np.ascontiguousarray(v, dtype=np.uint32).view(np.uint8).reshape(-1)
    bits = dtype.bits
    flat = np.ascontiguousarray(v, dtype=np.uint8).reshape(-1)
    per = 8 // bits
    flat = flat.reshape(-1, per)
    out = np.zeros(flat.shape[0], np.uint8)
    for k in range(per):
        out |= (flat[:, k] & ((1 << bits) - 1)) << (k * bits)
    return out


def noise(rng, nsamps, nchans, mean, sd, lo=None, hi=None, as_float=False):
    x = rng.normal(mean, sd, (nsamps, nchans))
    if as_float:
        return x.astype(np.float32)
    return np.clip(np.rint(x), lo, hi)


def inject(x, rng, mean, sd, hi=None, narrow=12, bursts=((1500, 3, 6.0),), rfi_chans=(), drop=None,
           dead=None):
    """Narrow-band spikes, broadband bursts (start, len, sigma), noisy
    channels, a dropout run (start, len) and a constant (dead) channel."""
    T, C = x.shape
    for _ in range(narrow):
        t, c = rng.integers(0, T), rng.integers(0, C)
        x[t, c] += 12 * sd
    for start, length, sig in bursts:
        if start < T:
            x[start:start + length, :] += sig * sd
    for c in rfi_chans:
        x[:, c] += rng.normal(0, 3 * sd, T)
    if drop is not None:
        # integer data drop to zero; float data to a flat spectrum at the mean
        x[drop[0]:drop[0] + drop[1], :] = 0 if hi is not None else mean
    if dead is not None:
        x[:, dead] = mean
    if hi is not None:
        x = np.clip(np.rint(x), 0, hi)
    return x


def layout(nchans, nsamps, dtype, tsamp=1e-3, f0=1500.0, df=-1.0):
    return BlockLayout(nchans, nsamps, dtype, tsamp, f0, df)


def everything(cfg: RfiConfig) -> RfiConfig:
    cfg.moments.enabled = True
    cfg.iqrm.enabled = True
    cfg.kadane_channel.enabled = True
    cfg.kadane_channel.min_duration = 0.02
    cfg.kadane_spectrum.enabled = True
    cfg.kadane_spectrum.min_bandwidth = 4.0
    cfg.dropout.enabled = True
    cfg.mask_grow = 1
    cfg.broad.boxcar_max = 8
    return cfg


def make_case(name: str):
    """Returns (RfiConfig, BlockLayout, baseline_length, [(packed block, nsamps), ...])."""
    seed = sum(map(ord, name)) * 7919 + 17
    rng = np.random.default_rng(seed)
    if name == "default_u8":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 128, 16, 0, 255), rng, 128, 16, hi=255)
        return RfiConfig(), layout(C, T, DataType.UINT8), 2.0, [(pack(x, DataType.UINT8), 0)]
    if name == "default_u8_partial":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 128, 16, 0, 255), rng, 128, 16, hi=255)
        return RfiConfig(), layout(C, T, DataType.UINT8), 2.0, [(pack(x, DataType.UINT8), 3001)]
    if name == "all_strategies_f32":
        C, T = 128, 6000
        x = noise(rng, T, C, 10.0, 2.0, as_float=True).astype(np.float64)
        x = inject(x, rng, 10.0, 2.0, narrow=30, bursts=((700, 4, 8.0), (4100, 20, 3.0)),
                   rfi_chans=(5, 6, 77), drop=(2500, 40), dead=100).astype(np.float32)
        # a weak long narrow-band drift for Kadane along time
        x[3000:3400, 40] += 1.5
        # a band-limited burst for Kadane across frequency
        x[5000:5003, 20:40] += 4.0
        cfg = everything(RfiConfig())
        cfg.zero_dm = ZeroDMMode.SUBTRACT
        cfg.zap_chans = [(0, 1), (120, 121)]
        cfg.zap_freqs = [(1450.2, 1452.8)]
        return cfg, layout(C, T, DataType.FLOAT32), 2.0, [(pack(x, DataType.FLOAT32), 0)]
    if name == "zdot_equalize_u8":
        C, T = 96, 5000
        x = inject(noise(rng, T, C, 100, 12, 0, 255), rng, 100, 12, hi=255,
                   bursts=((900, 5, 5.0), (3300, 2, 7.0)), rfi_chans=(11,))
        cfg = everything(RfiConfig())
        cfg.zero_dm = ZeroDMMode.ZDOT
        cfg.equalize = True
        return cfg, layout(C, T, DataType.UINT8, df=-0.5), 2.0, [(pack(x, DataType.UINT8), 0)]
    if name == "fill_noise_subtract":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 128, 16, 0, 255), rng, 128, 16, hi=255,
                   bursts=((1000, 3, 8.0), (3000, 2, 9.0)))
        cfg = RfiConfig()
        cfg.fill = FillMode.NOISE
        cfg.zero_dm = ZeroDMMode.SUBTRACT
        return cfg, layout(C, T, DataType.UINT8), 2.0, [(pack(x, DataType.UINT8), 0)]
    if name == "fill_mean_u4":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 8, 2, 0, 15), rng, 8, 2, hi=15)
        cfg = RfiConfig()
        cfg.fill = FillMode.MEAN
        return cfg, layout(C, T, DataType.UINT4), 2.0, [(pack(x, DataType.UINT4), 0)]
    if name == "u16_moments":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 3000, 100, 0, 65535), rng, 3000, 100, hi=65535, rfi_chans=(9, 33))
        cfg = RfiConfig()
        cfg.moments.enabled = True
        cfg.iqrm.enabled = True
        return cfg, layout(C, T, DataType.UINT16), 2.0, [(pack(x, DataType.UINT16), 0)]
    if name == "u32_u2_u1":
        C, T = 64, 4096
        x = inject(noise(rng, T, C, 1e6, 300, 0, 2**32 - 1), rng, 1e6, 300, hi=2**32 - 1)
        return RfiConfig(), layout(C, T, DataType.UINT32), 2.0, [(pack(x, DataType.UINT32), 0)]
    if name == "u2":
        C, T = 64, 4096
        x = noise(rng, T, C, 1.5, 0.8, 0, 3)
        return RfiConfig(), layout(C, T, DataType.UINT2), 2.0, [(pack(x, DataType.UINT2), 0)]
    if name == "u1":
        C, T = 64, 4096
        x = (rng.random((T, C)) < 0.5).astype(np.uint8)
        return RfiConfig(), layout(C, T, DataType.UINT1), 2.0, [(pack(x, DataType.UINT1), 0)]
    if name == "tail_sequence":
        C, T = 64, 4096
        cfg = RfiConfig()
        cfg.zero_dm = ZeroDMMode.SUBTRACT
        blocks = []
        for k, valid in enumerate((4096, 40, 4096, 10)):
            x = inject(noise(rng, T, C, 128, 16, 0, 255), rng, 128, 16, hi=255)
            blocks.append((pack(x, DataType.UINT8), valid))
        return cfg, layout(C, T, DataType.UINT8), 2.0, blocks
    if name == "short_cold":
        C, T = 64, 48
        x = noise(rng, T, C, 128, 16, 0, 255)
        return RfiConfig(), layout(C, T, DataType.UINT8), 2.0, [(pack(x, DataType.UINT8), 0)]
    if name == "all_masked":
        C, T = 32, 4096
        x = noise(rng, T, C, 128, 16, 0, 255)
        cfg = RfiConfig()
        cfg.zap_chans = [(0, 31)]
        return cfg, layout(C, T, DataType.UINT8), 2.0, [(pack(x, DataType.UINT8), 0)]
    if name == "ascending_dead_broadbox":
        C, T = 64, 8192
        x = inject(noise(rng, T, C, 128, 16, 0, 255), rng, 128, 16, hi=255,
                   bursts=((2000, 6, 2.5), (6000, 1, 9.0)), dead=17)
        cfg = RfiConfig()
        cfg.broad.boxcar_max = 16
        return cfg, layout(C, T, DataType.UINT8, df=0.25), 2.0, [(pack(x, DataType.UINT8), 0)]
    raise KeyError(name)


CASES = ["default_u8", "default_u8_partial", "all_strategies_f32", "zdot_equalize_u8",
         "fill_noise_subtract", "fill_mean_u4", "u16_moments", "u32_u2_u1", "u2", "u1",
         "tail_sequence", "short_cold", "all_masked", "ascending_dead_broadbox"]
