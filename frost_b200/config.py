"""Configuration types with frost's names, defaults and meanings.

RfiConfig and its strategy structs follow include/frost/prepare/rfi.hpp:
112-191, BlockLayout :194-201, DedispPlanConfig
include/frost/dedisp/dedisp.hpp:12-27 and the search settings
include/frost/config/config.hpp:56-97 (SearchConfig) with dmt's BoxcarConfig
fields as frost sets them (lib/pipeline/pipeline.cpp:316-330).
"""

from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import List, Tuple

from . import _abi


class DataType(enum.IntEnum):
    UINT1 = _abi.UINT1
    UINT2 = _abi.UINT2
    UINT4 = _abi.UINT4
    UINT8 = _abi.UINT8
    UINT16 = _abi.UINT16
    UINT32 = _abi.UINT32
    FLOAT32 = _abi.FLOAT32

    @property
    def bits(self) -> int:
        return _abi.DTYPE_BITS[int(self)]


class FillMode(enum.IntEnum):
    NEIGHBOUR = _abi.FILL_NEIGHBOUR
    MEAN = _abi.FILL_MEAN
    NOISE = _abi.FILL_NOISE


class ZeroDMMode(enum.IntEnum):
    OFF = _abi.ZERO_DM_OFF
    SUBTRACT = _abi.ZERO_DM_SUBTRACT
    ZDOT = _abi.ZERO_DM_ZDOT


class PeakMode(enum.IntEnum):
    PER_WIDTH = _abi.PEAK_PER_WIDTH
    ACROSS_WIDTHS = _abi.PEAK_ACROSS_WIDTHS
    ALL = _abi.PEAK_ALL


class Storage(enum.IntEnum):
    FP32 = _abi.STORAGE_FP32
    FP16 = _abi.STORAGE_FP16


@dataclass
class NarrowbandConfig:
    enabled: bool = True
    threshold: float = 5.0


@dataclass
class BroadbandConfig:
    enabled: bool = True
    threshold: float = 5.0
    boxcar_max: int = 1


@dataclass
class DropoutConfig:
    enabled: bool = False
    min_std_fraction: float = 0.1


@dataclass
class MomentsConfig:
    enabled: bool = False
    threshold: float = 4.0
    mean: bool = True
    std: bool = True
    skewness: bool = True
    kurtosis: bool = True
    autocorr: bool = True
    kurtosis_max: float = 0.0


@dataclass
class IqrmConfig:
    enabled: bool = False
    threshold: float = 3.0
    radius: int = 0


@dataclass
class KadaneChannelConfig:
    enabled: bool = False
    threshold: float = 7.0
    min_duration: float = 0.05


@dataclass
class KadaneSpectrumConfig:
    enabled: bool = False
    threshold: float = 7.0
    min_bandwidth: float = 10.0
    whole_band_fraction: float = 0.8


@dataclass
class RfiConfig:
    zap_chans: List[Tuple[int, int]] = field(default_factory=list)
    zap_freqs: List[Tuple[float, float]] = field(default_factory=list)
    narrow: NarrowbandConfig = field(default_factory=NarrowbandConfig)
    broad: BroadbandConfig = field(default_factory=BroadbandConfig)
    dropout: DropoutConfig = field(default_factory=DropoutConfig)
    moments: MomentsConfig = field(default_factory=MomentsConfig)
    iqrm: IqrmConfig = field(default_factory=IqrmConfig)
    mask_grow: int = 0
    kadane_channel: KadaneChannelConfig = field(default_factory=KadaneChannelConfig)
    kadane_spectrum: KadaneSpectrumConfig = field(default_factory=KadaneSpectrumConfig)
    zero_dm: ZeroDMMode = ZeroDMMode.OFF
    equalize: bool = False
    fill: FillMode = FillMode.NEIGHBOUR
    seed: int = 0x5EED

    @staticmethod
    def quiet() -> "RfiConfig":
        """Every automatic strategy off (only manual zaps apply)."""
        cfg = RfiConfig()
        cfg.narrow.enabled = False
        cfg.broad.enabled = False
        return cfg

    def to_c(self):
        """Returns (RfiConfigC, keepalive) — keep the second alive while the
        struct is in use, it owns the zap arrays."""
        zc = (_abi.ChannelRange * max(len(self.zap_chans), 1))(
            *[_abi.ChannelRange(int(a), int(b)) for a, b in self.zap_chans])
        zf = (_abi.FrequencyRange * max(len(self.zap_freqs), 1))(
            *[_abi.FrequencyRange(float(a), float(b)) for a, b in self.zap_freqs])
        c = _abi.RfiConfigC()
        c.zap_chans = C.cast(zc, C.POINTER(_abi.ChannelRange))
        c.n_zap_chans = len(self.zap_chans)
        c.zap_freqs = C.cast(zf, C.POINTER(_abi.FrequencyRange))
        c.n_zap_freqs = len(self.zap_freqs)
        c.narrow_enabled = int(self.narrow.enabled)
        c.narrow_threshold = self.narrow.threshold
        c.broad_enabled = int(self.broad.enabled)
        c.broad_threshold = self.broad.threshold
        c.broad_boxcar_max = int(self.broad.boxcar_max)
        c.dropout_enabled = int(self.dropout.enabled)
        c.dropout_min_std_fraction = self.dropout.min_std_fraction
        m = self.moments
        c.moments_enabled = int(m.enabled)
        c.moments_threshold = m.threshold
        c.moments_mean = int(m.mean)
        c.moments_std = int(m.std)
        c.moments_skewness = int(m.skewness)
        c.moments_kurtosis = int(m.kurtosis)
        c.moments_autocorr = int(m.autocorr)
        c.moments_kurtosis_max = m.kurtosis_max
        c.iqrm_enabled = int(self.iqrm.enabled)
        c.iqrm_threshold = self.iqrm.threshold
        c.iqrm_radius = int(self.iqrm.radius)
        c.mask_grow = int(self.mask_grow)
        c.kadane_channel_enabled = int(self.kadane_channel.enabled)
        c.kadane_channel_threshold = self.kadane_channel.threshold
        c.kadane_channel_min_duration = self.kadane_channel.min_duration
        ks = self.kadane_spectrum
        c.kadane_spectrum_enabled = int(ks.enabled)
        c.kadane_spectrum_threshold = ks.threshold
        c.kadane_spectrum_min_bandwidth = ks.min_bandwidth
        c.kadane_spectrum_whole_band_fraction = ks.whole_band_fraction
        c.zero_dm = int(self.zero_dm)
        c.equalize = int(self.equalize)
        c.fill = int(self.fill)
        c.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        return c, (zc, zf)


@dataclass
class BlockLayout:
    nchans: int = 0
    max_nsamps: int = 0
    dtype: DataType = DataType.UINT8
    tsamp: float = 0.0
    f0: float = 0.0
    df: float = 0.0

    @property
    def row_bytes(self) -> int:
        return self.nchans * DataType(self.dtype).bits // 8

    def to_c(self) -> _abi.BlockLayoutC:
        return _abi.BlockLayoutC(int(self.nchans), int(self.max_nsamps), int(self.dtype),
                                 float(self.tsamp), float(self.f0), float(self.df))


@dataclass
class DedispPlanConfig:
    nchans: int = 0
    dt: float = 0.0
    f0: float = 0.0
    df: float = 0.0
    dm_min: float = 0.0
    dm_max: float = 0.0
    dm_pulse_width: float = 0.0
    dm_tol: float = 1.25
    dm_dtype: DataType = DataType.FLOAT32
    block_nsamps: int = 0
    subband_depth: int = 0

    def to_c(self) -> _abi.DedispPlanConfigC:
        return _abi.DedispPlanConfigC(int(self.nchans), self.dt, self.f0, self.df, self.dm_min,
                                      self.dm_max, self.dm_pulse_width, self.dm_tol,
                                      int(self.dm_dtype), int(self.block_nsamps),
                                      int(self.subband_depth))


@dataclass
class BoxcarConfig:
    """dmt::BoxcarConfig as frost fills it (lib/pipeline/pipeline.cpp:316-330)
    plus the FDMT plane storage precision."""
    max_boxcar: int = 4096
    wtsp: float = 2.0
    use_trapezoid: bool = False
    detect_thresh: float = 6.0
    noise_sigma: float = 1.0
    peak_mode: PeakMode = PeakMode.PER_WIDTH
    max_candidates: int = 131072
    max_cands_per_dm: int = 4096
    skip_cold_prefix: bool = True
    storage: Storage = Storage.FP32
    tile_nsamps: int = 0  # FDMT tile in samples (multiple of 4096); 0 = the whole gulp
