"""TEST INFRASTRUCTURE ONLY — Python driver of the FP64 search oracle
(oracle/fdmt_oracle.c, built into oracle/_build/libfrost_oracle.so).

Restates, independently of frost_b200's C++ plan, which bands are searched
(full band; at depth s the 2^s halving bands and the 2^s - 1 staggered bands
that merge the adjacent depth-(s+1) bands across each boundary, as frost's
sub-band search describes: docs/user_guide/search.md:51-65,
tests/cpp/api/dedisp_test.cpp:30-54), which DM rows each band has (distinct
rounded delays of the DM list across the band), and computes every row,
variance and peak in FP64. Parity with dmt itself is unpinned (dmt is not
available); see the header of fdmt_oracle.c.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libfrost_oracle.so")
_lib = None


class OracleCand(C.Structure):
    _fields_ = [("row", C.c_int64), ("width_idx", C.c_int64), ("peak", C.c_int64),
                ("begin", C.c_int64), ("end", C.c_int64), ("snr", C.c_double)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is not built (make -C oracle oracle)")
        L = C.CDLL(LIB)
        i64p, f64p, u8p = C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_uint8)
        L.oracle_band_delay.restype = C.c_int64
        L.oracle_band_delay.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double]
        L.oracle_row_geometry.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_int64, C.c_int64,
                                          C.c_int64, i64p, C.c_int64, i64p, i64p]
        L.oracle_dedisperse.argtypes = [f64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, i64p, i64p,
                                        C.c_int64, f64p]
        L.oracle_variance.argtypes = [i64p, C.c_int64, C.c_int64, u8p, C.c_int64, C.c_int, f64p]
        L.oracle_dedisperse_rows.argtypes = [C.POINTER(C.c_float), C.c_int64, C.c_int64, C.c_int64,
                                             C.c_int64, i64p, i64p, C.c_int64, f64p]
        L.cpu_fdmt_search.restype = C.c_int64
        L.cpu_fdmt_search.argtypes = [C.POINTER(C.c_float), C.c_int64, C.c_int64, C.c_double,
                                      C.c_double, C.c_double, C.POINTER(C.c_float), C.c_int64,
                                      C.c_int64, i64p, C.c_int64, C.c_double]
        L.oracle_search.restype = C.c_int64
        L.oracle_search.argtypes = [f64p, C.c_int64, C.c_int64, i64p, i64p, C.c_int64, f64p, f64p,
                                    C.c_int64, u8p, C.c_double, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(OracleCand), C.c_int64]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


@dataclass
class Band:
    a: int
    m: int
    b: int
    level: int
    idx: int
    staggered: int
    delays: np.ndarray = field(default=None)
    dm: np.ndarray = field(default=None)
    dm_index: np.ndarray = field(default=None)


def bands(nchans: int, depth: int) -> List[Band]:
    """Searched bands in frost's plane order: full band, then per depth s the
    halving bands followed by the staggered bands."""
    def halve(a, b, d, out):
        out.setdefault(d, []).append((a, b))
        if b - a > 1:
            m = a + (b - a) // 2
            halve(a, m, d + 1, out)
            halve(m, b, d + 1, out)
    by_depth = {}
    halve(0, nchans, 0, by_depth)
    out = [Band(0, nchans // 2, nchans, 0, 0, 0)]
    for s in range(1, depth + 1):
        regular = by_depth[s]
        halves = by_depth[s + 1]
        for i, (a, b) in enumerate(regular):
            out.append(Band(a, a + (b - a) // 2, b, s, i, 0))
        for i in range(len(regular) - 1):
            a = halves[2 * i + 1][0]
            m = halves[2 * i + 1][1]
            b = halves[2 * i + 2][1]
            out.append(Band(a, m, b, s, len(regular) + i, 1))
    return out


def widths(max_boxcar: int, wtsp: float) -> List[int]:
    """1, then max(ceil(wtsp * w), w + 1) while <= max_boxcar."""
    w = [1]
    while True:
        n = max(int(np.ceil(float(np.float32(wtsp)) * w[-1])), w[-1] + 1)
        if n > max_boxcar:
            return w
        w.append(n)


class Oracle:
    """FP64 dedispersion search of a whole stream of gulps."""

    def __init__(self, nchans, f_min, f_max, tsamp, dm_list, depth, max_boxcar, wtsp=2.0,
                 trapezoid=False, thresh=6.0, peak_mode=0, skip_cold=True):
        self.nchans, self.f_min, self.f_max = nchans, float(f_min), float(f_max)
        self.tsamp = float(np.float32(tsamp))
        self.dm_list = np.asarray(dm_list, np.float32)
        self.widths = widths(max_boxcar, wtsp)
        self.trapezoid, self.thresh, self.peak_mode, self.skip_cold = trapezoid, thresh, peak_mode, skip_cold
        L = lib()
        self.bands = bands(nchans, depth)
        for band in self.bands:
            f_lo = self.edge(band.a)
            f_hi = self.edge(band.b)
            d = np.array([L.oracle_band_delay(float(dm), f_lo, f_hi, self.tsamp) for dm in self.dm_list],
                         np.int64)
            keep = np.concatenate([[True], d[1:] != d[:-1]])
            band.delays = d[keep]
            band.dm = self.dm_list[keep]
            band.dm_index = np.nonzero(keep)[0]

    def edge(self, c):
        bw = (self.f_max - self.f_min) / self.nchans
        return self.f_min + c * bw

    def geometry(self, band: Band, rows=None):
        """Per-channel shifts and window lengths of the band's rows (all, or
        the selected row indices), each [rows][b - a]."""
        n = band.b - band.a
        delays = np.ascontiguousarray(band.delays if rows is None else band.delays[np.asarray(rows)], np.int64)
        nr = delays.size
        shifts = np.zeros(nr * n, np.int64)
        lens = np.zeros(nr * n, np.int64)
        rc = lib().oracle_row_geometry(self.nchans, self.f_min, self.f_max, band.a, band.m, band.b,
                                       _p(delays, C.c_int64), nr, _p(shifts, C.c_int64),
                                       _p(lens, C.c_int64))
        assert rc == 0
        return shifts.reshape(nr, n), lens.reshape(nr, n)

    def dedisperse_rows(self, stream: np.ndarray, band: Band, rows) -> np.ndarray:
        """Selected rows of a band from a float32 [nchans][T] stream (masked
        channels already zero) -> [len(rows)][T] FP64, without an FP64 copy
        of the stream (sliding FP64 windows)."""
        x = np.ascontiguousarray(stream, np.float32)
        T = x.shape[1]
        shifts, lens = self.geometry(band, rows)
        out = np.zeros((shifts.shape[0], T), np.float64)
        shifts, lens = np.ascontiguousarray(shifts), np.ascontiguousarray(lens)
        rc = lib().oracle_dedisperse_rows(_p(x, C.c_float), self.nchans, T, band.a, band.b,
                                          _p(shifts, C.c_int64), _p(lens, C.c_int64), shifts.shape[0],
                                          _p(out, C.c_double))
        assert rc == 0
        return out

    def dedisperse(self, stream: np.ndarray, band: Band) -> np.ndarray:
        """stream: [nchans][T] (masked channels already zero) -> [rows][T] FP64."""
        x = np.ascontiguousarray(stream, np.float64)
        T = x.shape[1]
        shifts, lens = self.geometry(band)
        out = np.zeros((band.delays.size, T), np.float64)
        rc = lib().oracle_dedisperse(_p(x, C.c_double), self.nchans, T, band.a, band.b,
                                     _p(shifts, C.c_int64), _p(lens, C.c_int64), band.delays.size,
                                     _p(out, C.c_double))
        assert rc == 0
        return out

    def variance(self, band: Band, mask: np.ndarray, W: int, rows=None) -> np.ndarray:
        _, lens = self.geometry(band, rows)
        m = np.ascontiguousarray(mask[band.a:band.b], np.uint8)
        out = np.zeros(lens.shape[0], np.float64)
        lens = np.ascontiguousarray(lens)
        rc = lib().oracle_variance(_p(lens, C.c_int64), lens.shape[0], lens.shape[1], _p(m, C.c_uint8),
                                   W, int(self.trapezoid), _p(out, C.c_double))
        assert rc == 0
        return out

    def search(self, stream: np.ndarray, gulp: int, masks: List[np.ndarray], rows=None, data=None):
        """Searches the whole stream ([nchans][T], T a multiple of `gulp`,
        gulp g under masks[g] with its masked channels already zero).
        `rows` (optional) maps a band index to the row indices to search;
        other bands are skipped. `data` (optional) maps a band index to
        those rows' FP64 values already computed by dedisperse_rows.
        Returns a list of dicts sorted like the engine's results, with
        dm_idx the row index within the band."""
        T = stream.shape[1]
        ngulps = T // gulp
        assert ngulps * gulp == T and len(masks) == ngulps
        or_gulp = np.zeros(ngulps, np.uint8)
        for g in range(1, ngulps):
            or_gulp[g] = np.any(masks[g] != masks[g - 1])
        ws = np.array(self.widths, np.int64)
        out = []
        for bi, band in enumerate(self.bands):
            sel = None
            if rows is not None:
                if bi not in rows:
                    continue
                sel = np.asarray(sorted(set(int(r) for r in rows[bi])), np.int64)
                band = Band(band.a, band.m, band.b, band.level, band.idx, band.staggered,
                            band.delays[sel], band.dm[sel], band.dm_index[sel])
                if data is not None and bi in data:
                    rows_data = np.ascontiguousarray(data[bi], np.float64)
                    assert rows_data.shape == (sel.size, T)
                else:
                    rows_data = self.dedisperse_rows(stream, self.bands[bi], sel)
            else:
                rows_data = self.dedisperse(stream, band)
            # variance per gulp mask: the search uses one table per gulp, so
            # run gulp by gulp when masks differ
            var_by_mask = {}

            def var_of(mask, band=band, bi=bi, sel=sel):
                key = mask.tobytes()
                if key not in var_by_mask:
                    var_by_mask[key] = np.stack([self.variance(self.bands[bi], mask, W, sel)
                                                 for W in self.widths], 1)
                return var_by_mask[key]
            if all(np.array_equal(m, masks[0]) for m in masks):
                v = np.ascontiguousarray(var_of(masks[0]))
                found = self._search_rows(rows_data, band, ws, v, v, T, or_gulp, ngulps * gulp)
            else:
                # gulp-wise: S/N in gulp g uses masks[g] (OR with masks[g-1]
                # at the start); runs are carried by searching the stream once
                # per gulp-mask with the other gulps' S/N suppressed is not
                # equivalent, so assemble per-gulp S/N tables instead.
                found = self._search_mixed(rows_data, band, ws, masks, gulp, or_gulp, var_of)
            if sel is not None:
                for c in found:
                    c["dm_idx"] = int(sel[c["dm_idx"]])
            out += found
        return out

    def _search_rows(self, rows, band, ws, var, var_or, T, or_gulp, gulp):
        cap = 1 << 20
        buf = (OracleCand * cap)()
        rows = np.ascontiguousarray(rows)
        n = lib().oracle_search(_p(rows, C.c_double), rows.shape[0], T, _p(band.delays, C.c_int64),
                                _p(ws, C.c_int64), ws.size, _p(var, C.c_double),
                                _p(var_or, C.c_double), gulp, _p(or_gulp, C.c_uint8),
                                self.thresh, self.peak_mode, int(self.trapezoid),
                                int(self.skip_cold), buf, cap)
        assert 0 <= n <= cap
        return [self._cand(band, buf[i]) for i in range(n)]

    def _search_mixed(self, rows, band, ws, masks, gulp, or_gulp, var_of):
        # Per-gulp variance: scale each gulp's rows so that one table applies
        # would change the run extents' S/N, so instead evaluate S/N in
        # Python (FP64) and find runs here.
        nr, T = rows.shape
        nw = len(self.widths)
        snr = np.full((nw, nr, T), -np.inf)
        pre = np.concatenate([np.zeros((nr, 1)), np.cumsum(rows, axis=1)], axis=1)

        def P(i):
            i = np.clip(i, 0, None)
            return pre[:, i]
        t = np.arange(T)
        for wi, W in enumerate(self.widths):
            s = P(t + 1) - P(t + 1 - W)
            if self.trapezoid and W >= 3:
                e = (W + 1) // 4
                s = s - 0.5 * ((P(t + 1) - P(t + 1 - e)) + (P(t + 1 - W + e) - P(t + 1 - W)))
            for g in range(len(masks)):
                v = var_of(masks[g])[:, wi]
                vo = var_of(np.maximum(masks[g], masks[g - 1]) if g > 0 else masks[g])[:, wi]
                sl = slice(g * gulp, (g + 1) * gulp)
                tt = t[sl]
                use_or = or_gulp[g] & ((tt[None, :] - g * gulp) < (band.delays[:, None] + W - 1))
                vv = np.where(use_or, vo[:, None], v[:, None])
                with np.errstate(divide="ignore", invalid="ignore"):
                    val = np.where(vv > 0, s[:, sl] / np.sqrt(vv), -np.inf)
                if self.skip_cold:
                    val = np.where(tt[None, :] < band.delays[:, None] + W - 1, -np.inf, val)
                snr[wi, :, sl] = val
        out = []
        for r in range(nr):
            if self.peak_mode == 2:
                for wi in range(nw):
                    for tt in np.nonzero(snr[wi, r] > self.thresh)[0]:
                        out.append(self._mk(band, r, wi, tt, tt, tt, snr[wi, r, tt]))
                continue
            passes = range(nw) if self.peak_mode == 0 else [None]
            for wi in passes:
                if wi is None:
                    best_w = np.argmax(snr[:, r, :], axis=0)
                    series = snr[best_w, r, np.arange(T)]
                else:
                    series = snr[wi, r]
                up = series > self.thresh
                tt = 0
                while tt < T:
                    if not up[tt]:
                        tt += 1
                        continue
                    start = tt
                    while tt < T and up[tt]:
                        tt += 1
                    seg = series[start:tt]
                    k = int(np.argmax(seg))
                    pk = start + k
                    w = wi if wi is not None else int(best_w[pk])
                    out.append(self._mk(band, r, w, pk, start, tt - 1, seg[k]))
        return out

    def _mk(self, band, row, wi, peak, begin, end, snr):
        return {"plane": (band.level, band.idx), "dm_idx": int(row), "width_idx": int(wi),
                "width": self.widths[wi], "peak": int(peak), "begin": int(begin), "end": int(end),
                "snr": float(snr), "dm": float(band.dm[row])}

    def _cand(self, band, c):
        return self._mk(band, c.row, c.width_idx, c.peak, c.begin, c.end, c.snr)


def cpu_search(waterfall: np.ndarray, f_min: float, f_max: float, tsamp: float, dm_list,
               depth: int, widths_list, thresh: float = 6.0) -> int:
    """The CPU port of the search (oracle/cpu_fdmt.c) on one [nchans][T]
    float32 block with zero history; returns the peak count. Timed as the CPU
    baseline; not a correctness oracle."""
    x = np.ascontiguousarray(waterfall, np.float32)
    dms = np.ascontiguousarray(dm_list, np.float32)
    ws = np.ascontiguousarray(widths_list, np.int64)
    n = lib().cpu_fdmt_search(_p(x, C.c_float), x.shape[0], x.shape[1], float(f_min), float(f_max),
                              float(tsamp), _p(dms, C.c_float), dms.size, depth, _p(ws, C.c_int64),
                              ws.size, float(thresh))
    if n < 0:
        raise RuntimeError("cpu_fdmt_search failed")
    return int(n)
