"""Search parity at the benchmark geometries, through the RFI stage.

The 1024-channel full-band workload (1200-1500 MHz, 64 us, DM 0-500, boxcar
widths 1-64) and the 4096-channel 11-plane workload (1200-1536 MHz, DM
0-2000, widths 1-256) run as two 65536-sample gulps of a seeded uint8
filterbank with dispersed pulses (and, at 4096 channels, the narrow-band,
burst and dropout RFI recipe): the GPU cleaner normalises each gulp, the GPU
engine searches it with the cleaner's channel mask, and the FP64 oracle
(oracle/fdmt_oracle.c) searches the same normalised stream. The second gulp
carries the first one's FDMT history, so the checks cover the inter-gulp
carry.

Bars (frost's acceptance for this path): FP32 DM-time plane rows within
1e-5 of each row's RMS; candidate plane / DM / width / peak indices
identical and S/N within 1e-3 for every peak clear of the threshold; FP16
plane storage gives the FP32 candidate list above S/N 7 with an S/N error
of at most 1e-2 (tests/cpp/api/calibration_test.cpp:137-144,
tests/cpp/api/gpu_parity_test.cpp:214-270 for the row-for-row comparison).
At 4096 channels every plane is checked on a seeded subset of its DM rows
(random rows, the rows nearest the injected pulses' DMs and rows where the
engine reported detections), which reaches the 64/128/256-sample widths and
the ~35k-sample level histories.
"""

import numpy as np
import pytest

from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig, Storage, ZeroDMMode
from frost_b200.dedisp import band_edges, generate_dm_list
from frost_b200.pipeline import plan_for
from frost_b200.synth import Pulse, config2_gulp, make_filterbank
from oracle.fdmt import Oracle
from tests.search_cases import compare

pytestmark = pytest.mark.gpu

GULP = 65536
TSAMP = 64e-6
ROW_RTOL = 1e-5      # FP32 plane rows vs FP64, relative to the row's RMS
SNR_RTOL = 1e-3      # candidate S/N vs FP64
FP16_SNR_RTOL = 1e-2  # FP16 storage vs FP32 above S/N 7


def oracle_for(pc, bc):
    f_min, f_max = band_edges(pc)
    return Oracle(pc.nchans, f_min, f_max, pc.dt, generate_dm_list(pc), pc.subband_depth,
                  bc.max_boxcar, bc.wtsp, bc.use_trapezoid, bc.detect_thresh, int(bc.peak_mode),
                  bc.skip_cold_prefix)


def clean_gulps(rfi_cfg, lay, data):
    """Normalised gulps ([nchans][T] float32, low frequency first) and their
    channel masks in FDMT order, from the GPU cleaner."""
    from frost_b200.rfi import RFICleaner
    cl = RFICleaner(rfi_cfg, lay, 2.0)
    wfs, masks = [], []
    for g in range(data.shape[0] // GULP):
        wfs.append(cl.execute_normalized(np.ascontiguousarray(data[g * GULP:(g + 1) * GULP])))
        m = cl.channel_mask()
        masks.append((m[::-1] if lay.df < 0 else m).copy())
    cl.close()
    return wfs, masks


def search_gulps(pc, bc, wfs, masks, capture_last=False):
    """Candidates of every gulp plus the drain; the engine is returned with
    the last gulp's planes captured when asked."""
    from frost_b200.search import FDMTBoxcar
    eng = FDMTBoxcar(pc, bc)
    out = []
    for g, (wf, m) in enumerate(zip(wfs, masks)):
        if capture_last and g == len(wfs) - 1:
            eng.capture_planes(True)
        res = eng.execute(wf, m)
        assert not res.overflowed(), (res.dropped_global, res.dropped_per_dm)
        out.append(res.candidates.copy())
    dr = eng.drain()
    assert not dr.overflowed()
    out.append(dr.candidates.copy())
    return np.concatenate(out), eng


def check_rows(eng, orc, stream, plane, band, rows):
    """The engine's captured last-gulp rows against the oracle's FP64 rows
    (sorted row indices); returns the worst error relative to the row RMS
    and the oracle's rows over the whole stream."""
    mine = eng.plane_data(plane, GULP)[rows]
    full = orc.dedisperse_rows(stream, band, rows)
    ref = full[:, -GULP:]
    rms = np.sqrt(np.mean(ref ** 2, axis=1, keepdims=True)) + 1e-12
    return float(np.max(np.abs(mine - ref) / rms)), full


def on_rows(cands, plane_key, rows):
    sel = (cands["subband_level"] == plane_key[0]) & (cands["subband_idx"] == plane_key[1]) & \
          np.isin(cands["dm_idx"], np.asarray(rows))
    return cands[sel]


def test_full_band_1024_channels_two_gulps_match_oracle():
    """1024 channels from 1500 MHz (foff -0.29296875), DM 0-500 (886 trials),
    widths 1-64, default RFI, full band: every row of the plane and every
    candidate of both gulps and the drain."""
    rng = np.random.default_rng(0x46524F5354)
    nchans, T = 1024, 2 * GULP
    fch1, foff = 1500.0, -0.29296875
    pulses = []
    for k in range(6):
        dm = float(rng.uniform(50, 450))
        width = float(rng.uniform(1, 16))
        snr = float(rng.uniform(8, 30))
        # arrival at the top channel; the fourth pulse's sweep crosses the
        # gulp boundary
        t0 = GULP - 3000.0 if k == 3 else float(rng.uniform(500, T - 9000))
        pulses.append(Pulse(t0, dm, width, snr))
    fb = make_filterbank(nchans, T, fch1, foff, TSAMP, seed=11, pulses=pulses)
    lay = BlockLayout(nchans, GULP, DataType.UINT8, TSAMP, fch1, foff)
    pc = plan_for(lay, 0.0, 500.0, 0)
    bc = BoxcarConfig(max_boxcar=64, wtsp=2.0, detect_thresh=6.0, max_candidates=1 << 20,
                      max_cands_per_dm=0)
    wfs, masks = clean_gulps(RfiConfig(), lay, fb.data)
    cands, eng = search_gulps(pc, bc, wfs, masks, capture_last=True)
    stream = np.concatenate(wfs, axis=1)
    orc = oracle_for(pc, bc)
    assert len(orc.bands) == 1 and orc.bands[0].delays.size == 886
    plan = eng.get_search_plans()[0]
    assert np.array_equal(plan.warmup_samples, orc.bands[0].delays)
    rows = np.arange(orc.bands[0].delays.size)
    err, full = check_rows(eng, orc, stream, 0, orc.bands[0], rows)
    print(f"\n1024 ch: plane rows max |err|/rms {err:.2e} over {rows.size} rows")
    assert err < ROW_RTOL, err
    eng.close()
    ref = orc.search(stream, GULP, masks, rows={0: rows}, data={0: full})
    del full
    n, missing, extra, bad = compare(cands, ref, bc.detect_thresh, snr_rtol=SNR_RTOL)
    print(f"1024 ch: {n} oracle candidates, {cands.size} GPU candidates")
    assert n > 100
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])
    # every injected pulse is found near its DM
    dms = plan.dm_grid
    for p in pulses:
        near = np.abs(dms[cands["dm_idx"]] - p.dm) < 5.0
        assert np.any(near & (cands["snr"] > 7.0)), p


def config2_rfi():
    cfg = RfiConfig()
    cfg.moments.enabled = True
    cfg.iqrm.enabled = True
    cfg.kadane_channel.enabled = True
    cfg.kadane_spectrum.enabled = True
    cfg.zero_dm = ZeroDMMode.SUBTRACT
    return cfg


@pytest.fixture(scope="module")
def config2_stream():
    """Two 65536-sample gulps of the 4096-channel recipe (20 pulses at DM
    100-1900, widths 1-128, S/N 7-50; 5 % noisy channels, 20 bursts,
    3 dropouts) cleaned by the GPU cleaner with every strategy on."""
    fb = config2_gulp(seed=0x46524F5354, nsamps=2 * GULP)
    lay = BlockLayout(4096, GULP, DataType.UINT8, TSAMP, fb.fch1, fb.foff)
    wfs, masks = clean_gulps(config2_rfi(), lay, fb.data)
    pc = plan_for(lay, 0.0, 2000.0, 2)
    return fb, pc, wfs, masks


def test_4096_channels_eleven_planes_match_oracle_on_row_subsets(config2_stream):
    fb, pc, wfs, masks = config2_stream
    bc = BoxcarConfig(max_boxcar=256, wtsp=2.0, detect_thresh=6.0, max_candidates=1 << 22,
                      max_cands_per_dm=0)
    cands, eng = search_gulps(pc, bc, wfs, masks, capture_last=True)
    stream = np.concatenate(wfs, axis=1)
    orc = oracle_for(pc, bc)
    planes = eng.get_search_plans()
    assert len(planes) == 11 and len(orc.bands) == 11
    assert eng.widths() == [1, 2, 4, 8, 16, 32, 64, 128, 256]
    rng = np.random.default_rng(2000)
    subset, data, worst, nrows = {}, {}, 0.0, 0
    for p, band in enumerate(orc.bands):
        assert (planes[p].chan_begin, planes[p].chan_end) == (band.a, band.b)
        assert np.array_equal(planes[p].warmup_samples, band.delays)
        nd = band.delays.size
        rows = set(int(r) for r in rng.choice(nd, size=4, replace=False))
        for pulse in fb.pulses[p % 5::5]:
            rows.add(int(np.argmin(np.abs(band.dm - pulse.dm))))
        key = (planes[p].subband_level, planes[p].subband_idx)
        hit = np.unique(on_rows(cands, key, np.arange(nd))["dm_idx"])
        if hit.size:
            rows.update(int(r) for r in rng.choice(hit, size=min(4, hit.size), replace=False))
        rows = np.array(sorted(rows), np.int64)
        subset[p] = rows
        err, data[p] = check_rows(eng, orc, stream, p, orc.bands[p], rows)
        worst = max(worst, err)
        nrows += rows.size
    print(f"\n4096 ch: plane rows max |err|/rms {worst:.2e} over {nrows} rows of 11 planes")
    assert worst < ROW_RTOL, worst
    eng.close()
    ref = orc.search(stream, GULP, masks, rows=subset, data=data)
    mine = np.concatenate([on_rows(cands, (planes[p].subband_level, planes[p].subband_idx), r)
                           for p, r in subset.items()])
    n, missing, extra, bad = compare(mine, ref, bc.detect_thresh, snr_rtol=SNR_RTOL)
    widths = sorted(set(int(c["width"]) for c in ref if c["snr"] > bc.detect_thresh + 0.02))
    print(f"4096 ch: {n} oracle candidates on the subset, widths {widths}")
    assert n > 50 and max(widths) >= 64
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])


def test_4096_channels_fp16_storage_keeps_the_fp32_list_above_7(config2_stream):
    """The FP16-storage engine on the same cleaned gulps recovers the FP32
    engine's detections above S/N 7: the same plane, DM, width and peak
    sample with S/N within 1e-2, or (a near tie of the two precisions inside
    one run) the same run peaking at another sample with S/N within 1e-2.
    Nothing is missing on either side except runs that split or merge where
    they dip through the detection threshold (at most 1 in 1000)."""
    from frost_b200.search import candidate_list_diff
    _, pc, wfs, masks = config2_stream
    kw = dict(max_boxcar=256, wtsp=2.0, detect_thresh=6.0, max_candidates=1 << 22, max_cands_per_dm=0)
    c32, e32 = search_gulps(pc, BoxcarConfig(**kw), wfs, masks)
    e32.close()
    c16, e16 = search_gulps(pc, BoxcarConfig(storage=Storage.FP16, **kw), wfs, masks)
    e16.close()
    d = candidate_list_diff(c32, c16, 7.0)
    print("\nfp16 vs fp32 above S/N 7:", d)
    assert d["n_ref"] > 1000
    assert d["max_snr_rel_err"] <= FP16_SNR_RTOL, d
    assert d["only_ref"] + d["only_other"] <= d["n_ref"] // 1000, d
    assert d["moved"] <= d["n_ref"] // 200, d
