"""GPU parity of the streaming FDMT + boxcar search against the FP64 oracle
(oracle/fdmt_oracle.c): DM-time planes within 1e-5 of each row's RMS (FP32
storage), candidate plane/DM/width/peak indices identical and S/N within
1e-3 for every peak clear of the threshold; FP16 storage recovers the same
candidates above S/N 7 with its S/N error stated; noise S/N is unit in every
plane; tiling, masks, drain and the peak modes keep the same answers."""

import numpy as np
import pytest

from frost_b200.config import BoxcarConfig, PeakMode, Storage
from frost_b200.dedisp import band_edges, generate_dm_list
from oracle.fdmt import Oracle
from tests.search_cases import compare, make_stream, plan_config, run_engine, same_detections

pytestmark = pytest.mark.gpu


def oracle_for(pc, bc):
    f_min, f_max = band_edges(pc)
    return Oracle(pc.nchans, f_min, f_max, pc.dt, generate_dm_list(pc), pc.subband_depth,
                  bc.max_boxcar, bc.wtsp, bc.use_trapezoid, bc.detect_thresh, int(bc.peak_mode),
                  bc.skip_cold_prefix)


PULSES = ((1500, 20.0, 3.0, 1.2), (5000, 45.0, 8.0, 0.5), (9300, 5.0, 1.0, 2.5),
          (8190, 33.0, 4.0, 0.8))  # the last straddles the gulp boundary at 8192


@pytest.mark.parametrize("depth", [0, 2])
def test_planes_and_candidates_match_oracle(depth):
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=depth)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    stream = make_stream(pc, 3, seed=7 + depth, pulses=PULSES)
    eng = FDMTBoxcar(pc, bc)
    eng.capture_planes(True)
    orc = oracle_for(pc, bc)
    gulp = pc.block_nsamps
    # planes of the last gulp vs the oracle's rows over the whole stream
    cands = run_engine(eng, stream, gulp, drain=False)
    planes = eng.get_search_plans()
    assert len(planes) == (1 if depth == 0 else 11)
    for p, band in enumerate(orc.bands):
        assert (planes[p].chan_begin, planes[p].chan_end) == (band.a, band.b)
        assert np.array_equal(planes[p].warmup_samples, band.delays)
        rows = orc.dedisperse(stream, band)[:, -gulp:]
        mine = eng.plane_data(p, gulp)
        rms = np.sqrt(np.mean(rows ** 2, axis=1, keepdims=True)) + 1e-12
        err = np.max(np.abs(mine - rows) / rms)
        assert err < 1e-5, (p, err)
    cands = np.concatenate([cands, eng.drain().candidates])
    ref = orc.search(stream, gulp, [np.ones(pc.nchans, np.uint8)] * 3)
    n, missing, extra, bad = compare(cands, ref, bc.detect_thresh)
    assert n > 10
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])


def test_tiles_and_peak_modes_match():
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    stream = make_stream(pc, 2, seed=11, pulses=PULSES)
    for mode in (PeakMode.PER_WIDTH, PeakMode.ACROSS_WIDTHS, PeakMode.ALL):
        bc = BoxcarConfig(max_boxcar=16, detect_thresh=7.0, peak_mode=mode, use_trapezoid=True)
        whole = run_engine(FDMTBoxcar(pc, bc), stream, pc.block_nsamps)
        tiled = run_engine(FDMTBoxcar(pc, bc, tile_nsamps=4096), stream, pc.block_nsamps)
        assert np.array_equal(whole, tiled), mode
        ref = oracle_for(pc, bc).search(stream, pc.block_nsamps, [np.ones(pc.nchans, np.uint8)] * 2)
        n, missing, extra, bad = compare(whole, ref, bc.detect_thresh)
        assert n > 0 and not missing and not extra and not bad, (mode, missing[:3], extra[:3], bad[:3])


def test_changing_masks_use_or_variance():
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    stream = make_stream(pc, 3, seed=5, pulses=PULSES)
    rng = np.random.default_rng(3)
    masks = [(rng.random(pc.nchans) > p).astype(np.uint8) for p in (0.0, 0.2, 0.2)]
    masks[2][:8] = 0
    masked = stream.copy()
    for g, m in enumerate(masks):
        masked[:, g * pc.block_nsamps:(g + 1) * pc.block_nsamps] *= m[:, None]
    cands = run_engine(FDMTBoxcar(pc, bc), stream, pc.block_nsamps, masks=masks)
    ref = oracle_for(pc, bc).search(masked, pc.block_nsamps, masks)
    n, missing, extra, bad = compare(cands, ref, bc.detect_thresh)
    assert n > 0 and not missing and not extra and not bad, (missing[:3], extra[:3], bad[:3])


def test_fp16_storage_recovers_candidates_above_7():
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2)
    bc32 = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    bc16 = BoxcarConfig(max_boxcar=16, detect_thresh=6.0, storage=Storage.FP16)
    stream = make_stream(pc, 2, seed=21, pulses=PULSES)
    e32, e16 = FDMTBoxcar(pc, bc32), FDMTBoxcar(pc, bc16)
    e16.capture_planes(True)
    c32 = run_engine(e32, stream, pc.block_nsamps)
    c16 = run_engine(e16, stream, pc.block_nsamps)
    orc = oracle_for(pc, bc32)
    worst = 0.0
    for p, band in enumerate(orc.bands):
        rows = orc.dedisperse(stream, band)[:, -pc.block_nsamps:]
        rms = np.sqrt(np.mean(rows ** 2, axis=1, keepdims=True)) + 1e-12
        worst = max(worst, float(np.max(np.abs(e16.plane_data(p, pc.block_nsamps) - rows) / rms)))
    # FP16 keeps 11 significant bits: element error vs the FP64 oracle,
    # relative to each row's RMS, stays well under 1e-2 (measured ~5e-3).
    assert worst < 1e-2, worst
    print(f"fp16 plane max error / row RMS: {worst:.3e}")
    # Same list above S/N 7: every FP32 detection (plane, DM, width) has an
    # FP16 detection whose peak lies in the FP32 run (a near-tie inside a run
    # may move the argmax by a sample), and vice versa, except detections
    # whose S/N is within the FP16 error of 7.
    def runs(cs):
        out = {}
        for c in cs:
            if c["snr"] >= 7.0:
                k = (int(c["subband_level"]), int(c["subband_idx"]), int(c["dm_idx"]), int(c["filter_idx"]))
                out.setdefault(k, []).append((int(c["begin_sample"]), int(c["end_sample"]),
                                              int(c["peak_sample"]), float(c["snr"])))
        return out
    r32, r16 = runs(c32), runs(c16)

    def unmatched(a, b):
        bad, errs = [], []
        for k, lst in a.items():
            for beg, end, pk, snr in lst:
                hit = [x for x in b.get(k, []) if beg <= x[2] <= end or x[0] <= pk <= x[1]]
                if not hit:
                    if abs(snr - 7.0) > 0.05:
                        bad.append((k, pk, snr))
                else:
                    errs.append(abs(hit[0][3] - snr) / snr)
        return bad, errs
    bad32, errs = unmatched(r32, r16)
    bad16, _ = unmatched(r16, r32)
    assert not bad32 and not bad16, (bad32[:5], bad16[:5])
    exact = sum(1 for k, l in r32.items() for x in l if any(y[2] == x[2] for y in r16.get(k, [])))
    total = sum(len(l) for l in r32.values())
    print(f"fp16 vs fp32 above 7: {total} detections, {exact} identical peaks, "
          f"max S/N error {max(errs):.2e}")
    assert max(errs) < 1e-2


def test_unit_noise_snr_in_every_plane():
    """calibration_test.cpp:159-168 on the GPU engine: S/N of pure noise has
    sigma 1 +- 0.15 per plane and width (all-sample peak mode, threshold -inf
    equivalent via a low threshold on a short stream)."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2, gulp=8192)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=-1e30, peak_mode=PeakMode.ALL,
                      max_candidates=1 << 26, max_cands_per_dm=0)
    stream = make_stream(pc, 1, seed=0xCA11B)
    eng = FDMTBoxcar(pc, bc)
    res = eng.execute(stream)
    c = res.candidates
    assert not res.overflowed()
    for lvl, idx in {(int(a), int(b)) for a, b in zip(c["subband_level"], c["subband_idx"])}:
        for fi in np.unique(c["filter_idx"]):
            s = c["snr"][(c["subband_level"] == lvl) & (c["subband_idx"] == idx) & (c["filter_idx"] == fi)]
            assert abs(float(np.mean(s))) < 0.15 and abs(float(np.std(s)) - 1.0) < 0.15, (lvl, idx, fi)


def test_variance_grid_matches_oracle_and_errors():
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2)
    bc = BoxcarConfig(max_boxcar=16, use_trapezoid=True)
    eng = FDMTBoxcar(pc, bc)
    orc = oracle_for(pc, bc)
    mask = (np.arange(pc.nchans) % 3 != 0).astype(np.uint8)
    for p, band in enumerate(orc.bands):
        for W in (1, 4, 16):
            assert np.allclose(eng.get_subband_variance_grid(p, W, mask), orc.variance(band, mask, W),
                               rtol=1e-12)
    with pytest.raises(ValueError):
        FDMTBoxcar(plan_config(gulp=128), bc)  # gulp must exceed dt_max + boxcar_max
    with pytest.raises(ValueError):
        eng.execute(np.zeros((pc.nchans, pc.block_nsamps + 1), np.float32))
    info = eng.info()
    assert info["nplanes"] == 11 and info["dt_max"] > 0


def test_precision_variant_trapezoid_fifty_pulses_near_threshold():
    """The precision variant at test scale: trapezoid filters, fp16 planes
    with float accumulation, FP64 variances, 50 pulses at S/N 6-12. Every
    DM-time plane's error against the FP64 oracle is reported (fp32 and
    fp16), and the fp16 candidate list above S/N 7 equals the fp32 one
    (up to detections within the stated fp16 S/N error of 7)."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(nchans=128, gulp=8192, depth=2, dm_max=80.0)
    rng = np.random.default_rng(404)
    C = pc.nchans
    pulses = []
    for _ in range(50):
        w = float(rng.uniform(1.0, 16.0))
        snr = float(rng.uniform(6.0, 12.0))
        pulses.append((float(rng.uniform(2500, 3 * pc.block_nsamps - 200)), float(rng.uniform(2.0, 80.0)),
                       w, snr / np.sqrt(C * max(1.0, 1.064 * w))))
    stream = make_stream(pc, 3, seed=404, pulses=pulses)
    kw = dict(max_boxcar=32, detect_thresh=6.0, use_trapezoid=True)
    e32 = FDMTBoxcar(pc, BoxcarConfig(**kw))
    e16 = FDMTBoxcar(pc, BoxcarConfig(storage=Storage.FP16, **kw))
    e32.capture_planes(True)
    e16.capture_planes(True)
    c32 = run_engine(e32, stream, pc.block_nsamps)
    c16 = run_engine(e16, stream, pc.block_nsamps)
    orc = oracle_for(pc, BoxcarConfig(**kw))
    print("\nplane  fp32 max|err|/rms  fp16 max|err|/rms  fp16 rms(err)/rms")
    w32 = w16 = 0.0
    for p, band in enumerate(orc.bands):
        rows = orc.dedisperse(stream, band)[:, -pc.block_nsamps:]
        rms = np.sqrt(np.mean(rows ** 2, axis=1, keepdims=True)) + 1e-12
        d32 = np.abs(e32.plane_data(p, pc.block_nsamps) - rows) / rms
        d16 = np.abs(e16.plane_data(p, pc.block_nsamps) - rows) / rms
        print(f"{p:5d}  {d32.max():17.2e}  {d16.max():17.2e}  {np.sqrt(np.mean(d16 ** 2)):17.2e}")
        w32, w16 = max(w32, float(d32.max())), max(w16, float(d16.max()))
    assert w32 < 1e-5 and w16 < 1e-2, (w32, w16)
    ref = orc.search(stream, pc.block_nsamps, [np.ones(C, np.uint8)] * 3)
    n, missing, extra, bad = compare(c32, ref, 6.0)
    assert n > 20 and not missing and not extra and not bad, (missing[:3], extra[:3], bad[:3])

    def above7(cs):
        return {(int(c["subband_level"]), int(c["subband_idx"]), int(c["dm_idx"]), int(c["filter_idx"]),
                 int(c["peak_sample"])): float(c["snr"]) for c in cs if c["snr"] >= 7.0}
    a32, a16 = above7(c32), above7(c16)
    errs = [abs(a16[k] - v) / v for k, v in a32.items() if k in a16]
    tol = max(errs) if errs else 0.0
    only32 = [(k, v) for k, v in a32.items() if k not in a16 and abs(v - 7.0) > 7.0 * max(tol, 1e-3) * 2]
    only16 = [(k, v) for k, v in a16.items() if k not in a32 and abs(v - 7.0) > 7.0 * max(tol, 1e-3) * 2]
    print(f"above S/N 7: fp32 {len(a32)}, fp16 {len(a16)}, shared {len(errs)}, max S/N error {tol:.2e}")
    assert tol < 1e-2
    # a peak may move by a sample inside its run (a near tie); such pairs
    # share their run and are not counted as missing
    def moved(k, other):
        return any(k2[:4] == k[:4] and abs(k2[4] - k[4]) <= 2 for k2 in other)
    assert not [x for x in only32 if not moved(x[0], a16)], only32[:5]
    assert not [x for x in only16 if not moved(x[0], a32)], only16[:5]


def test_graph_replay_matches_direct_launches():
    """The per-gulp launch sequence captured once as a CUDA graph and
    replayed gives the candidates of direct launches, across mask changes
    (the OR-mask window), a short last gulp (a new capture) and drain."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2, gulp=8192)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0, storage=Storage.FP16)
    stream = make_stream(pc, 4, seed=77, pulses=PULSES)
    rng = np.random.default_rng(8)
    masks = [np.ones(pc.nchans, np.uint8)] + [(rng.random(pc.nchans) > 0.1).astype(np.uint8) for _ in range(3)]
    outs = []
    for graphs in (True, False):
        eng = FDMTBoxcar(pc, bc)
        eng.use_graphs(graphs)
        got = []
        for g in range(4):
            n = pc.block_nsamps if g < 3 else pc.block_nsamps - 1000
            wf = np.ascontiguousarray(stream[:, g * pc.block_nsamps:g * pc.block_nsamps + n] *
                                      masks[g][:, None].astype(np.float32))
            got.append(eng.execute(wf, masks[g]).candidates.copy())
        got.append(eng.drain().candidates.copy())
        outs.append(np.concatenate(got))
    assert outs[0].size > 0
    assert np.array_equal(outs[0], outs[1])


def test_autotune_keeps_results_and_caches_choice():
    """The autotuner measures the launch shapes, applies one, restarts the
    stream, caches the choice for the geometry, and the tuned engine finds
    what the default one finds (fused and single-level schedules give the
    same bits with float planes)."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    stream = make_stream(pc, 2, seed=91, pulses=PULSES)
    ref = run_engine(FDMTBoxcar(pc, bc), stream, pc.block_nsamps)
    tuned = FDMTBoxcar(pc, bc)
    t1 = tuned.autotune()
    assert t1["tiles_per_cta"] in (4, 8, 16, 32, 64, 128) and t1["ms"] > 0 and not t1["cached"]
    assert t1 == {**tuned.launch_shape(), "ms": t1["ms"], "cached": False}
    got = run_engine(tuned, stream, pc.block_nsamps)
    if t1["search_chunk"] == 4096:
        assert np.array_equal(got, ref)
    else:
        assert same_detections(got, ref, bc.detect_thresh)
    again = FDMTBoxcar(pc, bc).autotune()
    assert again["cached"] and again["fused"] == t1["fused"] and again["tiles_per_cta"] == t1["tiles_per_cta"]


@pytest.mark.parametrize("peak_mode", [PeakMode.PER_WIDTH, PeakMode.ACROSS_WIDTHS, PeakMode.ALL])
def test_every_launch_shape_gives_the_same_candidates(peak_mode):
    """Launch shapes (fused steps or single levels, tiles per CTA, bulk-copy
    stages) change how the work is cut, not the arithmetic: every shape with
    the same search chunk reports identical candidates, trapezoid and cold
    prefix included, with float planes and with fp16 planes (a fused step
    rounds its middle level as a stored one would be); the two search
    chunks agree within the S/N rounding of their prefix origins."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    stream = make_stream(pc, 3, seed=93, pulses=PULSES)
    for storage, shapes in ((Storage.FP32, [(False, 4, 0, 4096), (True, 8, 2, 2048), (True, 32, 3, 2048),
                                            (True, 16, 0, 4096), (False, 16, 0, 2048)]),
                            (Storage.FP16, [(True, 16, 0, 4096), (True, 4, 2, 2048), (True, 32, 4, 2048),
                                            (True, 8, 3, 4096), (False, 4, 0, 4096), (False, 16, 0, 2048)])):
        bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0, use_trapezoid=True, peak_mode=peak_mode,
                          storage=storage)
        ref = {}
        for fused, tpc, stages, chunk in shapes:
            eng = FDMTBoxcar(pc, bc)
            eng.set_launch_shape(fused, tpc, stages, chunk)
            assert eng.launch_shape() == {"fused": fused, "tiles_per_cta": tpc, "stages": stages,
                                          "search_chunk": chunk}
            got = run_engine(eng, stream, pc.block_nsamps)
            assert got.size > 0
            if chunk in ref:
                assert np.array_equal(got, ref[chunk]), (storage, fused, tpc, stages, chunk)
            else:
                ref[chunk] = got
        assert same_detections(ref[2048], ref[4096], bc.detect_thresh), storage
    with pytest.raises(ValueError):
        FDMTBoxcar(pc, BoxcarConfig(max_boxcar=16)).set_launch_shape(True, 16, 4, 1024)


@pytest.mark.parametrize("storage", [Storage.FP32, Storage.FP16])
def test_residency_caps_keep_the_candidates(storage):
    """A residency cap (level and search kernels at a few CTAs per SM, each
    looping over work items) changes which CTA does a row, not the
    arithmetic: the candidates and the last gulp's planes are bit-identical
    to the uncapped launches, for single and fused level steps."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    stream = make_stream(pc, 3, seed=95, pulses=PULSES)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0, storage=storage)
    for fused in (True, False):
        outs, planes = [], []
        for cap in (0, 1, 3):
            eng = FDMTBoxcar(pc, bc)
            eng.set_launch_shape(fused, 4, 2 if fused else 0, 4096)
            eng.set_residency(cap)
            assert eng.residency() == cap
            eng.capture_planes(True)
            outs.append(run_engine(eng, stream, pc.block_nsamps, drain=False))
            planes.append([eng.plane_data(p, pc.block_nsamps) for p in range(len(eng.get_search_plans()))])
        assert outs[0].size > 0
        for k in (1, 2):
            assert np.array_equal(outs[k], outs[0]), (fused, k)
            assert all(np.array_equal(a, b) for a, b in zip(planes[k], planes[0])), (fused, k)
    with pytest.raises(ValueError):
        FDMTBoxcar(pc, bc).set_residency(-1)


@pytest.mark.parametrize("storage", [Storage.FP32, Storage.FP16])
def test_fused_level_search_steps_are_bit_identical(storage):
    """A single level step into a searched level fused with its search (the
    search kernel computes, writes and searches each searched row; the level
    kernel computes only the rows no plane searches) gives the candidates and
    planes of the separate level and search launches bit for bit, over
    several gulps (the next levels and gulps read the fused rows), for single
    and two-level schedules and both search chunks."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=2, gulp=8192)
    stream = make_stream(pc, 3, seed=131, pulses=PULSES)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0, storage=storage)
    for fused, chunk in ((True, 4096), (False, 4096), (True, 2048)):
        outs, planes = [], []
        for mode in (0, 1, 2):  # off; one or two chunks staged at once
            eng = FDMTBoxcar(pc, bc)
            eng.set_launch_shape(fused, 4, 2 if fused else 0, chunk)
            eng.set_fused_search(mode)
            assert eng.fused_search() == mode
            eng.capture_planes(True)
            outs.append(np.concatenate([run_engine(eng, stream, pc.block_nsamps, drain=False),
                                        eng.drain().candidates]))
            planes.append([eng.plane_data(p, pc.block_nsamps) for p in range(len(eng.get_search_plans()))])
        assert outs[0].size > 0
        for k in (1, 2):
            assert np.array_equal(outs[k], outs[0]), (fused, chunk, k)
            assert all(np.array_equal(a, b) for a, b in zip(planes[k], planes[0])), (fused, chunk, k)
    with pytest.raises(ValueError):
        FDMTBoxcar(pc, bc).set_fused_search(3)


def test_uneven_widths_match_oracle():
    """Widths that are not powers of two (wtsp 1.5: 1, 2, 3, 5, ..., 93)
    take the table-driven steady-state tests (window starts straddling two
    4-sample groups, per-thread bounds for the widest): identical candidate
    indices and S/N within 1e-3 of the oracle."""
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    bc = BoxcarConfig(max_boxcar=100, wtsp=1.5, detect_thresh=6.0)
    stream = make_stream(pc, 3, seed=97, pulses=PULSES)
    eng = FDMTBoxcar(pc, bc)
    cands = run_engine(eng, stream, pc.block_nsamps)
    widths = sorted(set(int(w) for w in cands["width"]))
    assert any(w % 2 == 1 and w > 2 for w in widths), widths
    ref = oracle_for(pc, bc).search(stream, pc.block_nsamps, [np.ones(pc.nchans, np.uint8)] * 3)
    n, missing, extra, bad = compare(cands, ref, bc.detect_thresh)
    assert n > 10
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])


def test_device_waterfall_written_on_a_caller_stream():
    """A waterfall written on the caller's stream (an async copy from pinned
    memory behind other work on that stream) and passed with that stream is
    read after the writes: the candidates equal the host-input run. The
    null stream is refused for device input, as frost refuses it
    (lib/cuda/device_rfi_detail.cuh:77-83)."""
    import ctypes as C

    import torch

    from frost_b200._lib import lib
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    stream = make_stream(pc, 2, seed=31, pulses=PULSES)
    gulp = pc.block_nsamps
    ref = run_engine(FDMTBoxcar(pc, bc), stream, gulp)
    eng = FDMTBoxcar(pc, bc)
    s = torch.cuda.Stream()
    wf = torch.zeros((pc.nchans, gulp), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    junk = torch.empty((4096, 4096), device="cuda")
    out = []
    for g in range(2):
        host = torch.from_numpy(np.ascontiguousarray(stream[:, g * gulp:(g + 1) * gulp])).pin_memory()
        with torch.cuda.stream(s):
            for _ in range(8):           # other work queued ahead of the copy
                junk.normal_()
                junk = junk @ junk
            wf.copy_(host, non_blocking=True)
        out.append(eng.execute_device(wf.data_ptr(), gulp, None, stream=s.cuda_stream).candidates.copy())
    out.append(eng.drain().candidates.copy())
    assert np.array_equal(np.concatenate(out), ref)
    rc = lib().frost_search_execute(eng._h, C.cast(C.c_void_p(wf.data_ptr()), C.POINTER(C.c_float)),
                                    gulp, 1, None, None)
    assert rc == -1 and "null stream" in lib().frost_last_error().decode()


def test_bounded_wait_timeout_is_reported_and_the_stream_restarts():
    """The level and search kernels' bounded waits on their bulk copies:
    with the first-wait bound at zero every kernel gives up at once, lets
    its copies in flight land (waiting with the default bound) and sets the
    error flag, so execute fails with FROST_ERR_TIMEOUT instead of hanging
    (frost maps device failures to exceptions, lib/cuda/gpu_utils.cuh:13-20).
    After the default bound is restored and the stream restarted, the engine
    gives a fresh engine's candidates, graphs on or off."""
    from frost_b200._lib import FrostError
    from frost_b200.search import FDMTBoxcar
    pc = plan_config(depth=1, gulp=8192)
    bc = BoxcarConfig(max_boxcar=16, detect_thresh=6.0)
    stream = make_stream(pc, 2, seed=33, pulses=PULSES)
    gulp = pc.block_nsamps
    ref = run_engine(FDMTBoxcar(pc, bc), stream, gulp)
    assert ref.size > 0
    for graphs in (True, False):
        eng = FDMTBoxcar(pc, bc)
        eng.use_graphs(graphs)
        eng.set_wait_limit(0)
        with pytest.raises(FrostError) as e:
            eng.execute(np.ascontiguousarray(stream[:, :gulp]))
        assert e.value.code == -4 and "bounded wait" in str(e.value)
        eng.set_wait_limit(-1)
        eng.restart()
        assert np.array_equal(run_engine(eng, stream, gulp), ref), graphs
