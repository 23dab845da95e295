"""The multi-beam server on one GPU: beams served together, with gulps queued
up front and taken by two worker slots, give exactly the candidates each beam
gives alone through the single-beam pipeline; admission refuses a beam that
would exceed the memory budget and takes it once another beam is removed;
latency statistics and searched beam-seconds add up."""

import numpy as np
import pytest

from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig
from frost_b200.synth import make_filterbank

pytestmark = pytest.mark.gpu

NCHANS, GULP, NGULPS, TSAMP = 256, 8192, 3, 1e-3


def _beam_stream(seed):
    fb = make_filterbank(NCHANS, GULP * NGULPS, 1500.0, -1.0, TSAMP, seed, n_pulses=6,
                         dm_range=(5.0, 60.0), snr_range=(10.0, 25.0), rfi_channel_fraction=0.03,
                         n_bursts=2)
    return fb.data


def _setup():
    from frost_b200.pipeline import plan_for
    layout = BlockLayout(NCHANS, GULP, DataType.UINT8, TSAMP, 1500.0, -1.0)
    plan = plan_for(layout, 0.0, 80.0, subband_depth=1)
    bc = BoxcarConfig(max_boxcar=32, detect_thresh=7.0)
    return RfiConfig(), layout, plan, bc


def _nread(g):
    return GULP if g < NGULPS - 1 else GULP - 1000  # a short last gulp


def test_served_beams_match_each_beam_alone():
    from frost_b200.pipeline import GulpPipeline
    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    streams = [_beam_stream(s) for s in (21, 22, 23)]
    alone = []
    for st in streams:
        p = GulpPipeline(rfi, layout, 1.0, plan, bc)
        p.search.autotune()  # the launch shape the server gives each beam (cached per geometry)
        per = [p.execute(st[g * GULP:(g + 1) * GULP], _nread(g)).candidates for g in range(NGULPS)]
        per.append(p.flush().candidates)
        alone.append(per)
    srv = BeamServer(slots=2)
    beams = [srv.add_beam(rfi, layout, 1.0, plan, bc) for _ in streams]
    tickets = [[srv.submit(b, st[g * GULP:(g + 1) * GULP], _nread(g)) for g in range(NGULPS)]
               for b, st in zip(beams, streams)]
    for i, b in enumerate(beams):
        for g, t in enumerate(tickets[i]):
            cands, latency = srv.wait(t)
            assert latency > 0
            assert np.array_equal(cands, alone[i][g]), (i, g)
        assert np.array_equal(srv.drain(b), alone[i][NGULPS]), i
    assert sum(len(c) for per in alone for c in per) > 0
    s = srv.stats()
    assert s.completed == 3 * NGULPS and s.beams == 3
    expect = 3 * sum(_nread(g) for g in range(NGULPS)) * TSAMP
    assert abs(s.beam_seconds - expect) < 1e-6 * expect
    assert 0 < s.p50_latency_s <= s.p99_latency_s <= s.max_latency_s
    assert s.wall_seconds > 0 and s.launches > 10 * s.completed
    srv.reset_stats()
    assert srv.stats().completed == 0 and srv.stats().launches == 0
    srv.close()


def test_device_resident_gulps_match_host_gulps():
    import torch

    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    st = _beam_stream(31)
    srv = BeamServer(slots=2)
    host_beam, dev_beam = srv.add_beam(rfi, layout, 1.0, plan, bc), srv.add_beam(rfi, layout, 1.0, plan, bc)
    dev = torch.from_numpy(st.reshape(-1)).cuda()
    gulp_bytes = GULP * NCHANS
    for g in range(NGULPS):
        th = srv.submit(host_beam, st[g * GULP:(g + 1) * GULP], _nread(g))
        td = srv.submit_ptr(dev_beam, dev.data_ptr() + g * gulp_bytes, gulp_bytes, _nread(g), on_device=True)
        a, _ = srv.wait(th)
        b, _ = srv.wait(td)
        assert np.array_equal(a, b), g
    assert np.array_equal(srv.drain(host_beam), srv.drain(dev_beam))
    srv.close()


def test_staged_host_gulps_match_unstaged():
    """Pinned host gulps uploaded into staging blocks when they are
    submitted, with every gulp queued at once (more gulps than blocks, so
    some are copied when processed), give the candidates of the same gulps
    uploaded when they are processed; the blocks are charged to the budget
    and given back."""
    import torch

    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    st = _beam_stream(41)
    pinned = torch.from_numpy(st.reshape(-1)).pin_memory()
    gulp_bytes = GULP * NCHANS
    srv = BeamServer(slots=2)
    plain, staged = srv.add_beam(rfi, layout, 1.0, plan, bc), srv.add_beam(rfi, layout, 1.0, plan, bc)
    before = srv.stats().device_bytes
    srv.set_staging(staged, 2)
    assert srv.stats().device_bytes == before + 2 * gulp_bytes
    order = [(g, GULP) for g in range(NGULPS)] + [(g, _nread(g)) for g in range(NGULPS)]
    tp = [srv.submit(plain, st[g * GULP:(g + 1) * GULP], n) for g, n in order]
    ts = [srv.submit_ptr(staged, pinned.data_ptr() + g * gulp_bytes, gulp_bytes, n, on_device=False)
          for g, n in order]
    total = 0
    for k in range(len(order)):
        a, _ = srv.wait(tp[k])
        b, _ = srv.wait(ts[k])
        assert np.array_equal(a, b), k
        total += len(a)
    assert total > 0
    assert np.array_equal(srv.drain(plain), srv.drain(staged))
    srv.set_staging(staged, 0)
    assert srv.stats().device_bytes == before
    srv.close()


def test_set_staging_while_another_thread_submits():
    """A thread that changes a beam's staging blocks (1, 2, 0, ...) while
    another thread keeps submitting pinned gulps to that beam: gulps that
    arrive while the beam is being reconfigured are uploaded when they are
    processed, and every gulp gives the candidates of an unstaged beam fed
    the same gulps."""
    import threading

    import torch

    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    st = _beam_stream(43)
    pinned = torch.from_numpy(st.reshape(-1)).pin_memory()
    gulp_bytes = GULP * NCHANS
    srv = BeamServer(slots=2)
    plain, staged = srv.add_beam(rfi, layout, 1.0, plan, bc), srv.add_beam(rfi, layout, 1.0, plan, bc)
    order = [g % NGULPS for g in range(12)]
    ref = [srv.wait(srv.submit(plain, st[g * GULP:(g + 1) * GULP], GULP))[0] for g in order]
    stop, errors, toggles = threading.Event(), [], [0]

    def toggler():
        while not stop.is_set():
            try:
                srv.set_staging(staged, (1, 2, 0)[toggles[0] % 3])
            except Exception as e:  # reported below
                errors.append(e)
                return
            toggles[0] += 1
    th = threading.Thread(target=toggler)
    th.start()
    got = []
    try:
        for i in range(0, len(order), 2):
            ts = [srv.submit_ptr(staged, pinned.data_ptr() + g * gulp_bytes, gulp_bytes, GULP, on_device=False)
                  for g in order[i:i + 2]]
            got += [srv.wait(t)[0] for t in ts]
    finally:
        stop.set()
        th.join()
    assert not errors, errors
    assert toggles[0] > 0
    assert sum(len(a) for a in ref) > 0
    for k, (a, b) in enumerate(zip(ref, got)):
        assert np.array_equal(a, b), k
    srv.set_staging(staged, 0)
    srv.close()


def test_admission_by_device_memory():
    from frost_b200._abi import ERR_OUT_OF_MEMORY
    from frost_b200._lib import FrostError
    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    probe = BeamServer(slots=1)
    probe.add_beam(rfi, layout, 1.0, plan, bc)
    need = probe.stats().device_bytes
    probe.close()
    assert need > 0
    srv = BeamServer(memory_budget=int(1.5 * need), slots=1)
    first = srv.add_beam(rfi, layout, 1.0, plan, bc)
    with pytest.raises(FrostError) as e:
        srv.add_beam(rfi, layout, 1.0, plan, bc)
    assert e.value.code == ERR_OUT_OF_MEMORY
    srv.remove_beam(first)
    second = srv.add_beam(rfi, layout, 1.0, plan, bc)
    assert srv.stats().beams == 1 and second != first
    srv.close()


def test_gulp_arriving_while_slots_are_busy_waits_for_a_slot_and_gives_its_solo_result():
    """Continuous batching: with both worker slots busy on two beams' gulps,
    a third beam's gulp that arrives meanwhile is queued, starts when a slot
    frees (its latency includes the wait) and gives exactly the candidates
    of that beam run alone; so do the first two."""
    import time

    from frost_b200.pipeline import GulpPipeline
    from frost_b200.serve import BeamServer
    rfi, layout, plan, bc = _setup()
    streams = [_beam_stream(s) for s in (61, 62, 63)]
    alone = []
    for st in streams:
        p = GulpPipeline(rfi, layout, 1.0, plan, bc)
        p.search.autotune()
        alone.append(p.execute(st[:GULP], GULP).candidates)
    srv = BeamServer(slots=2)
    ids = [srv.add_beam(rfi, layout, 1.0, plan, bc) for _ in streams]
    t_busy = [srv.submit(ids[k], streams[k][:GULP], GULP) for k in range(2)]
    time.sleep(0.002)  # the two gulps are on the device
    t_late = srv.submit(ids[2], streams[2][:GULP], GULP)
    lat = []
    for k, t in enumerate(t_busy + [t_late]):
        cands, l = srv.wait(t)
        lat.append(l)
        assert np.array_equal(cands, alone[k]), k
    assert sum(len(a) for a in alone) > 0
    # the late gulp waited for a slot: its latency exceeds the faster busy
    # gulp's service time less the head start it was given
    assert lat[2] > min(lat[0], lat[1]) - 0.002
    assert srv.stats().completed == 3
    srv.close()


UNEVEN = [  # channels, dtype, gulp, DM max, sub-band depth (1 / 4 / 11 planes)
    (1024, "uint8", 32768, 500.0, 0),
    (2048, "float32", 32768, 800.0, 1),
    (4096, "uint8", 32768, 500.0, 2),
    (1024, "float32", 65536, 2500.0, 2),
]


def _uneven(i):
    from frost_b200.config import BlockLayout, DataType
    from frost_b200.pipeline import plan_for
    C, dt, gulp, dm_max, depth = UNEVEN[i]
    foff = -336.0 / C
    fb = make_filterbank(C, gulp * 2, 1536.0 + foff / 2, foff, 64e-6, 500 + i, dtype=dt, n_pulses=2,
                         dm_range=(50.0, dm_max * 0.8), snr_range=(15.0, 30.0),
                         rfi_channel_fraction=0.02, n_bursts=1)
    layout = BlockLayout(C, gulp, DataType.UINT8 if dt == "uint8" else DataType.FLOAT32, 64e-6,
                         1536.0 + foff / 2, foff)
    plan = plan_for(layout, 0.0, dm_max, subband_depth=depth)
    return fb.data, layout, plan


def test_uneven_beams_served_together_match_each_alone():
    """Beams of different channel counts, sample types, gulp lengths, DM
    ranges and plane counts (1, 4, 11) served together on one GPU give the
    candidates each gives alone."""
    from frost_b200.pipeline import GulpPipeline
    from frost_b200.serve import BeamServer
    bc = BoxcarConfig(max_boxcar=64, detect_thresh=7.0)
    beams = [_uneven(i) for i in range(len(UNEVEN))]
    alone = []
    for data, layout, plan in beams:
        p = GulpPipeline(RfiConfig(), layout, 1.0, plan, bc)
        p.search.autotune()  # the launch shape the server gives each beam (cached per geometry)
        g = layout.max_nsamps
        alone.append([p.execute(data[k * g:(k + 1) * g], g).candidates for k in range(2)] +
                     [p.flush().candidates])
    srv = BeamServer(slots=3)
    ids = [srv.add_beam(RfiConfig(), layout, 1.0, plan, bc) for _, layout, plan in beams]
    tickets = [[srv.submit(b, data[k * layout.max_nsamps:(k + 1) * layout.max_nsamps], layout.max_nsamps)
                for k in range(2)] for b, (data, layout, _) in zip(ids, beams)]
    for i, b in enumerate(ids):
        for k, t in enumerate(tickets[i]):
            cands, _ = srv.wait(t)
            assert np.array_equal(cands, alone[i][k]), (i, k)
        assert np.array_equal(srv.drain(b), alone[i][2]), i
    assert sum(len(c) for per in alone for c in per) > 0
    srv.close()


def test_served_postprocessing_matches_pipeline_and_oracle():
    """A served beam with a post-processor gives per gulp the giants of the
    single-beam pipeline with post-processing, and both equal the CPU
    oracle's plan fed the same raw candidates (samples read, gulp rows and
    the engine's frontier, as Pipeline::publish passes them)."""
    from frost_b200.pipeline import GulpPipeline
    from frost_b200.postprocess import CandidatePostprocessLayout, SearchConfig
    from frost_b200.serve import BeamServer
    from oracle import postprocess as op
    from tests.postprocess_cases import same_giants
    rfi, layout, plan, bc = _setup()
    ppcfg = SearchConfig(boxcar_max=bc.max_boxcar, detect_thresh=bc.detect_thresh, max_candidates=bc.max_candidates)
    streams = [_beam_stream(s) for s in (31, 32)]
    srv = BeamServer(slots=2)
    beams = [srv.add_beam(rfi, layout, 1.0, plan, bc) for _ in streams]
    for b in beams:
        srv.set_postprocess(b, ppcfg)
    tickets = [[srv.submit(b, st[g * GULP:(g + 1) * GULP], _nread(g)) for g in range(NGULPS)]
               for b, st in zip(beams, streams)]
    total = 0
    for i, b in enumerate(beams):
        p = GulpPipeline(rfi, layout, 1.0, plan, bc, postprocess=ppcfg)
        p.search.autotune()
        orc = op.backend("oracle").plan(ppcfg, CandidatePostprocessLayout(layout.nchans, layout.tsamp, layout.df))
        for g, t in enumerate(tickets[i]):
            giants, _ = srv.wait_giants(t)
            res = p.execute(streams[i][g * GULP:(g + 1) * GULP], _nread(g))
            ref, _ = orc.execute(res.candidates, p.samples_read, _nread(g), False, p.search.get_candidate_frontier())
            assert same_giants(giants, p.postprocessed.candidates), (i, g)
            assert same_giants(giants, ref), (i, g)
            total += giants.size
        last = srv.drain_giants(b)
        res = p.flush()
        ref, pend = orc.execute(res.candidates, p.samples_read, _nread(NGULPS - 1), True,
                                p.search.get_candidate_frontier())
        assert same_giants(last, p.postprocessed.candidates) and same_giants(last, ref) and pend == 0
        total += last.size
    assert total > 0
