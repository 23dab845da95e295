"""Batched multi-beam search: beams of different channel counts (1024,
2048, 4096), sample types, gulp lengths, DM ranges and plane counts (1, 4,
11) searched together, their level steps and searches run as single
launches over all beams, give for every gulp and the drain exactly the
candidates each beam gives alone through the single-beam pipeline, with the
rounds replayed from a CUDA graph and launched directly."""

import numpy as np
import pytest

from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig
from frost_b200.synth import make_filterbank

pytestmark = pytest.mark.gpu

BEAMS = [  # channels, dtype, gulp, DM max, sub-band depth (1 / 4 / 11 planes)
    (1024, "uint8", 32768, 500.0, 0),
    (2048, "float32", 32768, 800.0, 1),
    (4096, "uint8", 65536, 1000.0, 2),
    (1024, "float32", 65536, 2500.0, 2),
    (2048, "uint8", 32768, 600.0, 2),
]


def _beam(i):
    from frost_b200.pipeline import plan_for
    C, dt, gulp, dm_max, depth = BEAMS[i]
    foff = -336.0 / C
    fb = make_filterbank(C, gulp * 2, 1536.0 + foff / 2, foff, 64e-6, 700 + i, dtype=dt, n_pulses=3,
                         dm_range=(50.0, dm_max * 0.8), snr_range=(12.0, 30.0), width_range=(1.0, 32.0),
                         rfi_channel_fraction=0.02, n_bursts=1)
    layout = BlockLayout(C, gulp, DataType.UINT8 if dt == "uint8" else DataType.FLOAT32, 64e-6,
                         1536.0 + foff / 2, foff)
    return fb.data, layout, plan_for(layout, 0.0, dm_max, subband_depth=depth)


@pytest.mark.parametrize("graphs", [True, False])
def test_batched_beams_match_each_beam_alone(graphs):
    from frost_b200.batch import BeamBatch
    from frost_b200.pipeline import GulpPipeline
    bc = BoxcarConfig(max_boxcar=64, detect_thresh=7.0, tile_nsamps=32768)
    beams = [_beam(i) for i in range(len(BEAMS))]
    alone = []
    for data, layout, plan in beams:
        p = GulpPipeline(RfiConfig(), layout, 1.0, plan, bc)
        p.search.autotune()  # the launch shape the batch gives each beam (cached per geometry)
        g = layout.max_nsamps
        alone.append([p.execute(data[k * g:(k + 1) * g], g).candidates for k in range(2)] + [p.flush().candidates])
    batch = BeamBatch()
    batch.use_graph(graphs)
    for _, layout, plan in beams:
        batch.add_beam(RfiConfig(), layout, 1.0, plan, bc)
    for k in range(2):
        got = batch.execute([d[k * lay.max_nsamps:(k + 1) * lay.max_nsamps] for d, lay, _ in beams])
        for i in range(len(beams)):
            assert np.array_equal(got[i], alone[i][k]), (i, k)
    for i in range(len(beams)):
        assert np.array_equal(batch.drain(i), alone[i][2]), i
    assert sum(len(c) for per in alone for c in per) > 0
    st = batch.stats()
    assert st["executes"] == 2 and st["beams"] == len(BEAMS)
    # one level launch and one search launch per round cover several beams
    assert st["merged_level_launches"] < st["rounds"] * len(BEAMS)
    if graphs:
        assert st["graph_replays"] == 1
    batch.close()
