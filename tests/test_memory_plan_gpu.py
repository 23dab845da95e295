"""The memory planner against real allocations: for pipelines of several
shapes (channels, DM range, depth, storage, autotuned or not), after
gulps have run, the estimate of the RFI cleaner and of the FDMT/search
engine is never below what they hold on the device and exceeds it by a few
percent at most (buffers sized by data counted at their largest; level
buffers under either schedule the autotuner may try)."""

import numpy as np
import pytest

from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig, Storage
from frost_b200.memory import estimate_memory
from frost_b200.synth import make_filterbank

pytestmark = pytest.mark.gpu

MIB = 1 << 20


@pytest.mark.parametrize("nchans,gulp,dm_max,depth,storage,tune", [
    (256, 8192, 80.0, 1, Storage.FP16, False),
    (256, 8192, 80.0, 2, Storage.FP32, True),
    (512, 16384, 150.0, 0, Storage.FP16, True),
])
def test_estimate_bounds_the_allocations(nchans, gulp, dm_max, depth, storage, tune):
    from frost_b200.pipeline import GulpPipeline, plan_for
    layout = BlockLayout(nchans, gulp, DataType.UINT8, 1e-3, 1500.0, -1.0)
    plan = plan_for(layout, 0.0, dm_max, subband_depth=depth)
    bc = BoxcarConfig(max_boxcar=32, detect_thresh=7.0, storage=storage)
    rfi = RfiConfig()
    e = estimate_memory(rfi, layout, 1.0, plan, bc)
    pipe = GulpPipeline(rfi, layout, 1.0, plan, bc)
    if tune:
        pipe.search.autotune()
    fb = make_filterbank(nchans, gulp * 2, 1500.0, -1.0, 1e-3, 5, n_pulses=3, dm_range=(5.0, dm_max / 2),
                         snr_range=(10.0, 20.0), rfi_channel_fraction=0.03, n_bursts=2)
    for g in range(2):
        pipe.execute(np.ascontiguousarray(fb.data[g * gulp:(g + 1) * gulp]), gulp)
    rfi_used = pipe.rfi.memory_usage()
    eng_used = pipe.search.info()["device_bytes"]
    assert rfi_used <= e.rfi_bytes <= 1.05 * rfi_used + 4 * MIB, (rfi_used, e.rfi_bytes)
    est = e.fdmt_bytes + e.search_bytes
    # untuned engines allocate the fused schedule only; the estimate also
    # covers the single-level one autotune may try
    assert eng_used <= est <= (1.1 if tune else 1.4) * eng_used + 4 * MIB, (eng_used, est)
