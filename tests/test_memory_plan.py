"""The device memory planner (check_memory, lib/pipeline/memory.cpp:294-508;
MemoryEstimate, include/frost/pipeline/memory.hpp) on the host: component
estimates that add up and grow with the gulp, DM range and storage; the
check that fits a default gulp into 90 % of the budget (largest multiple of
1024 samples, never below max_delay + boxcar_max), refuses an explicit one
naming the largest gulp that fits, caps the budget by a memory limit, and
enforces nothing when availability is unknown. No GPU: the estimates come
from the plans alone."""

import pytest

from frost_b200._lib import FrostError
from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig, Storage
from frost_b200.memory import check_memory, estimate_memory
from frost_b200.pipeline import plan_for

GIB = 1 << 30


def _setup(gulp=65536, nchans=1024, dm_max=500.0, storage=Storage.FP16, depth=1):
    layout = BlockLayout(nchans, gulp, DataType.UINT8, 64e-6, 1500.0, -0.29296875)
    plan = plan_for(layout, 0.0, dm_max, subband_depth=depth)
    bc = BoxcarConfig(max_boxcar=64, detect_thresh=6.0, storage=storage)
    return RfiConfig(), layout, plan, bc


def test_estimate_components_add_up_and_grow():
    rfi, layout, plan, bc = _setup()
    e = estimate_memory(rfi, layout, 1.0, plan, bc)
    assert min(e.rfi_bytes, e.fdmt_bytes, e.search_bytes, e.transient_bytes) > 0 and e.postprocess_bytes == 0
    assert e.total_bytes == e.rfi_bytes + e.fdmt_bytes + e.search_bytes + e.postprocess_bytes + e.transient_bytes
    assert 0 < e.max_delay < layout.max_nsamps
    # the raw block and the float work / output waterfalls are in the RFI share
    assert e.rfi_bytes >= layout.max_nsamps * layout.nchans * (1 + 4 + 4)
    big = estimate_memory(*_setup(gulp=131072)[:2], 1.0, *_setup(gulp=131072)[2:])
    assert big.rfi_bytes > e.rfi_bytes and big.fdmt_bytes > e.fdmt_bytes
    more_dm = estimate_memory(*_setup(dm_max=900.0)[:2], 1.0, *_setup(dm_max=900.0)[2:])
    assert more_dm.fdmt_bytes > e.fdmt_bytes and more_dm.max_delay > e.max_delay
    fp32 = estimate_memory(*_setup(storage=Storage.FP32)[:2], 1.0, *_setup(storage=Storage.FP32)[2:])
    assert 1.9 * e.fdmt_bytes < fp32.fdmt_bytes < 2.1 * e.fdmt_bytes
    assert fp32.rfi_bytes == e.rfi_bytes


def test_postprocessor_is_charged_when_given():
    from frost_b200.postprocess import SearchConfig
    rfi, layout, plan, bc = _setup()
    pp = SearchConfig(max_candidates=1 << 16)
    e0 = estimate_memory(rfi, layout, 1.0, plan, bc)
    e1 = estimate_memory(rfi, layout, 1.0, plan, bc, post=pp)
    assert e1.postprocess_bytes > 0 and e1.total_bytes == e0.total_bytes + e1.postprocess_bytes


def test_check_fits_lowers_or_refuses():
    rfi, layout, plan, bc = _setup()
    need = estimate_memory(rfi, layout, 1.0, plan, bc).total_bytes
    ok = check_memory(rfi, layout, 1.0, plan, bc, available_bytes=2 * need)
    assert not ok.lowered and ok.gulp_used == ok.gulp_requested == 65536
    assert ok.requested_bytes == need and ok.available_bytes == 2 * need and ok.device_memory
    # a budget of 60 % of the request: the default gulp is lowered
    avail = int(need * 0.6)
    rfi, layout, plan, bc = _setup()
    low = check_memory(rfi, layout, 1.0, plan, bc, available_bytes=avail)
    assert low.lowered and low.gulp_used % 1024 == 0 and low.gulp_used < 65536
    assert layout.max_nsamps == plan.block_nsamps == low.gulp_used
    budget = avail - avail // 10
    assert low.estimate.total_bytes <= budget
    assert low.gulp_used > low.estimate.max_delay + bc.max_boxcar
    nxt = _setup(gulp=low.gulp_used + 1024)
    assert estimate_memory(nxt[0], nxt[1], 1.0, nxt[2], nxt[3]).total_bytes > budget  # the largest that fits
    # an explicit gulp is refused with the largest that fits
    rfi, layout, plan, bc = _setup()
    with pytest.raises(FrostError) as err:
        check_memory(rfi, layout, 1.0, plan, bc, gulp_is_default=False, available_bytes=avail)
    assert err.value.code == -2 and f"largest nsamps_gulp that fits is {low.gulp_used}" in str(err.value)
    assert layout.max_nsamps == 65536
    # nothing fits, not even the smallest valid gulp
    with pytest.raises(FrostError) as err:
        check_memory(rfi, layout, 1.0, plan, bc, available_bytes=64 << 20)
    assert "not even nsamps_gulp" in str(err.value)


def test_memory_limit_caps_the_budget_and_unknown_enforces_nothing():
    rfi, layout, plan, bc = _setup()
    need = estimate_memory(rfi, layout, 1.0, plan, bc).total_bytes
    capped = check_memory(rfi, layout, 1.0, plan, bc, available_bytes=64 * GIB, memory_limit_bytes=int(need * 0.6))
    assert capped.available_bytes == int(need * 0.6) and capped.lowered
    rfi, layout, plan, bc = _setup()
    limit_only = check_memory(rfi, layout, 1.0, plan, bc, available_bytes=0, memory_limit_bytes=4 * need)
    assert 0 < limit_only.available_bytes <= 4 * need
    assert not limit_only.lowered


def test_headline_beam_estimate():
    """4096 channels, DM 0-2000, 262144-sample gulps, 11 planes, fp16: about
    50 GB a beam (level buffers ~40 GB), which is what admits three such
    beams on one 180 GB B200."""
    layout = BlockLayout(4096, 262144, DataType.UINT8, 64e-6, 1535.958984375, -0.08203125)
    plan = plan_for(layout, 0.0, 2000.0, subband_depth=2)
    bc = BoxcarConfig(max_boxcar=256, detect_thresh=6.0, storage=Storage.FP16, max_candidates=1 << 20)
    e = estimate_memory(RfiConfig(), layout, 2.0, plan, bc)
    assert e.max_delay == 35088
    assert 40 * GIB < e.total_bytes < 56 * GIB and 30 * GIB < e.fdmt_bytes < 45 * GIB


def test_invalid_configurations_are_refused():
    rfi, layout, plan, bc = _setup()
    plan.block_nsamps = 32768
    with pytest.raises(ValueError):
        estimate_memory(rfi, layout, 1.0, plan, bc)
    rfi, layout, plan, bc = _setup(gulp=4096, dm_max=500.0)  # gulp below max_delay + boxcar_max
    with pytest.raises(ValueError):
        estimate_memory(rfi, layout, 1.0, plan, bc)
