"""GPU parity of the RFI cleaner against the reference's own CPU cleaner
(strict IEEE build, oracle/_ref) and the committed golden digests.

The bar is bit-exact: channel masks, report counts and every float of the
normalized [channel][time] waterfall."""

import hashlib
import json
import os

import numpy as np
import pytest

from tests.rfi_cases import CASES, make_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rfi_cases.json")
COUNTS = ("nsamps", "chans_zapped", "chans_dead", "chans_moments", "chans_iqrm", "chans_grown",
          "chans_masked", "samps_broad", "samps_dropout", "samps_kadane", "samps_flagged",
          "cells_narrow", "cells_kadane_spectrum", "cells_kadane_channel", "fill_fallbacks",
          "calibration_reused")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def describe_diff(mine, theirs):
    d = np.abs(mine.astype(np.float64) - theirs.astype(np.float64))
    i = np.unravel_index(np.argmax(d), d.shape)
    return (f"{np.count_nonzero(mine.view(np.uint32) != theirs.view(np.uint32))} floats differ, "
            f"max |diff| {d.max():.3g} at {i}: {mine[i]!r} vs {theirs[i]!r}")


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_rfi_bit_exact_against_reference(ref, name):
    from frost_b200.rfi import RFICleaner
    golden = json.load(open(GOLDEN))[name]
    cfg, layout, baseline, blocks = make_case(name)
    gpu = RFICleaner(cfg, layout, baseline)
    cpu = ref.RefRFICleaner(cfg, layout, baseline)
    for step, (block, nsamps) in enumerate(blocks):
        mine = gpu.execute_normalized(block, nsamps)
        theirs = cpu.execute_normalized(block, nsamps)
        rep_m, rep_t = gpu.report(), cpu.report()
        for k in COUNTS:
            assert rep_m[k] == rep_t[k], f"step {step} report.{k}: {rep_m[k]} vs {rep_t[k]}"
        assert np.array_equal(gpu.channel_mask(), cpu.channel_mask()), f"step {step} mask"
        assert mine.shape == theirs.shape
        assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32)), \
            f"step {step}: " + describe_diff(mine, theirs)
        assert digest(mine) == golden[step]["out_sha256"]
        assert digest(gpu.channel_mask()) == golden[step]["mask_sha256"]


@pytest.mark.gpu
def test_rfi_rejects_bad_input_before_work():
    from frost_b200.config import BlockLayout, DataType, RfiConfig
    from frost_b200.rfi import RFICleaner
    lay = BlockLayout(16, 128, DataType.FLOAT32, 1e-3, 1400.0, -1.0)
    gpu = RFICleaner(RfiConfig(), lay, 2.0)
    x = np.ones((128, 16), np.float32)
    x[70, 3] = np.inf
    with pytest.raises(ValueError, match="sample 70, channel 3"):
        gpu.execute_normalized(x)
    with pytest.raises(ValueError):
        gpu.execute_normalized(np.ones(16 * 4 * 3 + 1, np.uint8))
    with pytest.raises(ValueError):
        gpu.execute_normalized(np.ones((129, 16), np.float32))
    with pytest.raises(ValueError):
        RFICleaner(RfiConfig(), BlockLayout(0, 128, DataType.UINT8, 1e-3, 1400.0, -1.0), 2.0)


@pytest.mark.gpu
def test_rfi_full_size_channel_mask_and_flags_match_reference(ref):
    """A config-2-like gulp at 1/4 length (4096 channels x 65536 samples,
    every strategy): masks, flags and reports bit-exact, normalized waterfall
    bit-exact."""
    from frost_b200.config import BlockLayout, DataType, RfiConfig, ZeroDMMode
    from frost_b200.rfi import RFICleaner
    from frost_b200.synth import config2_gulp
    fb = config2_gulp(nsamps=65536, n_pulses=4)
    cfg = RfiConfig()
    cfg.moments.enabled = True
    cfg.iqrm.enabled = True
    cfg.kadane_channel.enabled = True
    cfg.kadane_spectrum.enabled = True
    cfg.zero_dm = ZeroDMMode.SUBTRACT
    lay = BlockLayout(fb.nchans, fb.nsamps, DataType.UINT8, fb.tsamp, fb.fch1, fb.foff)
    block = fb.data.reshape(-1)
    gpu = RFICleaner(cfg, lay, 2.0)
    cpu = ref.RefRFICleaner(cfg, lay, 2.0)
    mine = gpu.execute_normalized(block)
    theirs = cpu.execute_normalized(block)
    rep_m, rep_t = gpu.report(), cpu.report()
    for k in COUNTS:
        assert rep_m[k] == rep_t[k], f"report.{k}: {rep_m[k]} vs {rep_t[k]}"
    assert np.array_equal(gpu.channel_mask(), cpu.channel_mask())
    assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32)), describe_diff(mine, theirs)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["zdot_equalize_u8", "all_strategies_f32"])
def test_rfi_unaligned_device_block_matches_aligned(name):
    """A device block that does not start on a 16-byte boundary (here one
    byte past it) is copied to an aligned buffer first; the result is the
    same bits as from the aligned block."""
    import torch

    from frost_b200.rfi import RFICleaner
    cfg, layout, baseline, blocks = make_case(name)
    block, nsamps = blocks[0]
    buf = torch.zeros(block.size + 16, dtype=torch.uint8, device="cuda")
    outs = []
    for off in (0, 1):
        buf[off:off + block.size].copy_(torch.from_numpy(block))
        gpu = RFICleaner(cfg, layout, baseline)
        gpu.execute_normalized_device(buf.data_ptr() + off, block.size, nsamps, on_device=True)
        outs.append((gpu.download().copy(), gpu.channel_mask().copy()))
    assert np.array_equal(outs[0][0].view(np.uint32), outs[1][0].view(np.uint32))
    assert np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.gpu
def test_rfi_device_block_needs_a_stream_and_orders_after_it():
    """A device block is read after the work queued on the caller's stream
    (an async copy written behind other work on that stream gives the
    host-input result), and the null stream is refused for a device block."""
    import ctypes as C

    import torch

    from frost_b200._lib import lib
    from frost_b200.rfi import RFICleaner
    cfg, layout, baseline, blocks = make_case("default_u8")
    block, nsamps = blocks[0]
    ref = RFICleaner(cfg, layout, baseline)
    want = ref.execute_normalized(block, nsamps)
    gpu = RFICleaner(cfg, layout, baseline)
    s = torch.cuda.Stream()
    dev = torch.zeros(block.size, dtype=torch.uint8, device="cuda")
    host = torch.from_numpy(np.ascontiguousarray(block)).pin_memory()
    junk = torch.empty((4096, 4096), device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        for _ in range(8):
            junk.normal_()
            junk = junk @ junk
        dev.copy_(host, non_blocking=True)
    gpu.execute_normalized_device(dev.data_ptr(), block.size, nsamps, on_device=True, stream=s.cuda_stream)
    got = gpu.download()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    out = C.c_void_p()
    rc = lib().frost_rfi_execute_normalized(gpu._h, C.c_void_p(dev.data_ptr()), block.size, nsamps, 1, None,
                                            C.byref(out))
    assert rc == -1 and "null stream" in lib().frost_last_error().decode()
