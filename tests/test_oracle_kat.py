"""Known-answer tests that pin the oracle (the reference's own CPU code built
into oracle/_ref) and this library to the reference's own golden vectors.
The library's IQRM runs on the GPU, so its cases are marked gpu; the rest
is CPU only."""

import json
import os

import numpy as np
import pytest

from frost_b200 import dedisp as fdedisp
from frost_b200 import rfi as frfi
from frost_b200.config import DedispPlanConfig, RfiConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def flagged(m):
    return list(np.nonzero(m)[0])


def iqrm_cases():
    g = json.load(open(os.path.join(GOLDEN, "iqrm_golden.json")))
    x = np.array(g["x"], np.float32)
    for case in g["cases"]:
        ig = None
        if case["ignore"]:
            ig = np.zeros(x.size, np.uint8)
            ig[case["ignore"]] = 1
        yield x, case, ig


GPU_IMPL = pytest.param("frost_b200", marks=pytest.mark.gpu)


@pytest.mark.parametrize("impl", ["reference", GPU_IMPL])
def test_iqrm_golden_vectors(ref, impl):
    """rfi_test.cpp:213-257: Morello et al. (2022) synthetic channels."""
    fn = ref.iqrm_mask if impl == "reference" else frfi.iqrm_mask
    for x, case, ig in iqrm_cases():
        assert flagged(fn(x, case["radius"], case["threshold"], ig)) == case["expected"], case


@pytest.mark.parametrize("impl", ["reference", GPU_IMPL])
def test_iqrm_noise_tophat_and_limits(ref, impl):
    fn = ref.iqrm_mask if impl == "reference" else frfi.iqrm_mask
    rng = np.random.default_rng(3)
    y = rng.standard_normal(1024).astype(np.float32)
    for radius in (1, 2, 5, 100):
        assert flagged(fn(y, radius, 4.0)) == []
    y = np.random.default_rng(5).standard_normal(256).astype(np.float32)
    y[100:104] += 50.0
    assert flagged(fn(y, 6, 3.0)) == [100, 101, 102, 103]
    x = next(iqrm_cases())[0]
    with pytest.raises(ValueError):
        fn(x, 0, 3.0)
    with pytest.raises(ValueError):
        fn(x, 3, 0.0)


@pytest.mark.gpu
def test_iqrm_matches_reference_on_random_inputs(ref):
    """Lag saturation and ignore handling (iqrm_limits_test.cpp:8-28) plus
    random statistics with ignored channels: identical flags."""
    rng = np.random.default_rng(11)
    for count in (1, 2, 3, 8, 32, 97, 500, 4096):
        v = ((np.arange(count) * 17 + 3) % 11).astype(np.float32)
        v[count // 2] += 100
        for edge in (0, 1):
            ig = np.zeros(count, np.uint8)
            ig[-1] = edge
            for radius in (2 * count, 2**62):
                assert np.array_equal(frfi.iqrm_mask(v, radius, 3, ig), ref.iqrm_mask(v, radius, 3, ig))
        x = rng.gamma(2.0, 1.0, count).astype(np.float32)
        ig = (rng.random(count) < 0.05).astype(np.uint8)
        for radius in (1, max(count // 10, 1), count):
            for thr in (1.5, 3.0):
                assert np.array_equal(frfi.iqrm_mask(x, radius, thr, ig), ref.iqrm_mask(x, radius, thr, ig))


def test_kadane_brute_force_and_chunked_combine(ref):
    """rfi_kernels_test.cpp:20-81: the reference monoid finds the maximum-sum
    run sequentially and in randomly cut chunks."""
    rng = np.random.default_rng(9)
    for _ in range(20):
        u = rng.normal(-0.1, 1.0, 200)
        best, bs, be = 0.0, 0, -1
        for i in range(200):
            s = 0.0
            for j in range(i, 200):
                s += u[j]
                if s > best:
                    best, bs, be = s, i, j
        for chunk in (0, 1, 7, 60):
            s, a, b, _ = ref.kadane(u, chunk_len=chunk)
            assert s == pytest.approx(best) and (a, b) == (bs, be)
    s, a, b, _ = ref.kadane(np.array([-1.0, 2.0, 1.0, -5.0, 0.5]), idx=np.array([0, 3, 4, 9, 12]))
    assert (s, a, b) == (3.0, 3, 4)


def test_broadband_whole_series_flags(ref):
    """device_rfi_flags_test.cpp:36-55: whole-series MAD, exact flags."""
    n = 8192
    t = np.arange(n)
    amp = np.where(t < 3125, 1.0, 8.0)
    series = np.where(t % 2 == 1, -amp, amp).astype(np.float32)
    series[6000], series[7000] = 80, -80
    flags = np.zeros(n, np.uint8)
    flags[10] = 1
    count, out = ref.broadband_time_flags(series, n, 5, 1, flags)
    assert count == 2
    assert flagged(out) == [10, 6000, 7000]


def test_dedisp_band_edges_and_validation(ref):
    """dedisp_test.cpp:69-93: f_min 1384.5 / f_max 1400.5 for 16 ch at
    1400 MHz, df = -1, either axis; invalid setups raise."""
    cfg = DedispPlanConfig(nchans=16, dt=1e-3, f0=1400.0, df=-1.0, dm_min=0, dm_max=50,
                           dm_pulse_width=1000.0, dm_tol=1.25, block_nsamps=1024)
    for fn in (ref.fdmt_band_edges, fdedisp.band_edges):
        assert fn(cfg) == (1384.5, 1400.5)
        asc = DedispPlanConfig(**{**cfg.__dict__, "f0": 1385.0, "df": 1.0})
        assert fn(asc) == (1384.5, 1400.5)
        for bad in ({"df": 0.0}, {"nchans": 1}, {"f0": 0.1}):
            with pytest.raises(ValueError):
                fn(DedispPlanConfig(**{**cfg.__dict__, **bad}))


def test_dm_lists_bit_exact_against_golden(ref):
    """generate_dm_list (lib/dedisp/dedisp.cpp:16-69) reproduced bit for bit
    against the reference's lists for the benchmark setups."""
    from tests.golden.make_golden import DM_SETUPS
    golden = np.load(os.path.join(GOLDEN, "dm_lists.npz"))
    for name, (n, dt, f0, df, lo, hi, pw) in DM_SETUPS.items():
        cfg = DedispPlanConfig(nchans=n, dt=dt, f0=f0, df=df, dm_min=lo, dm_max=hi,
                               dm_pulse_width=pw, dm_tol=1.25)
        mine = fdedisp.generate_dm_list(cfg)
        assert np.array_equal(mine.view(np.uint32), golden[name].view(np.uint32)), name
        assert np.array_equal(ref.generate_dm_list(cfg).view(np.uint32), golden[name].view(np.uint32))
        assert mine[0] == lo and mine[-1] >= hi and np.all(np.diff(mine) > 0)
    assert golden["config2"].size == 3625 and golden["config1"].size == 886
    with pytest.raises(ValueError):
        fdedisp.generate_dm_list(DedispPlanConfig(nchans=16, dt=1e-3, f0=1400, df=-1, dm_max=50,
                                                  dm_tol=1.0))


def test_kill_file_and_manual_zaps(ref, tmp_path):
    """kill_file_test semantics: strict 0/1 lines, comments, merged ranges."""
    p = tmp_path / "k.txt"
    p.write_text("1\n0 # killed\n\n0\n1\n# c\n0\n1\n1\n0\n")
    for fn in (ref.read_kill_file, frfi.read_kill_file):
        assert fn(str(p), 8) == [(1, 2), (4, 4), (7, 7)]
        with pytest.raises(ValueError):
            fn(str(p), 9)
    bad = tmp_path / "bad.txt"
    bad.write_text("1\n2\n")
    for fn in (ref.read_kill_file, frfi.read_kill_file):
        with pytest.raises(ValueError):
            fn(str(bad), 2)
    with pytest.raises(Exception):
        frfi.read_kill_file(str(tmp_path / "missing.txt"), 2)
    m = frfi.apply_manual_killmask(np.ones(16, np.uint8), [(2, 4), (10, 10)])
    assert list(m) == [1, 1, 0, 0, 0, 1, 1, 1, 1, 1, 0, 1, 1, 1, 1, 1]
    assert list(frfi.apply_manual_killmask(np.ones(4, np.uint8), [(2, 100), (50, 60)])) == [1, 1, 0, 0]


def test_rfi_config_validation_matches_reference(ref):
    import ctypes
    from frost_b200 import _lib
    bad = []
    for field, val in (("narrow.threshold", -1.0), ("broad.threshold", float("nan")),
                       ("dropout.min_std_fraction", 1.5), ("kadane_spectrum.min_bandwidth", -1.0),
                       ("broad.boxcar_max", 0)):
        cfg = RfiConfig()
        obj, attr = field.split(".")
        setattr(getattr(cfg, obj), attr, val)
        bad.append(cfg)
    z = RfiConfig()
    z.zap_chans = [(5, 2)]
    bad.append(z)
    for cfg in bad + [RfiConfig()]:
        c, keep = cfg.to_c()
        mine = _lib.lib().frost_rfi_config_validate(ctypes.byref(c))
        try:
            ref.rfi_config_validate(cfg)
            theirs = 0
        except ValueError:
            theirs = -1
        assert mine == theirs
