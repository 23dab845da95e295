"""The `.cand` writer: the reference tests' known answers
(tests/cpp/api/cand_writer_test.cpp) and byte-for-byte equality with the
reference's own writer (lib/output/cand_writer.cpp, compiled into
oracle/_ref) on seeded giants, appends, offsets and file names."""

import math
import os

import numpy as np
import pytest

from frost_b200.output import CandWriter, cand_filename
from frost_b200.postprocess import make_giants
from oracle import postprocess as op
from tests.postprocess_cases import random_giants

REF = pytest.mark.skipif(not op.ref_available(), reason="reference sources not built (make -C oracle ref)")


def _giant():
    g = make_giants(1)
    g["snr"], g["samp_idx"], g["filter_idx"], g["dm_idx"], g["dm"] = 12.5, 100, 3, 7, 42.5
    g["members"], g["begin"], g["end"] = 4, 98, 102
    g["f_low"], g["f_high"], g["chan_begin"], g["chan_end"] = 1200.5, 1500.25, 4, 19
    return g


def _cols(path):
    with open(path) as f:
        return [line.rstrip("\n").split("\t") for line in f]


def test_standard_layout(tmp_path):
    p = os.path.join(tmp_path, "a.cand")
    with CandWriter(p, 0.001) as w:
        w.write(_giant())
    c = _cols(p)[0]
    assert len(c) == 23
    assert [float(c[0]), int(c[1]), float(c[2]), int(c[3]), int(c[4]), float(c[5]), int(c[6]), int(c[7]),
            int(c[8]), float(c[9]), float(c[10]), int(c[11]), int(c[12])] == \
        [12.5, 100, 0.1, 3, 7, 42.5, 4, 98, 102, 1200.5, 1500.25, 4, 19]
    assert (float(c[13]), int(c[14]), int(c[15]), int(c[16])) == (12.5, 4, 19, 1)


def test_strongest_subband_and_location(tmp_path):
    g = _giant()
    g["snr_best"], g["best_chan_begin"], g["best_chan_end"], g["n_extents"] = 40.0, 0, 3, 3
    p = os.path.join(tmp_path, "sub", "best.cand")  # parent directory created
    with CandWriter(p, 0.001) as w:
        w.write(g)
    c = _cols(p)[0]
    assert c[13:17] == ["40", "0", "3", "3"]
    g = _giant()
    g["snr_best"], g["best_chan_begin"], g["best_chan_end"] = 30, 8, 15
    g["has_location_best"], g["loc_samp_idx"], g["loc_dm"], g["loc_filter_width"] = 1, 120, 80.5, 16
    g["loc_f_low"], g["loc_f_high"] = 1300, 1400
    with CandWriter(p, 0.001) as w:
        w.write(g, 1000)
    c = _cols(p)[0]
    assert c[1] == "1100" and c[17] == "1120" and c[19] == "80.5" and c[20] == "16"
    assert math.isclose(float(c[18]), 1.12) and c[21] == "1300" and c[22] == "1400"


def test_appends_across_calls(tmp_path):
    p = os.path.join(tmp_path, "c.cand")
    with CandWriter(p, 0.001) as w:
        w.write(_giant())
        w.write(_giant(), 5)
    with CandWriter(p, 0.001, append=True) as w:
        w.write(_giant(), 10)
    assert [r[1] for r in _cols(p)] == ["100", "105", "110"]


@REF
@pytest.mark.parametrize("seed", range(3))
def test_bytes_equal_reference_writer(tmp_path, seed):
    R = op.backend("reference")
    g = random_giants(seed, 300)
    rng = np.random.default_rng(seed)
    g["snr"][::17] = rng.uniform(1e-3, 1e6, g[::17].size)
    g["dm"][::13] = rng.uniform(0, 5000, g[::13].size)
    g["samp_idx"][::11] += np.uint64(1) << np.uint64(40)
    for dt, first, append in ((64e-6, 0, False), (1e-3, 123456789, True), (0.000256, 7, True)):
        a, b = os.path.join(tmp_path, "mine.cand"), os.path.join(tmp_path, "ref.cand")
        with CandWriter(a, dt, append=append) as w:
            w.write(g[:150], first)
            w.write(g[150:], first + 1)
        R.cand_write(b, dt, append, g[:150], first)
        R.cand_write(b, dt, True, g[150:], first + 1)
        assert open(a, "rb").read() == open(b, "rb").read()


@REF
def test_filename_matches_reference():
    R = op.backend("reference")
    for utc, beam in ((0, 1), (1733270400, 7), (1900000000, 13), (2000000000, 123)):
        assert cand_filename(utc, beam) == R.cand_filename(utc, beam)
    assert cand_filename(1733270400, 7) == "2024-12-04-00:00:00_07.cand"
