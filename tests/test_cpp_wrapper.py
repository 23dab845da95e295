"""The C++20 wrapper (include/frost_b200.hpp), compiled with g++ against the
in-tree library the way a frost host program would use it: host-only calls
and frost's error types on CPU; on the GPU, gulps through its GulpPipeline
give exactly the candidates of the Python GulpPipeline on the same bytes."""

import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "frost_b200", "lib")


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "wrapper_test")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "wrapper_test.cpp"), "-L", LIB, "-lfrost_b200",
           f"-Wl,-rpath,{LIB}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def test_host_calls_and_error_types(binary):
    r = subprocess.run([binary, "cpu"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ndm 886" in r.stdout and "invalid_argument" in r.stdout and r.stdout.strip().endswith("ok")


@pytest.mark.gpu
def test_cpp_pipeline_matches_python_pipeline(binary, tmp_path):
    from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig
    from frost_b200.pipeline import GulpPipeline, plan_for
    from frost_b200.search import CANDIDATE_DTYPE
    from frost_b200.synth import make_filterbank

    nchans, gulp, ngulps = 256, 8192, 3
    data = make_filterbank(nchans, gulp * ngulps, 1500.0, -1.0, 1e-3, 41, n_pulses=5,
                           dm_range=(5.0, 60.0), snr_range=(10.0, 25.0), rfi_channel_fraction=0.03,
                           n_bursts=2).data
    blk = tmp_path / "block.bin"
    data.tofile(blk)
    out = tmp_path / "cands.bin"
    r = subprocess.run([binary, "gpu", str(blk), str(nchans), str(gulp), str(ngulps), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    mine = np.fromfile(out, CANDIDATE_DTYPE)

    layout = BlockLayout(nchans, gulp, DataType.UINT8, 1e-3, 1500.0, -1.0)
    plan = plan_for(layout, 0.0, 80.0, subband_depth=1)
    bc = BoxcarConfig(max_boxcar=32, detect_thresh=7.0, max_candidates=1 << 16, max_cands_per_dm=0)
    p = GulpPipeline(RfiConfig(), layout, 1.0, plan, bc)
    ref = [p.execute(data[g * gulp:(g + 1) * gulp], gulp).candidates for g in range(ngulps)]
    ref.append(p.flush().candidates)
    ref = np.concatenate(ref)
    assert ref.size > 0
    assert np.array_equal(mine, ref)
