"""Input staging (the B200 form of frost's GulpPrefetch,
lib/pipeline/pipeline.cpp:105-262): gulps read and copied to the device by
the library's reader thread, 2-3 slots ahead, give the per-gulp pipeline
exactly the candidates it gives when fed the same bytes directly; whole and
partial last gulps end the stream; a failing source surfaces at its gulp;
a caller stream orders the copy before the gulp's kernels."""

import os

import numpy as np
import pytest

from frost_b200.config import BlockLayout, BoxcarConfig, DataType, RfiConfig
from frost_b200.synth import make_filterbank

pytestmark = pytest.mark.gpu

NCHANS, GULP, TSAMP = 256, 8192, 1e-3


def _setup(ngulps, tail):
    from frost_b200.pipeline import plan_for
    fb = make_filterbank(NCHANS, GULP * ngulps, 1500.0, -1.0, TSAMP, 51, n_pulses=5, dm_range=(5.0, 60.0),
                         snr_range=(10.0, 25.0), rfi_channel_fraction=0.03, n_bursts=1)
    data = np.ascontiguousarray(fb.data[:GULP * ngulps - tail])
    layout = BlockLayout(NCHANS, GULP, DataType.UINT8, TSAMP, 1500.0, -1.0)
    return data, layout, plan_for(layout, 0.0, 80.0, subband_depth=1), BoxcarConfig(max_boxcar=32,
                                                                                    detect_thresh=7.0)


def _direct(data, layout, plan, bc):
    from frost_b200.pipeline import GulpPipeline
    p = GulpPipeline(RfiConfig(), layout, 1.0, plan, bc)
    out = []
    for g in range(0, data.shape[0], GULP):
        block = np.zeros((GULP, NCHANS), np.uint8)
        n = min(GULP, data.shape[0] - g)
        block[:n] = data[g:g + n]
        out.append(p.execute(block, n).candidates)
    out.append(p.flush().candidates)
    return out


def _through(pf, layout, plan, bc, stream=None):
    from frost_b200.pipeline import GulpPipeline
    p = GulpPipeline(RfiConfig(), layout, 1.0, plan, bc)
    out = []
    while True:
        ptr, n = pf.next(stream.cuda_stream if stream is not None else None)
        if n == 0:
            break
        out.append(p.execute_device(ptr, n, on_device=True,
                                    stream=stream.cuda_stream if stream is not None else None).candidates)
    out.append(p.flush().candidates)
    return out


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("depth,tail", [(2, 1500), (3, 0)])
def test_memory_source_matches_direct(depth, tail):
    from frost_b200.staging import GulpPrefetch
    data, layout, plan, bc = _setup(4, tail)
    ref = _direct(data, layout, plan, bc)
    with GulpPrefetch.from_memory(data, GULP, depth=depth) as pf:
        got = _through(pf, layout, plan, bc)
        st = pf.stats()
    _same(got, ref)
    assert st.gulps == 4 and st.bytes == data.size
    assert sum(len(c) for c in ref) > 0


def test_file_source_and_caller_stream(tmp_path):
    import torch
    from frost_b200.staging import GulpPrefetch
    data, layout, plan, bc = _setup(3, 700)
    ref = _direct(data, layout, plan, bc)
    path = os.path.join(tmp_path, "beam.fil")
    header = b"HEADER_START" + bytes(100) + b"HEADER_END"
    with open(path, "wb") as f:
        f.write(header)
        f.write(data.tobytes())
    with GulpPrefetch.from_file(path, len(header), GULP, NCHANS, depth=2) as pf:
        _same(_through(pf, layout, plan, bc), ref)
    s = torch.cuda.Stream()
    with GulpPrefetch.from_file(path, len(header), GULP, NCHANS, depth=3) as pf:
        _same(_through(pf, layout, plan, bc, stream=s), ref)


def test_sigproc_filterbank_source(tmp_path):
    """A SIGPROC filterbank written as frost's fake filterbank writes one:
    the prefetch parses its header, and the layout taken from the header
    gives the pipeline the candidates of the same rows fed directly."""
    from frost_b200.staging import GulpPrefetch, sigproc_layout
    from tests.test_sigproc import write_filterbank
    data, layout, plan, bc = _setup(3, 300)
    ref = _direct(data, layout, plan, bc)
    path = os.path.join(tmp_path, "beam.fil")
    write_filterbank(path, nchans=NCHANS, nbits=8, fch1=1500.0, foff=-1.0, tsamp=TSAMP, data=data)
    pf = GulpPrefetch.from_sigproc(path, GULP, depth=2)
    assert pf.header["data_rows"] == data.shape[0] and pf.header["nchans"] == NCHANS
    assert sigproc_layout(pf.header, GULP) == layout
    with pf:
        _same(_through(pf, layout, plan, bc), ref)


def test_callback_source_and_its_failure():
    from frost_b200._lib import FrostError
    from frost_b200.staging import GulpPrefetch
    data, layout, plan, bc = _setup(3, 0)
    pos = [0]

    def read(buf):
        n = min(buf.shape[0], data.shape[0] - pos[0])
        buf[:n] = data[pos[0]:pos[0] + n]
        pos[0] += n
        return n

    ref = _direct(data, layout, plan, bc)
    with GulpPrefetch.from_source(read, GULP, NCHANS) as pf:
        _same(_through(pf, layout, plan, bc), ref)

    calls = [0]

    def failing(buf):
        calls[0] += 1
        if calls[0] == 2:
            return -1
        buf[:] = data[:buf.shape[0]]
        return buf.shape[0]

    with GulpPrefetch.from_source(failing, GULP, NCHANS) as pf:
        ptr, n = pf.next()
        assert n == GULP and ptr != 0
        with pytest.raises(FrostError):
            pf.next()
