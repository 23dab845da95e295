"""SIGPROC filterbank headers as frost's file input reads them
(lib/pipeline/input.cpp:32-69, through psrio): files written the way
frost's fake filterbank writes them (tests/cpp/support/fake_filterbank.hpp:
80-96) parse to their fields, the data offset and the row count; channel
tables and source names are skipped or kept; malformed headers, unknown
keywords and multi-IF data are refused. Host code only."""

import struct

import numpy as np
import pytest

from frost_b200._lib import FrostError
from frost_b200.config import DataType
from frost_b200.staging import read_sigproc_header, sigproc_layout


def _s(text):
    b = text.encode()
    return struct.pack("<i", len(b)) + b


def write_filterbank(path, nchans=32, nsamps=100, nbits=8, fch1=1400.0, foff=-1.0, tsamp=1e-3, tstart=58000.0,
                     nifs=1, extra=b"", data=None):
    """Header records in the order frost's fake filterbank writes them."""
    h = _s("HEADER_START")
    h += _s("telescope_id") + struct.pack("<i", 4)
    h += _s("machine_id") + struct.pack("<i", 10)
    h += _s("data_type") + struct.pack("<i", 1)
    h += _s("fch1") + struct.pack("<d", fch1)
    h += _s("foff") + struct.pack("<d", foff)
    h += _s("nchans") + struct.pack("<i", nchans)
    h += _s("nbits") + struct.pack("<i", nbits)
    h += _s("nifs") + struct.pack("<i", nifs)
    h += _s("tsamp") + struct.pack("<d", tsamp)
    h += _s("tstart") + struct.pack("<d", tstart)
    h += _s("ibeam") + struct.pack("<i", 0)
    h += extra
    h += _s("HEADER_END")
    if data is None:
        data = (np.arange(nsamps * nchans * nbits // 8) % 251).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(h)
        f.write(np.ascontiguousarray(data).tobytes())
    return len(h)


def test_fake_filterbank_header(tmp_path):
    p = tmp_path / "a.fil"
    hb = write_filterbank(p, nchans=64, nsamps=1000, fch1=1500.0, foff=-0.29296875, tsamp=64e-6)
    h = read_sigproc_header(p)
    assert h["header_bytes"] == hb
    assert (h["nchans"], h["nbits"], h["nifs"], h["row_bytes"], h["data_rows"]) == (64, 8, 1, 64, 1000)
    assert (h["fch1"], h["foff"], h["tsamp"], h["tstart"]) == (1500.0, -0.29296875, 64e-6, 58000.0)
    assert (h["telescope_id"], h["machine_id"], h["data_type"], h["ibeam"]) == (4, 10, 1, 0)
    lay = sigproc_layout(h, 512)
    assert (lay.nchans, lay.max_nsamps, lay.dtype, lay.tsamp, lay.f0, lay.df) == \
        (64, 512, DataType.UINT8, 64e-6, 1500.0, -0.29296875)


def test_channel_table_source_name_and_sample_types(tmp_path):
    extra = _s("source_name") + _s("FRB 20201124A") + _s("FREQUENCY_START")
    for f in (1400.0, 1399.0):
        extra += _s("fchannel") + struct.pack("<d", f)
    extra += _s("FREQUENCY_END") + _s("signed") + struct.pack("<b", 0) + _s("nsamples") + struct.pack("<i", 77)
    for nbits, dtype in ((1, DataType.UINT1), (2, DataType.UINT2), (4, DataType.UINT4), (16, DataType.UINT16),
                         (32, DataType.FLOAT32)):
        p = tmp_path / f"b{nbits}.fil"
        hb = write_filterbank(p, nchans=32, nsamps=10, nbits=nbits, extra=extra)
        h = read_sigproc_header(p)
        assert h["header_bytes"] == hb and h["source_name"] == "FRB 20201124A" and h["nsamples"] == 77
        assert h["row_bytes"] == 32 * nbits // 8 and h["data_rows"] == 10
        assert sigproc_layout(h, 4).dtype == dtype


def test_bad_headers_are_refused(tmp_path):
    p = tmp_path / "x.fil"
    p.write_bytes(_s("NOT_A_HEADER") + b"\0" * 64)
    with pytest.raises(ValueError, match="HEADER_START"):
        read_sigproc_header(p)
    write_filterbank(p, extra=_s("mystery_key") + struct.pack("<i", 1))
    with pytest.raises(ValueError, match="unknown header keyword"):
        read_sigproc_header(p)
    write_filterbank(p, nifs=2)
    with pytest.raises(ValueError, match="nifs"):
        read_sigproc_header(p)
    write_filterbank(p)
    p.write_bytes(p.read_bytes()[:60])
    with pytest.raises(ValueError, match="ends inside"):
        read_sigproc_header(p)
    with pytest.raises(FrostError) as e:
        read_sigproc_header(tmp_path / "missing.fil")
    assert e.value.code == -7
    write_filterbank(p, nbits=3, nchans=8)
    with pytest.raises(ValueError, match="nbits"):
        sigproc_layout(read_sigproc_header(p), 8)
