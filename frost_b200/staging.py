"""Input staging for one beam, the B200 form of frost's GulpPrefetch
(lib/pipeline/pipeline.cpp:105-262): a reader thread in the library fills
pinned host slots from a block source and copies them to device slots, so
the next gulp is read and transferred while the current one is searched.
SIGPROC filterbanks (frost's file input, lib/pipeline/input.cpp:32-69) are
opened by their header:

    pf = GulpPrefetch.from_sigproc(path, block_rows)
    layout = sigproc_layout(pf.header, block_rows)
    with pf:
        for ptr, nread in pf:
            pipe.execute_device(ptr, nread, on_device=True)
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Iterator, Optional, Tuple

import numpy as np

from . import _abi
from ._lib import check, lib


def read_sigproc_header(path: str) -> dict:
    """The SIGPROC header of the filterbank at `path` (header_bytes, nchans,
    nbits, row_bytes, data_rows, fch1, foff, tsamp, tstart, ...)."""
    h = _abi.SigprocHeaderC()
    check(lib().frost_sigproc_read_header(str(path).encode(), C.byref(h)))
    return h.as_dict()


def sigproc_layout(header: dict, block_rows: int):
    """frost_b200.config.BlockLayout of a SIGPROC file's rows for gulps of
    `block_rows` samples."""
    from .config import BlockLayout, DataType
    h = _abi.SigprocHeaderC()
    for k, _ in h._fields_:
        v = header[k]
        setattr(h, k, v.encode() if k == "source_name" else v)
    out = _abi.BlockLayoutC()
    check(lib().frost_sigproc_layout(C.byref(h), int(block_rows), C.byref(out)))
    return BlockLayout(out.nchans, out.max_nsamps, DataType(out.dtype), out.tsamp, out.f0, out.df)


@dataclass
class PrefetchStats:
    gulps: int
    bytes: int
    read_s: float
    wait_s: float


class GulpPrefetch:
    """Gulps of `block_rows` packed rows of `row_bytes`, `depth` slots ahead,
    delivered on `device`. Build with from_file, from_memory or from_source."""

    def __init__(self, handle: C.c_void_p, keep=()):
        self._h = handle
        self._keep = keep  # objects the library reads until close

    @classmethod
    def from_file(cls, path: str, header_bytes: int, block_rows: int, row_bytes: int, depth: int = 2,
                  device: int = 0) -> "GulpPrefetch":
        h = C.c_void_p()
        check(lib().frost_prefetch_create_file(path.encode(), int(header_bytes), int(block_rows), int(row_bytes),
                                               int(depth), int(device), C.byref(h)))
        return cls(h)

    @classmethod
    def from_sigproc(cls, path: str, block_rows: int, depth: int = 2, device: int = 0) -> "GulpPrefetch":
        """The rows of a SIGPROC filterbank after its parsed header; the
        header is `self.header`."""
        h = C.c_void_p()
        hdr = _abi.SigprocHeaderC()
        check(lib().frost_prefetch_create_sigproc(str(path).encode(), int(block_rows), int(depth), int(device),
                                                  C.byref(hdr), C.byref(h)))
        pf = cls(h)
        pf.header = hdr.as_dict()
        return pf

    @classmethod
    def from_memory(cls, rows: np.ndarray, block_rows: int, depth: int = 2, device: int = 0) -> "GulpPrefetch":
        """Rows of a [nrows][row_bytes] uint8 array (kept alive by the object)."""
        a = np.ascontiguousarray(rows).view(np.uint8)
        if a.ndim != 2:
            raise ValueError("rows must be [nrows][row_bytes]")
        h = C.c_void_p()
        check(lib().frost_prefetch_create_memory(a.ctypes.data if a.size else None, a.shape[0], int(block_rows),
                                                 a.shape[1], int(depth), int(device), C.byref(h)))
        return cls(h, keep=(a,))

    @classmethod
    def from_source(cls, read: Callable[[np.ndarray], int], block_rows: int, row_bytes: int, depth: int = 2,
                    device: int = 0) -> "GulpPrefetch":
        """`read(buf)` fills a [block_rows][row_bytes] uint8 view and returns
        the rows written (fewer at the end, 0 once exhausted); it runs on the
        library's reader thread."""
        def cb(_ctx, buf, max_rows):
            try:
                view = np.ctypeslib.as_array(buf, shape=(int(max_rows) * int(row_bytes),))
                return int(read(view.reshape(int(max_rows), int(row_bytes))))
            except Exception:
                return -1
        fn = _abi.READ_FN(cb)
        h = C.c_void_p()
        check(lib().frost_prefetch_create(int(block_rows), int(row_bytes), int(depth), int(device), fn, None,
                                          C.byref(h)))
        return cls(h, keep=(fn,))

    def next(self, stream: Optional[int] = None) -> Tuple[int, int]:
        """(device pointer, rows) of the next gulp; rows = 0 at the end."""
        ptr, n = C.c_void_p(), C.c_size_t()
        check(lib().frost_prefetch_next(self._h, C.c_void_p(stream) if stream else None, C.byref(ptr),
                                        C.byref(n)))
        return (ptr.value or 0), n.value

    def __iter__(self) -> Iterator[Tuple[int, int]]:
        while True:
            ptr, n = self.next()
            if n == 0:
                return
            yield ptr, n

    def stats(self) -> PrefetchStats:
        s = _abi.PrefetchStatsC()
        check(lib().frost_prefetch_get_stats(self._h, C.byref(s)))
        return PrefetchStats(s.gulps, s.bytes, s.read_s, s.wait_s)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().frost_prefetch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
