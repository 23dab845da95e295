"""The allocation-free entry point frost_rfi_normalize_static, for callers
that cannot call cudaMalloc while processing (a real-time consumer whose
device memory is all sized at start-up, or a program whose device memory
belongs to another framework's pool): through the C ABI, two calls in a row
must give exactly what the allocating frost_rfi_execute_normalized gives for
the same blocks with every excision strategy off, later calls must leave the
device's free memory unchanged, and requests larger than its fixed static
scratch (or without a stream) must be refused with a clear error.

Named to be collected last, so a run that stops at the first failure has
already run every other test."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _blocks(nchans, nsamps, seed, dtype):
    rng = np.random.default_rng(seed)
    if dtype == "uint8":
        x = np.clip(np.rint(rng.normal(120, 14, (nsamps, nchans))), 0, 255).astype(np.uint8)
        x[1000:1003, :] = 255   # a burst the quiet configuration keeps
        x[:, 5] = 77            # a dead (constant) channel
        return x
    x = rng.normal(3.0, 0.5, (nsamps, nchans)).astype(np.float32)
    x[:, 9] = 1.25
    return x


def _static(layout, raw, nsamps, out, stream):
    from frost_b200 import _lib
    lay = layout.to_c()
    return _lib.lib().frost_rfi_normalize_static(C.byref(lay), C.c_float(2.0), C.c_void_p(raw.data_ptr()),
                                                 raw.numel(), nsamps, C.c_void_p(out.data_ptr()),
                                                 out.numel(), C.c_void_p(stream) if stream else None)


def _run_both(layout, block_np, nsamps=0):
    import torch

    from frost_b200 import _lib
    from frost_b200.config import RfiConfig
    from frost_b200.rfi import RFICleaner

    raw = torch.from_numpy(np.ascontiguousarray(block_np).view(np.uint8).reshape(-1)).cuda()
    capacity = raw.numel() // layout.row_bytes
    out = torch.empty(layout.nchans * capacity, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    _lib.check(_static(layout, raw, nsamps, out, s.cuda_stream))
    static_out = out.cpu().numpy().reshape(layout.nchans, capacity)

    cleaner = RFICleaner(RfiConfig.quiet(), layout, 2.0)
    cleaner.execute_normalized_device(raw.data_ptr(), raw.numel(), nsamps, on_device=True)
    alloc_out = cleaner.download()
    return static_out, alloc_out


def test_static_scratch_matches_allocating_cleaner_twice():
    from frost_b200.config import BlockLayout, DataType
    lay = BlockLayout(1024, 65536, DataType.UINT8, 64e-6, 1500.0, -0.29296875)
    for seed in (1, 2):  # two calls in a row: stale scratch must not leak
        mine, theirs = _run_both(lay, _blocks(1024, 65536, seed, "uint8"))
        assert mine.shape == theirs.shape
        assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32)), seed
        assert not mine[1024 - 1 - 5].any()  # dead channel (flipped order) zeroed


def test_static_scratch_calls_after_the_first_allocate_nothing():
    """After the first call on the device, repeated calls leave the device's
    free memory (cudaMemGetInfo) exactly as it was."""
    import torch

    from frost_b200 import _lib
    from frost_b200.config import BlockLayout, DataType
    lay = BlockLayout(512, 32768, DataType.UINT8, 64e-6, 1500.0, -0.5)
    raw = torch.from_numpy(_blocks(512, 32768, 7, "uint8").reshape(-1)).cuda()
    out = torch.empty(512 * 32768, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    _lib.check(_static(lay, raw, 0, out, s.cuda_stream))  # start-up call
    torch.cuda.synchronize()
    first = out.clone()  # torch allocates here, before the free-memory reading
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        _lib.check(_static(lay, raw, 0, out, s.cuda_stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.equal(out.view(torch.int32), first.view(torch.int32))


def test_static_scratch_float_partial_block():
    from frost_b200.config import BlockLayout, DataType
    lay = BlockLayout(256, 8192, DataType.FLOAT32, 1e-3, 800.0, 1.0)
    for nsamps in (0, 5000):
        mine, theirs = _run_both(lay, _blocks(256, 8192, 3, "float32"), nsamps)
        assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32)), nsamps


def test_static_scratch_refuses_oversize_and_short_blocks():
    import torch

    from frost_b200 import _lib
    from frost_b200.config import BlockLayout, DataType
    L = _lib.lib()
    s = torch.cuda.Stream()
    big = BlockLayout(4096, 65536, DataType.UINT8, 64e-6, 1500.0, -0.1)  # 2 windows x 4096 > 2684
    raw = torch.zeros(4096 * 65536, dtype=torch.uint8, device="cuda")
    out = torch.empty(4096 * 65536, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    lay = big.to_c()
    rc = L.frost_rfi_normalize_static(C.byref(lay), C.c_float(2.0), C.c_void_p(raw.data_ptr()),
                                      raw.numel(), 0, C.c_void_p(out.data_ptr()), out.numel(),
                                      C.c_void_p(s.cuda_stream))
    assert rc == -1 and "static scratch" in L.frost_last_error().decode()
    small = BlockLayout(64, 4096, DataType.UINT8, 1e-3, 1500.0, -1.0)
    lay = small.to_c()
    rc = L.frost_rfi_normalize_static(C.byref(lay), C.c_float(2.0), C.c_void_p(raw.data_ptr()),
                                      64 * 4096, 40, C.c_void_p(out.data_ptr()), out.numel(),
                                      C.c_void_p(s.cuda_stream))
    assert rc == -1 and "at least 64" in L.frost_last_error().decode()
    rc = L.frost_rfi_normalize_static(C.byref(lay), C.c_float(2.0), C.c_void_p(raw.data_ptr()),
                                      64 * 4096, 0, C.c_void_p(out.data_ptr()), out.numel(), None)
    assert rc == -1 and "null stream" in L.frost_last_error().decode()
    f32 = BlockLayout(64, 4096, DataType.FLOAT32, 1e-3, 1500.0, -1.0)
    lay = f32.to_c()
    rc = L.frost_rfi_normalize_static(C.byref(lay), C.c_float(2.0), C.c_void_p(raw.data_ptr() + 2),
                                      64 * 4096 * 4, 0, C.c_void_p(out.data_ptr()), out.numel(),
                                      C.c_void_p(s.cuda_stream))
    assert rc == -1 and "aligned" in L.frost_last_error().decode()
