"""Error paths of the drop-in C ABI on a device.

* cujpegxl_encoder_encode into a 16-byte host buffer returns
  CUJPEGXL_BUFFER_TOO_SMALL with `size` set to the file's length, and a second
  call with that capacity returns the same file as an ample buffer (the
  reference's src/cujpegxl_encode_gpu_test.cc:128-146).
* An allocation that fails while cujpegxl_encoder_create acquires its stream,
  device arena or pinned staging buffer gives CUJPEGXL_INTERNAL_ERROR, no
  encoder, and no leaked resource; the next create succeeds.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cujpegxl_b200 import Encoder, _capi
from cujpegxl_b200.synth import make_nv12

from .gpu_util import device_nv12

pytestmark = pytest.mark.gpu


def test_encode_into_small_buffer_reports_required_size():
    w, h = 512, 384
    nv = make_nv12(w, h, 5)
    keep, luma, chroma, lp, cp = device_nv12(nv, w, h)
    L = _capi.lib()
    with Encoder(w, h, 1.0) as enc:
        full = enc.encode_device(luma, chroma, lp, cp)
        small = np.zeros(16, np.uint8)
        inp = _capi.Nv12Input(luma, chroma, lp, cp)
        out = _capi.Output(small.ctypes.data, 0, small.size)
        code = L.cujpegxl_encoder_encode(enc.handle, ctypes.byref(inp), ctypes.byref(out))
        assert code == _capi.BUFFER_TOO_SMALL
        assert out.size == len(full)
        assert not small.any(), "nothing may be written into a buffer that is too small"
        exact = np.zeros(out.size, np.uint8)
        out2 = _capi.Output(exact.ctypes.data, 0, exact.size)
        assert L.cujpegxl_encoder_encode(enc.handle, ctypes.byref(inp), ctypes.byref(out2)) == _capi.OK
        assert out2.size == len(full) and exact.tobytes() == full


def test_failed_allocation_at_create_is_reported_and_leaks_nothing():
    import torch

    L = _capi.lib()
    cfg = _capi.Config(1280, 720, 1.0, 0)
    torch.cuda.synchronize()
    live0 = L.cujpegxl_b200_debug_live_allocations()
    free0 = torch.cuda.mem_get_info()[0]
    try:
        # create acquires a stream, the device arena and the pinned staging
        # buffer: fail each in turn.
        for nth in (1, 2, 3):
            L.cujpegxl_b200_debug_fail_allocation(nth)
            h = ctypes.c_void_p(None)
            code = L.cujpegxl_encoder_create(ctypes.byref(cfg), ctypes.byref(h))
            assert code == _capi.INTERNAL_ERROR, (nth, _capi.status_string(code))
            assert not h.value
            assert L.cujpegxl_b200_debug_live_allocations() == live0, nth
    finally:
        L.cujpegxl_b200_debug_fail_allocation(0)
    torch.cuda.synchronize()
    # No device memory held by the failed attempts (allow for driver slack).
    assert torch.cuda.mem_get_info()[0] >= free0 - (8 << 20)
    h = ctypes.c_void_p(None)
    assert L.cujpegxl_encoder_create(ctypes.byref(cfg), ctypes.byref(h)) == _capi.OK
    assert L.cujpegxl_b200_debug_live_allocations() == live0 + 3
    L.cujpegxl_encoder_destroy(h)
    assert L.cujpegxl_b200_debug_live_allocations() == live0


def test_failed_allocation_at_configure_keeps_encoder_usable():
    w, h = 512, 384
    nv = make_nv12(w, h, 6)
    keep, luma, chroma, lp, cp = device_nv12(nv, w, h)
    L = _capi.lib()
    with Encoder(1280, 720, 1.0) as enc:
        live = L.cujpegxl_b200_debug_live_allocations()
        L.cujpegxl_b200_debug_fail_allocation(1)  # the new geometry's arena
        try:
            cfg = _capi.Config(w, h, 1.0, 0)
            assert L.cujpegxl_encoder_configure(enc.handle, ctypes.byref(cfg)) == _capi.INTERNAL_ERROR
        finally:
            L.cujpegxl_b200_debug_fail_allocation(0)
        assert L.cujpegxl_b200_debug_live_allocations() == live - 2  # old arena and pinned buffer released
        enc.configure(w, h, 1.0)
        with Encoder(w, h, 1.0) as ref:
            assert enc.encode_device(luma, chroma, lp, cp) == ref.encode_device(luma, chroma, lp, cp)


def test_page_locked_output_takes_the_one_wait_path():
    """cujpegxl_encoder_encode into page-locked memory (the device-side copy
    behind the encode) gives the same file as into pageable memory, and the
    same BUFFER_TOO_SMALL answer for a 16-byte page-locked buffer."""
    import torch

    w, h = 1280, 720
    nv = make_nv12(w, h, 8)
    keep, luma, chroma, lp, cp = device_nv12(nv, w, h)
    L = _capi.lib()
    inp = _capi.Nv12Input(luma, chroma, lp, cp)
    with Encoder(w, h, 1.0) as enc:
        pageable = enc.encode_device(luma, chroma, lp, cp)
        for offset in (0, 3):   # 16-byte aligned and unaligned destinations
            pinned = torch.zeros(len(pageable) + 64, dtype=torch.uint8).pin_memory()
            out = _capi.Output(pinned.data_ptr() + offset, 0, len(pageable))
            assert L.cujpegxl_encoder_encode(enc.handle, ctypes.byref(inp), ctypes.byref(out)) == _capi.OK
            assert out.size == len(pageable)
            got = pinned.numpy()
            assert got[offset:offset + out.size].tobytes() == pageable
            assert not got[:offset].any() and not got[offset + out.size:].any()
        tiny = torch.zeros(16, dtype=torch.uint8).pin_memory()
        out = _capi.Output(tiny.data_ptr(), 0, 16)
        assert L.cujpegxl_encoder_encode(enc.handle, ctypes.byref(inp), ctypes.byref(out)) == _capi.BUFFER_TOO_SMALL
        assert out.size == len(pageable) and not tiny.numpy().any()


def test_enqueue_readback_rejects_pageable_memory():
    w, h = 512, 384
    L = _capi.lib()
    with Encoder(w, h, 1.0) as enc:
        buf = np.zeros(1 << 16, np.uint8)
        words = np.zeros(2, np.uint64)
        code = L.cujpegxl_b200_encoder_enqueue_readback(enc.handle, buf.ctypes.data, buf.size, words.ctypes.data)
        assert code == _capi.INVALID_ARGUMENT
