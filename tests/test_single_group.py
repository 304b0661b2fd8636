"""Frames of a single 256x256 AC group (the reference's production path
rejects them): the combined-section layout of the CPU restatement against the
reference's own single-group codestream writer, decoder round trips, and the
library's options for accepting such frames."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cujpegxl_b200 import SINGLE_GROUP, _capi, max_output_size
from cujpegxl_b200.decode import decode, decode_planes, psnr_y
from cujpegxl_b200.synth import make_nv12
from oracle import api

SIZES = [(8, 8), (128, 96), (248, 56), (200, 136), (256, 256)]


def _tools_codestream(r, d: float, rqf: int) -> bytes:
    """tools/bitstream/vardct_frame.cc:666-677 (write_vardct_codestream) on the
    same quantised planes with a uniform quant field."""
    s = api.scalars(d)
    ac32 = r.ac.astype(np.int32)
    out = np.zeros(1 << 22, np.uint8)
    n = api.ref().ref_write_codestream(r.width, r.height, api._ptr(ac32), api._ptr(r.dc), api._ptr(r.acs),
                                       api._ptr(r.ytox), api._ptr(r.ytob), s["global_scale"], s["quant_dc"], rqf,
                                       api._ptr(out), out.size)
    return out[:n].tobytes()


@pytest.mark.skipif(not api.ref_available(), reason="reference-built checker not present")
@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("d", [0.5, 1.0, 3.0])
def test_combined_section_matches_reference_writer(w, h, d):
    r = api.frontend(make_nv12(w, h, w + h), w, h, d)
    q = int(np.median(r.qf))
    r.qf[:] = q
    mine = api.assemble(r, d)
    box = mine.find(b"jxlc")
    assert mine[box + 4:] == _tools_codestream(r, d, q)


@pytest.mark.parametrize("w,h", SIZES)
def test_combined_section_round_trips(w, h):
    nv = make_nv12(w, h, 3)
    o = api.frontend(nv, w, h, 1.0)
    data = api.encode(nv, w, h, 1.0)
    got = decode_planes(data)
    for k in ("acs", "dc", "ytox", "ytob", "ac"):
        np.testing.assert_array_equal(got[k], getattr(o, k).ravel(), err_msg=k)
    first = o.acs.ravel() != 0
    np.testing.assert_array_equal(got["qf"][first], o.qf.ravel()[first])
    assert decode(data).width == w
    if w * h >= 128 * 96:
        assert psnr_y(nv, data) > 32.0


def test_library_options():
    L = _capi.lib()
    enc = ctypes.c_void_p()
    small = _capi.Config(128, 96, 1.0, 0)
    assert L.cujpegxl_encoder_create(ctypes.byref(small), ctypes.byref(enc)) == _capi.UNSUPPORTED_RESOLUTION
    assert L.cujpegxl_b200_encoder_create_ex(ctypes.byref(small), 0, ctypes.byref(enc)) == \
        _capi.UNSUPPORTED_RESOLUTION
    assert L.cujpegxl_b200_encoder_create_ex(ctypes.byref(small), 6, ctypes.byref(enc)) == _capi.INVALID_ARGUMENT
    size = ctypes.c_size_t(0)
    assert L.cujpegxl_max_output_size(ctypes.byref(small), ctypes.byref(size)) == _capi.UNSUPPORTED_RESOLUTION
    assert max_output_size(128, 96, flags=SINGLE_GROUP) > 0
    assert max_output_size(264, 264) == max_output_size(264, 264, flags=SINGLE_GROUP)
    bad = _capi.Config(120, 100, 1.0, 0)
    assert L.cujpegxl_b200_encoder_create_ex(ctypes.byref(bad), SINGLE_GROUP, ctypes.byref(enc)) == \
        _capi.UNSUPPORTED_RESOLUTION
