"""The host subset decoder against files whose content is known: the
reference's own assemblies of its entropy-test patterns (golden fixtures) and
the CPU restatement's files. Decoding must recover the quantised planes
exactly (an encode -> decode round trip), every section must end where the TOC
says, and the reconstruction must be close to the encoder's input."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from cujpegxl_b200.decode import DecodeError, decode, decode_planes, psnr_y
from cujpegxl_b200.synth import make_nv12
from oracle import api

from . import patterns as P

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", ["dct8_512x384", "mixed_512x384", "mixed_qf_264x264"])
def test_reference_files_decode_to_their_planes(name):
    meta = json.loads((GOLD / "files.json").read_text())[name]
    data = np.load(GOLD / f"file_{name}.npy").tobytes()
    w, h = (int(v) for v in name.rsplit("_", 1)[1].split("x"))
    if name.startswith("dct8"):
        f = P.empty(w, h)
        P.fill_ac_pattern(f)
        P.fill_dc_pattern(f)
    else:
        f = P.mixed_full(w, h, seed=5 if "qf" in name else None)
    got = decode_planes(data)
    assert (got["width"], got["height"]) == (w, h)
    assert (got["global_scale"], got["quant_dc"]) == (meta["global_scale"], meta["quant_dc"])
    flat = P.flat(f)
    first = flat["acs"] != 0
    np.testing.assert_array_equal(got["acs"], flat["acs"])
    np.testing.assert_array_equal(got["qf"][first], flat["qf"][first])
    np.testing.assert_array_equal(got["dc"], flat["dc"])
    np.testing.assert_array_equal(got["ytox"], flat["ytox"])
    np.testing.assert_array_equal(got["ytob"], flat["ytob"])
    # The LLF corner of a DCT16/32 is carried by the DC, not coded as AC: the
    # pattern's values there are not part of the file.
    expected = flat["ac"].copy()
    bw = w // 8
    for blk in np.flatnonzero(flat["acs"] > 8):
        n = int(flat["acs"][blk])
        m = n // 8
        for c in range(3):
            for fx in range(m):
                for fy in range(m):
                    slot = P.covered_slot(n, blk % bw, blk // bw, bw, fx * n + fy)
                    expected[c * (w // 8) * (h // 8) * 64 + slot] = 0
    np.testing.assert_array_equal(got["ac"], expected)


@pytest.mark.parametrize("w,h,d,seed", [(512, 384, 1.0, 0), (520, 392, 2.0, 2), (264, 264, 4.0, 1)])
def test_encoded_frames_round_trip_and_reconstruct(w, h, d, seed):
    nv = make_nv12(w, h, seed)
    o = api.frontend(nv, w, h, d, debug=True)
    data = api.encode(nv, w, h, d)
    got = decode_planes(data)
    for k in ("acs", "dc", "ytox", "ytob", "ac"):
        np.testing.assert_array_equal(got[k], getattr(o, k).ravel(), err_msg=k)
    first = o.acs.ravel() != 0
    np.testing.assert_array_equal(got["qf"][first], o.qf.ravel()[first])
    img = decode(data)
    ref = o.xyb.reshape(3, h, w)
    rms_y = float(np.sqrt(np.mean((img.xyb[1] - ref[1]) ** 2)))
    assert rms_y < 0.02, rms_y       # Y spans ~0..0.85
    assert psnr_y(nv, data) > 32.0


def test_quality_falls_with_distance():
    w, h = 512, 384
    nv = make_nv12(w, h, 4)
    psnr = [psnr_y(nv, api.encode(nv, w, h, d)) for d in (0.5, 1.0, 2.0, 4.0)]
    assert all(a > b for a, b in zip(psnr, psnr[1:])), psnr


def test_malformed_files_are_reported():
    w, h = 512, 384
    data = bytearray(api.encode(make_nv12(w, h, 0), w, h, 1.0))
    with pytest.raises(DecodeError):
        decode(bytes(data[: len(data) // 2]))
    with pytest.raises(DecodeError):
        decode(b"not a jxl file at all")
