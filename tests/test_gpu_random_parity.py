"""The CUDA path against the restatement on seeded random geometries,
distances and row pitches: narrow and tall frames, partial tiles and groups,
distances from 0.1 (token-pool overflow) to 8. Every file must be equal byte
for byte."""

from __future__ import annotations

import random

import pytest

from cujpegxl_b200 import Encoder
from cujpegxl_b200.synth import make_nv12
from oracle import api

from .gpu_util import device_nv12

pytestmark = pytest.mark.gpu

_rng = random.Random(20261204)
CASES = []
for _i in range(24):
    _w = _rng.choice([64, 72, 128, 200, 264, 328, 512, 640, 1000, 1280, 1920, 2048, 2560])
    _h = _rng.choice([64, 80, 136, 256, 264, 392, 480, 720, 1080, 1440])
    if _w < 264 and _h < 264:  # one AC group needs the single-group mode
        _w = 264
    CASES.append((_w, _h, _rng.choice([0.1, 0.3, 0.5, 0.8, 1.0, 1.5, 2.0, 3.0, 5.0, 8.0]),
                  _rng.choice([0, 0, 16, 64]), 1000 + _i))


@pytest.mark.parametrize("w,h,d,pad,seed", CASES)
def test_random_geometry_file_bit_exact(w, h, d, pad, seed):
    nv = make_nv12(w, h, seed)
    keep, luma, chroma, lp, cp = device_nv12(nv, w, h, w + pad, w + pad)
    with Encoder(w, h, d) as enc:
        data = enc.encode_device(luma, chroma, lp, cp)
    assert data == api.encode(nv, w, h, d)
