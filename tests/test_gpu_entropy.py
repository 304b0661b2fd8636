"""Device entropy coding and assembly vs the CPU restatement and (when built)
the reference's own host code, on the reference's entropy test patterns,
through cujpegxl_b200_encode_planes. Byte-exact, including partial AC and DC
groups (the reference's 2560x2304 case) and a random per-block quant field.
"""

from __future__ import annotations

import numpy as np
import pytest

from cujpegxl_b200 import Encoder
from oracle import api

from . import patterns as P

pytestmark = pytest.mark.gpu


def _oracle_file(f: dict, gs: int, qdc: int) -> bytes:
    r = api.FrontendResult(f["w"], f["h"])
    for k, v in P.flat(f).items():
        getattr(r, k)[...] = v
    n = api.oracle().oracle_assemble(f["w"], f["h"], r.ac.ctypes.data, r.dc.ctypes.data, r.acs.ctypes.data,
                                     r.qf.ctypes.data, r.ytox.ctypes.data, r.ytob.ctypes.data, gs, qdc,
                                     None, 0)
    out = np.zeros(n, np.uint8)
    api.oracle().oracle_assemble(f["w"], f["h"], r.ac.ctypes.data, r.dc.ctypes.data, r.acs.ctypes.data,
                                 r.qf.ctypes.data, r.ytox.ctypes.data, r.ytob.ctypes.data, gs, qdc,
                                 out.ctypes.data, n)
    if api.ref_available():
        ac32 = r.ac.astype(np.int32)
        ref = np.zeros(n + 4096, np.uint8)
        m = api.ref().ref_encode_frame(f["w"], f["h"], ac32.ctypes.data, r.dc.ctypes.data, r.acs.ctypes.data,
                                       r.ytox.ctypes.data, r.ytob.ctypes.data, r.qf.ctypes.data, gs, qdc,
                                       ref.ctypes.data, ref.size)
        assert out.tobytes() == ref[:m].tobytes(), "oracle disagrees with the reference"
    return out.tobytes()


def _device_file(f: dict, gs: int, qdc: int) -> bytes:
    with Encoder(f["w"], f["h"], 1.0) as enc:
        return enc.encode_planes(P.flat(f), gs, qdc)


def test_dct8_only_pattern():
    f = P.empty(512, 384)
    P.fill_ac_pattern(f)
    P.fill_dc_pattern(f)
    assert _device_file(f, 4096, 32) == _oracle_file(f, 4096, 32)


@pytest.mark.parametrize("w,h", [(512, 384), (2560, 256), (2560, 2304)])
def test_mixed_pattern(w, h):
    f = P.mixed_full(w, h)
    assert _device_file(f, 4096, 32) == _oracle_file(f, 4096, 32)


def test_random_quant_field_and_zero_frame():
    f = P.mixed_full(1024, 768, seed=7)
    assert _device_file(f, 9502, 64) == _oracle_file(f, 9502, 64)
    z = P.empty(512, 512)
    assert _device_file(z, 1, 1) == _oracle_file(z, 1, 1)


def test_large_magnitudes():
    f = P.empty(768, 512)
    rng = np.random.Generator(np.random.PCG64(3))
    f["ac"][:] = rng.integers(-20000, 20000, f["ac"].shape).astype(np.int16) * (rng.random(f["ac"].shape) < 0.05)
    f["dc"][:] = rng.integers(-(1 << 20), 1 << 20, f["dc"].shape)
    assert _device_file(f, 65536, 1) == _oracle_file(f, 65536, 1)
