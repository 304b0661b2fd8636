"""Single-AC-group frames on the GPU (encoders created with
CUJPEGXL_B200_ENCODER_SINGLE_GROUP): the combined-section file is
bit-identical to the CPU restatement's (itself pinned to the reference's
single-group writer), decodes to its planes, and works with learned
decisions and through configure."""

from __future__ import annotations

import numpy as np
import pytest

from cujpegxl_b200 import SINGLE_GROUP, Encoder
from cujpegxl_b200.decode import decode_planes
from cujpegxl_b200.synth import make_nv12
from oracle import api

from .gpu_util import device_nv12

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h", [(8, 8), (16, 16), (128, 96), (248, 56), (200, 136), (256, 256)])
@pytest.mark.parametrize("d", [0.5, 1.0, 4.0])
def test_single_group_file_bit_exact(w, h, d):
    nv = make_nv12(w, h, w * 7 + h)
    keep, luma, chroma, lp, cp = device_nv12(nv, w, h)
    with Encoder(w, h, d, flags=SINGLE_GROUP) as enc:
        data = enc.encode_device(luma, chroma, lp, cp)
        planes = enc.read_planes()
    assert data == api.encode(nv, w, h, d)
    got = decode_planes(data)
    for k in ("acs", "dc", "ac"):
        np.testing.assert_array_equal(got[k], planes[k], err_msg=k)


def test_configure_between_single_and_multi_group():
    nv_s = make_nv12(256, 128, 1)
    nv_m = make_nv12(264, 264, 2)
    with Encoder(256, 128, 1.0, flags=SINGLE_GROUP) as enc:
        a = enc.encode_host(nv_s)
        enc.configure(264, 264, 1.0)
        b = enc.encode_host(nv_m)
        enc.configure(256, 128, 1.0)
        c = enc.encode_host(nv_s)
    assert a == c == api.encode(nv_s, 256, 128, 1.0)
    assert b == api.encode(nv_m, 264, 264, 1.0)


def test_single_group_with_learned_decisions():
    from cujpegxl_b200.acsnet import QF, SPLIT, AcsNet
    w, h = 256, 256
    nv = make_nv12(w, h, 9)
    net = AcsNet.load()
    with Encoder(w, h, 1.0, flags=SINGLE_GROUP) as enc:
        enc.set_acsnet(net, 0.2, SPLIT | QF)
        data = enc.encode_host(nv)
        planes = enc.read_planes()
        decided, regions = enc.acsnet_stats()
        enc.set_acsnet(None)
    net.close()
    assert regions == 64 and decided > 0
    got = decode_planes(data)
    np.testing.assert_array_equal(got["acs"], planes["acs"])
    np.testing.assert_array_equal(got["ac"], planes["ac"])
